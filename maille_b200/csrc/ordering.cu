// ordering.cu -- the ordering of the free nodes on the device (see ordering.cuh).
//
// Reference counterparts: Graph::from_elements (iterative.rs:38-76) builds the adjacency from the
// elements, reverse_cuthill_mckee and bfs_levels (solve.rs:200-270) order it. The host analysis
// (setup.cpp) runs the same algorithms sequentially on nodes; here each one is restated in a
// form whose result does not depend on the order the GPU's threads run in, so the device and the
// host produce the same permutation:
//  * graph: every element emits the (row, column) keys of its kept node pairs; a radix sort and a
//    unique pass give every node's neighbours by ascending index (the host sorts its lists too);
//  * breadth-first search, level by level in one cooperative launch: a node of the next level
//    takes as parent its neighbour of the current level that came first (the largest key of an
//    atomicMax over (search id, complement of the parent's position)), which is the node that
//    discovers it in a sequential search; children of one parent are placed by ascending index
//    (plain search) or by ascending (degree, index) (Cuthill-McKee: the stable sort by degree of
//    an index-ordered list), after their parents' children counts are scanned;
//  * greedy colouring in a visit order: the colour of a node is the smallest one its
//    earlier-visited neighbours do not hold. Warps take nodes in visit order on a fixed
//    round-robin schedule and wait (bounded) for the colours of those neighbours, so a node is
//    coloured exactly as the sequential loop colours it; the level of a row in the RCM ordering
//    (one more than the largest level of its earlier neighbours) is the same dataflow.

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdio>
#include <cstdlib>

#include <cooperative_groups.h>
#include <cub/cub.cuh>

#include "cuda_host.hpp"
#include "ordering.cuh"

namespace cg = cooperative_groups;

namespace maille {

extern std::atomic<long long> g_kernel_launches;

namespace {

constexpr int kT = 256;
constexpr int kW = kT / 32;
constexpr int32_t kVisited = INT_MAX;          // mark of a node an ordering search has placed
constexpr unsigned int kSpin = 1u << 22;       // polls of one neighbour value before a wait gives up
constexpr int kMaxColourWords = 32;            // colours below 32 x 32 = 1024

inline unsigned grid_of(int64_t n) {
    const int64_t g = (n + kT - 1) / kT;
    return (unsigned)(g < 1 ? 1 : (g > (1 << 20) ? (1 << 20) : g));
}
inline void counted(int n = 1) { g_kernel_launches.fetch_add(n, std::memory_order_relaxed); }

#define GRID_STRIDE(t, n) \
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < (n); t += (int64_t)gridDim.x * blockDim.x)

template <typename K>
__device__ __forceinline__ int64_t lower_bound_dev(const K* a, int64_t n, K key) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (a[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// (I << 32) | J for every ordered pair of distinct kept nodes of an element; ~0 otherwise
__global__ void k_graph_keys(int npe, int64_t ne, const int32_t* __restrict__ conn,
                             const int32_t* __restrict__ kept_of, uint64_t* __restrict__ keys) {
    const int64_t per = (int64_t)npe * (npe - 1);
    GRID_STRIDE(t, ne * per) {
        const int64_t e = t / per;
        const int rem = (int)(t - e * per);
        const int a = rem / (npe - 1), bi = rem % (npe - 1), b = bi < a ? bi : bi + 1;
        const int32_t I = kept_of[conn[e * npe + a]], J = kept_of[conn[e * npe + b]];
        keys[t] = (I < 0 || J < 0 || I == J) ? ~0ull : (((uint64_t)(uint32_t)I << 32) | (uint64_t)(uint32_t)J);
    }
}

// row pointers and degrees of the unique sorted keys (m valid keys, all below nk << 32)
__global__ void k_graph_csr(const uint64_t* __restrict__ keys, int64_t m, int32_t nk, int64_t* __restrict__ off,
                            int32_t* __restrict__ deg) {
    GRID_STRIDE(k, (int64_t)nk + 1) {
        const int64_t o = lower_bound_dev<uint64_t>(keys, m, (uint64_t)k << 32);
        off[k] = o;
        if (k < nk) deg[k] = (int32_t)(lower_bound_dev<uint64_t>(keys, m, (uint64_t)(k + 1) << 32) - o);
    }
}

__global__ void k_graph_adj(const uint64_t* __restrict__ keys, int64_t m, int32_t* __restrict__ adj) {
    GRID_STRIDE(p, m) adj[p] = (int32_t)(keys[p] & 0xFFFFFFFFull);
}

__device__ __forceinline__ void warp_min_atomic(unsigned long long b, unsigned long long* best) {
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long u = __shfl_xor_sync(0xffffffffu, b, o);
        b = u < b ? u : b;
    }
    if ((threadIdx.x & 31) == 0 && b != ~0ull) atomicMin(best, b);
}

// the first (by index) node of minimum degree among the nodes not ordered yet: min of (deg, index)
__global__ void k_seed(int32_t nk, const int32_t* __restrict__ deg, const int32_t* __restrict__ mark,
                       unsigned long long* __restrict__ best) {
    unsigned long long b = ~0ull;
    GRID_STRIDE(v, (int64_t)nk) {
        if (mark[v] != kVisited) {
            const unsigned long long k = ((unsigned long long)(uint32_t)deg[v] << 32) | (unsigned long long)v;
            b = k < b ? k : b;
        }
    }
    warp_min_atomic(b, best);
}

// the first (in discovery order) node of minimum degree of the positions [lb, le) of queue:
// min of (deg, position)
__global__ void k_far(int32_t lb, int32_t le, const int32_t* __restrict__ queue, const int32_t* __restrict__ deg,
                      unsigned long long* __restrict__ best) {
    unsigned long long b = ~0ull;
    GRID_STRIDE(t, (int64_t)(le - lb)) {
        const int32_t q = lb + (int32_t)t;
        const unsigned long long k = ((unsigned long long)(uint32_t)deg[queue[q]] << 32) | (unsigned long long)q;
        b = k < b ? k : b;
    }
    warp_min_atomic(b, best);
}

struct BfsArgs {
    int32_t nk;
    const int64_t* off;
    const int32_t* adj;
    const int32_t* deg;
    int32_t* mark;                 // id of the search that reached the node, or kVisited
    unsigned long long* par;       // (id << 32) | (~parent position): the largest is the first parent
    int32_t* queue;                // nodes by position
    int32_t* cnt;                  // per position: children count, then the children's first position
    int32_t* bsum;                 // [grid] per-block children totals
    int32_t id;                    // this search's id (> 0, increasing over the searches of a run)
    int32_t markval;               // mark written on discovery: id, or kVisited for an ordering search
    int32_t start, qbase;          // start node, its position
    int32_t by_degree;             // children by (degree, index) instead of index
    int32_t* out;                  // [0] levels, [1] queue end, [2] last level's first position
};

__device__ __forceinline__ bool unreached(int32_t m, int32_t id) { return m != id && m != kVisited; }

__device__ __forceinline__ unsigned long long parent_key(unsigned long long idk, int32_t pos) {
    return idk | (unsigned long long)(0xFFFFFFFFu - (uint32_t)pos);
}

// One breadth-first search from a.start, level by level, in one cooperative launch (three grid
// barriers a level): parents by atomicMax, children counts, a scan of the counts over the
// level's positions, placement. A node w is a child of v exactly when par[w] holds v's key: the
// key carries this search's id, and a node placed earlier kept the key of a parent of an earlier
// level. Out: levels, queue end, first position of the last level.
__global__ void __launch_bounds__(kT) k_bfs(BfsArgs a) {
    cg::grid_group grid = cg::this_grid();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const unsigned long long idk = (unsigned long long)(uint32_t)a.id << 32;
    __shared__ int32_t sh_sum[kW];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.queue[a.qbase] = a.start;
        a.mark[a.start] = a.markval;
    }
    int32_t lb = a.qbase, le = a.qbase + 1, levels = 1;
    grid.sync();
    for (;;) {
        const int32_t F = le - lb;
        // 1. every unreached neighbour of a level node keeps its first parent
        for (int64_t i = gw; i < F; i += nwarps) {
            const int32_t v = a.queue[lb + i];
            const unsigned long long key = parent_key(idk, lb + (int32_t)i);
            for (int64_t p = a.off[v] + lane; p < a.off[v + 1]; p += 32) {
                const int32_t w = a.adj[p];
                if (unreached(a.mark[w], a.id)) atomicMax(&a.par[w], key);
            }
        }
        grid.sync();
        // 2. children counts, block b owning the level positions [p0, p1)
        const int32_t chunk = (F + (int32_t)gridDim.x - 1) / (int32_t)gridDim.x;
        const int32_t p0 = min(F, (int32_t)blockIdx.x * chunk), p1 = min(F, p0 + chunk);
        int32_t mine = 0;
        for (int32_t i = p0 + wib; i < p1; i += kW) {
            const int32_t v = a.queue[lb + i];
            const unsigned long long key = parent_key(idk, lb + i);
            int32_t c = 0;
            for (int64_t q0 = a.off[v]; q0 < a.off[v + 1]; q0 += 32) {
                const int64_t p = q0 + lane;
                const bool child = p < a.off[v + 1] && a.par[a.adj[p]] == key;
                c += __popc(__ballot_sync(0xffffffffu, child));
            }
            if (lane == 0) a.cnt[lb + i] = c;
            mine += c;  // the same c in every lane
        }
        if (lane == 0) sh_sum[wib] = mine;
        __syncthreads();
        if (threadIdx.x == 0) {
            int32_t t = 0;
            for (int k = 0; k < kW; ++k) t += sh_sum[k];
            a.bsum[blockIdx.x] = t;
        }
        grid.sync();
        // 3. the level's total, this block's base, and the exclusive scan of its counts
        int32_t total = 0, base = 0;
        for (int k = lane; k < (int)gridDim.x; k += 32) {
            const int32_t s = a.bsum[k];
            total += s;
            base += k < (int)blockIdx.x ? s : 0;
        }
        total = __reduce_add_sync(0xffffffffu, total);
        base = __reduce_add_sync(0xffffffffu, base);
        if (wib == 0) {
            int32_t run = le + base;  // the next level starts at position le
            for (int32_t i0 = p0; i0 < p1; i0 += 32) {
                const int32_t i = i0 + lane;
                const int32_t c = i < p1 ? a.cnt[lb + i] : 0;
                int32_t incl = c;
                for (int o = 1; o < 32; o <<= 1) {
                    const int32_t u = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += u;
                }
                if (i < p1) a.cnt[lb + i] = run + incl - c;
                run += __shfl_sync(0xffffffffu, incl, 31);
            }
        }
        __syncthreads();
        // 4. placement of each level node's children from their first position
        for (int32_t i = p0 + wib; i < p1; i += kW) {
            const int32_t v = a.queue[lb + i];
            const unsigned long long key = parent_key(idk, lb + i);
            const int32_t first = a.cnt[lb + i];
            const int64_t b0 = a.off[v], b1 = a.off[v + 1];
            int32_t before = 0;  // children in the earlier adjacency chunks (index order)
            for (int64_t q0 = b0; q0 < b1; q0 += 32) {
                const int64_t p = q0 + lane;
                const int32_t w = p < b1 ? a.adj[p] : -1;
                const bool child = w >= 0 && a.par[w] == key;
                const unsigned int bal = __ballot_sync(0xffffffffu, child);
                int32_t rank = before + __popc(bal & ((1u << lane) - 1u));
                if (a.by_degree) {
                    // rank by (degree, index) among all children of v: the children of every
                    // adjacency chunk with a smaller key
                    const unsigned long long mk =
                        child ? (((unsigned long long)(uint32_t)a.deg[w] << 32) | (unsigned long long)(uint32_t)w) : 0ull;
                    rank = 0;
                    for (int64_t r0 = b0; r0 < b1; r0 += 32) {
                        const int64_t rp = r0 + lane;
                        const int32_t u = rp < b1 ? a.adj[rp] : -1;
                        const bool uc = u >= 0 && a.par[u] == key;
                        const unsigned long long uk =
                            uc ? (((unsigned long long)(uint32_t)a.deg[u] << 32) | (unsigned long long)(uint32_t)u) : ~0ull;
                        for (int s = 0; s < 32; ++s) {
                            const unsigned long long ok = __shfl_sync(0xffffffffu, uk, s);
                            rank += (child && ok < mk) ? 1 : 0;
                        }
                    }
                }
                if (child) {
                    a.queue[first + rank] = w;
                    a.mark[w] = a.markval;
                }
                before += __popc(bal);
            }
        }
        grid.sync();
        if (total == 0) break;
        lb = le;
        le += total;
        ++levels;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.out[0] = levels;
        a.out[1] = le;
        a.out[2] = lb;
    }
}

__device__ __forceinline__ int32_t ld_val(const int32_t* p) {
    int32_t v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_val(int32_t* p, int32_t v) {
    asm volatile("st.relaxed.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Greedy colouring (mode 0) or dependency levels (mode 1) of the nodes in visit order: visit[q]
// is the node at visit position q, rpos its inverse. Warps claim visit positions in increasing
// order from a counter (*next, 0 at launch); for the node at position q a warp waits for the
// values of its neighbours of smaller visit position and sets the smallest colour none of them
// holds (mode 0) or one more than their largest level (mode 1). The smallest unfinished position
// was claimed by a warp that waits only on smaller, finished positions, so the launch always
// progresses (every warp is co-resident); a warp stuck behind a slow node does not hold up the
// positions after it, as a fixed schedule would. Values start at -1. *fail is set when a wait
// ran out or a colour reached 1024.
// Folds the neighbour values of one pass into the node's state: lane j of `words` collects the
// colours 32 j .. 32 j + 31 (mode 0), `top` the largest level (mode 1). c < 0: no value.
template <int N>
__device__ __forceinline__ void fold_values(const int32_t (&c)[N], int mode, int lane, unsigned int& words,
                                            int32_t& top, bool& bad) {
    int32_t cm = -1;
#pragma unroll
    for (int j = 0; j < N; ++j) cm = max(cm, c[j]);
    const int32_t cmax = __reduce_max_sync(0xffffffffu, cm);
    if (mode != 0) {
        top = max(top, cmax);
        return;
    }
    if (cm >= kMaxColourWords * 32) bad = true;
    for (int w = 0; w < kMaxColourWords && w * 32 <= cmax; ++w) {
        unsigned int bit = 0u;
#pragma unroll
        for (int j = 0; j < N; ++j)
            if (c[j] >= 0 && (c[j] >> 5) == w) bit |= 1u << (c[j] & 31);
        const unsigned int word = __reduce_or_sync(0xffffffffu, bit);
        if (lane == w) words |= word;
    }
}

// Waits for the pending entries of c (earlier neighbours whose value is still -1), polling them
// together with a growing pause: thousands of warps wait on the same few nodes of the frontier,
// and back-to-back polls of those lines slow down the stores they wait for. Returns false when
// the wait ran out.
template <int N>
__device__ __forceinline__ bool await_values(const int32_t* value, const int32_t (&u)[N], const bool (&early)[N],
                                             int32_t (&c)[N], unsigned int pause0, unsigned int pause_cap) {
    bool pend = false;
#pragma unroll
    for (int j = 0; j < N; ++j) pend = pend || (early[j] && c[j] < 0);
    unsigned int k = 0, pause = pause0;
    while (pend && k < kSpin) {
        if (pause_cap) __nanosleep(pause);
        pause = pause < pause_cap ? 2 * pause : pause_cap;
        ++k;
        pend = false;
#pragma unroll
        for (int j = 0; j < N; ++j)
            if (early[j] && c[j] < 0) {
                c[j] = ld_val(value + u[j]);
                pend = pend || c[j] < 0;
            }
    }
    return !pend;
}

constexpr int kGreedyChunks = 4;  // neighbour lists of up to 4 x 32 entries are held in registers
// Pause between polls of a pending neighbour, in ns: starts at kGreedyPause0 and doubles up to
// kGreedyPauseCap (0: no pause). Passed as launch arguments: that form of the poll loop colours
// the Tet10 40^3 nodes in 6.7 ms, the same loop with the bounds as literals in 10 ms.
constexpr unsigned int kGreedyPause0 = 16, kGreedyPauseCap = 64;

__global__ void __launch_bounds__(kT) k_greedy(int32_t nk, const int64_t* __restrict__ off,
                                               const int32_t* __restrict__ adj, const int32_t* __restrict__ visit,
                                               const int32_t* __restrict__ rpos, int32_t* value, int mode,
                                               int32_t* fail, int32_t* next, unsigned int pause0,
                                               unsigned int pause_cap) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        int32_t qq = 0;
        if (lane == 0) qq = atomicAdd(next, 1);
        const int64_t q = __shfl_sync(0xffffffffu, qq, 0);
        if (q >= nk) break;
        const int32_t v = visit[q];
        const int64_t b = off[v], e = off[v + 1];
        unsigned int words = 0;  // lane j: colours 32 j .. 32 j + 31 held by earlier neighbours
        int32_t top = -1;         // mode 1: largest level of an earlier neighbour
        bool bad = false;
        if (e - b <= 32 * kGreedyChunks) {
            // the whole list at once: its index loads, then its value loads, are issued together,
            // so a node that became ready is finished after one round of polls
            int32_t u[kGreedyChunks], c[kGreedyChunks];
            bool early[kGreedyChunks];
#pragma unroll
            for (int j = 0; j < kGreedyChunks; ++j) {
                const int64_t p = b + 32 * j + lane;
                u[j] = p < e ? adj[p] : -1;
            }
#pragma unroll
            for (int j = 0; j < kGreedyChunks; ++j) early[j] = u[j] >= 0 && rpos[u[j]] < q;
#pragma unroll
            for (int j = 0; j < kGreedyChunks; ++j) c[j] = early[j] ? ld_val(value + u[j]) : -1;
            if (!await_values(value, u, early, c, pause0, pause_cap)) bad = true;
            fold_values(c, mode, lane, words, top, bad);
        } else {
            for (int64_t p0 = b; p0 < e; p0 += 32) {
                const int64_t p = p0 + lane;
                int32_t u[1] = {-1}, c[1] = {-1};
                bool early[1] = {false};
                if (p < e) {
                    u[0] = adj[p];
                    early[0] = rpos[u[0]] < q;
                    if (early[0]) c[0] = ld_val(value + u[0]);
                }
                if (!await_values(value, u, early, c, pause0, pause_cap)) bad = true;
                fold_values(c, mode, lane, words, top, bad);
            }
        }
        bad = __any_sync(0xffffffffu, bad);
        int32_t result;
        if (mode == 0) {
            const unsigned int freebits = ~words;
            const unsigned int has = __ballot_sync(0xffffffffu, freebits != 0u);
            const int j = __ffs(has) - 1;
            const unsigned int fw = __shfl_sync(0xffffffffu, freebits, j < 0 ? 0 : j);
            result = j < 0 ? 0 : 32 * j + __ffs(fw) - 1;
            if (j < 0) bad = true;
        } else {
            result = top + 1;
        }
        if (lane == 0) {
            if (bad) atomicExch(fail, 1);
            st_val(value + v, bad ? 0 : result);  // a failed node still unblocks the later ones
        }
        __syncwarp();
    }
}

// visit position q holds queue position nk - 1 - q (the reversed search order); rpos inverts it
__global__ void k_reverse(int32_t nk, const int32_t* __restrict__ queue, int32_t* __restrict__ visit,
                          int32_t* __restrict__ rpos) {
    GRID_STRIDE(q, (int64_t)nk) {
        const int32_t v = queue[nk - 1 - q];
        visit[q] = v;
        rpos[v] = (int32_t)q;
    }
}

__global__ void k_order_keys(int32_t nk, const int32_t* __restrict__ value, const int32_t* __restrict__ rpos,
                             uint64_t* __restrict__ keys, int32_t* __restrict__ ids) {
    GRID_STRIDE(v, (int64_t)nk) {
        keys[v] = ((uint64_t)(uint32_t)value[v] << 32) | (uint64_t)(uint32_t)rpos[v];
        ids[v] = (int32_t)v;
    }
}

// visit keys of an iterated-greedy pass: classes from the last to the first, RCM position inside
__global__ void k_class_keys(int32_t nk, int32_t top, const int32_t* __restrict__ value,
                             const int32_t* __restrict__ rpos, uint64_t* __restrict__ keys, int32_t* __restrict__ ids) {
    GRID_STRIDE(v, (int64_t)nk) {
        keys[v] = ((uint64_t)(uint32_t)(top - value[v]) << 32) | (uint64_t)(uint32_t)rpos[v];
        ids[v] = (int32_t)v;
    }
}

// rpos of a visit order given as an array of nodes
__global__ void k_inverse(int32_t nk, const int32_t* __restrict__ visit, int32_t* __restrict__ rpos) {
    GRID_STRIDE(q, (int64_t)nk) rpos[visit[q]] = (int32_t)q;
}

__global__ void k_fill_i32(int64_t n, int32_t v, int32_t* __restrict__ a) {
    GRID_STRIDE(i, n) a[i] = v;
}

template <typename T>
struct Buf {
    T* p = nullptr;
    explicit Buf(size_t n) : p(dalloc<T>(n)) {}
    ~Buf() { dfree(p); }
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
};

struct Temp {
    void* p = nullptr;
    size_t bytes = 0;
    void reserve(size_t n) {
        if (n <= bytes) return;
        dfree(p);
        p = dalloc<unsigned char>(n);
        bytes = n;
    }
    ~Temp() { dfree(p); }
};

__global__ void k_narrow(int64_t n, const int64_t* __restrict__ in, int32_t* __restrict__ out) {
    GRID_STRIDE(k, n) out[k] = (int32_t)in[k];
}

__global__ void k_iota(int64_t n, int32_t* __restrict__ out) {
    GRID_STRIDE(k, n) out[k] = (int32_t)k;
}

// ptr[v] = first position of key v in the sorted keys (n_nodes + 1 entries)
__global__ void k_run_starts(int64_t n_nodes, const uint32_t* __restrict__ keys, int64_t n,
                             int64_t* __restrict__ ptr) {
    GRID_STRIDE(v, n_nodes + 1) ptr[v] = lower_bound_dev<uint32_t>(keys, n, (uint32_t)v);
}

__global__ void k_zero_free(int64_t n, const uint8_t* __restrict__ fixed, double* __restrict__ v) {
    GRID_STRIDE(k, n) if (!fixed[k]) v[k] = 0.0;
}

// blocks of a cooperative launch of fn: every block co-resident
int coop_grid(const void* fn, int threads) {
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, 0));
    const int g = per_sm * device_sms();
    if (g <= 0) throw CudaFailure{"the ordering kernels cannot be made co-resident on this device"};
    return g;
}

}  // namespace

void gpu_ordering(int npe, int64_t n_elems, const int32_t* conn, const int32_t* kept_of, int32_t nk,
                  int ordering, cudaStream_t st, std::vector<int32_t>& order, std::vector<int32_t>& level) {
    if (nk <= 0) throw CudaFailure{"no kept node to order"};
    // MAILLE_SETUP_TIMING: wall time of each step (stream synchronised)
    const bool timing = std::getenv("MAILLE_SETUP_TIMING") != nullptr;
    double t_mark = now_ms();
    auto tmark = [&](const char* name, int extra = -1) {
        if (!timing) return;
        cudaStreamSynchronize(st);
        const double t = now_ms();
        std::fprintf(stderr, "maille ordering %-16s %8.2f ms %d\n", name, t - t_mark, extra);
        t_mark = t;
    };
    // the kept-node graph, neighbours by ascending index
    const int64_t nkeys = n_elems * npe * (npe - 1);
    if (nkeys >= INT_MAX || nkeys <= 0) throw CudaFailure{"mesh size outside the device ordering's range"};
    Temp temp;
    Buf<int64_t> off((size_t)nk + 1);
    Buf<int32_t> deg(nk);
    int64_t m = 0;
    int32_t* adj = nullptr;
    {
        Buf<uint64_t> ka(nkeys), kb(nkeys), uk(nkeys);
        Buf<int> nsel(1);
        counted();
        k_graph_keys<<<grid_of(nkeys), kT, 0, st>>>(npe, n_elems, conn, kept_of, ka.p);
        CK(cudaGetLastError());
        cub::DoubleBuffer<uint64_t> db(ka.p, kb.p);
        size_t bytes = 0;
        CK(cub::DeviceRadixSort::SortKeys(nullptr, bytes, db, (int)nkeys, 0, 64, st));
        temp.reserve(bytes);
        CK(cub::DeviceRadixSort::SortKeys(temp.p, bytes, db, (int)nkeys, 0, 64, st));
        bytes = 0;
        CK(cub::DeviceSelect::Unique(nullptr, bytes, db.Current(), uk.p, nsel.p, (int)nkeys, st));
        temp.reserve(bytes);
        CK(cub::DeviceSelect::Unique(temp.p, bytes, db.Current(), uk.p, nsel.p, (int)nkeys, st));
        counted(2);
        int n = 0;
        CK(cudaMemcpyAsync(&n, nsel.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        uint64_t last = 0;
        if (n > 0) CK(cudaMemcpy(&last, uk.p + (n - 1), sizeof(uint64_t), cudaMemcpyDeviceToHost));
        m = (n > 0 && last == ~0ull) ? n - 1 : n;
        adj = dalloc<int32_t>((size_t)std::max<int64_t>(1, m));
        counted(2);
        k_graph_csr<<<grid_of((int64_t)nk + 1), kT, 0, st>>>(uk.p, m, nk, off.p, deg.p);
        k_graph_adj<<<grid_of(std::max<int64_t>(1, m)), kT, 0, st>>>(uk.p, m, adj);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));  // the key buffers are freed below
    }
    struct AdjFree {
        int32_t* p;
        ~AdjFree() { dfree(p); }
    } adj_free{adj};
    tmark("graph", (int)m);

    Buf<int32_t> mark(nk), queue(nk), cnt(nk), out(4);
    Buf<unsigned long long> par(nk), best(1);
    counted();
    k_fill_i32<<<grid_of(nk), kT, 0, st>>>(nk, 0, mark.p);
    CK(cudaMemsetAsync(par.p, 0, (size_t)nk * sizeof(unsigned long long), st));
    const int bfs_grid = coop_grid((const void*)k_bfs, kT);
    Buf<int32_t> bsum(bfs_grid);
    int32_t next_id = 1;
    auto bfs = [&](int32_t start, int32_t qbase, bool ordering_search, bool by_degree, int32_t& levels,
                   int32_t& qend, int32_t& last_begin) {
        BfsArgs a{nk, off.p, adj, deg.p, mark.p, par.p, queue.p, cnt.p, bsum.p, next_id,
                  ordering_search ? kVisited : next_id, start, qbase, by_degree ? 1 : 0, out.p};
        ++next_id;
        void* args[] = {&a};
        counted();
        CK(cudaLaunchCooperativeKernel((const void*)k_bfs, dim3(bfs_grid), dim3(kT), args, 0, st));
        int32_t h[3];
        CK(cudaMemcpyAsync(h, out.p, 3 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        levels = h[0];
        qend = h[1];
        last_begin = h[2];
        tmark(ordering_search ? "ordering search" : "peripheral search", levels);
    };
    auto argmin = [&](auto launch) -> int64_t {
        static const unsigned long long none = ~0ull;
        CK(cudaMemcpyAsync(best.p, &none, sizeof(none), cudaMemcpyHostToDevice, st));
        launch();
        unsigned long long h = 0;
        CK(cudaMemcpyAsync(&h, best.p, sizeof(h), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return h == none ? -1 : (int64_t)(h & 0xFFFFFFFFull);
    };
    // component by component: the seed, the George-Liu pseudo-peripheral search (RCM and
    // MULTICOLOR), the ordering search; the queue holds the concatenated searches
    int32_t ordered = 0;
    while (ordered < nk) {
        const int64_t seed = argmin([&] {
            counted();
            k_seed<<<grid_of(nk), kT, 0, st>>>(nk, deg.p, mark.p, best.p);
        });
        if (seed < 0) throw CudaFailure{"device ordering: no seed while nodes remain"};
        int32_t start = (int32_t)seed, levels = 0, qend = 0, lastb = 0;
        if (ordering != MAILLE_ORDER_MULTICOLOR_BFS) {
            bfs(start, ordered, false, false, levels, qend, lastb);
            int32_t depth = levels;
            for (;;) {
                const int32_t lb = lastb, le = qend;
                const int64_t fpos = argmin([&] {
                    counted();
                    k_far<<<grid_of(le - lb), kT, 0, st>>>(lb, le, queue.p, deg.p, best.p);
                });
                if (fpos < 0) throw CudaFailure{"device ordering: empty last level"};
                int32_t far = 0;
                CK(cudaMemcpy(&far, queue.p + fpos, sizeof(int32_t), cudaMemcpyDeviceToHost));
                int32_t fd = 0;
                bfs(far, ordered, false, false, fd, qend, lastb);
                if (fd <= depth) break;
                start = far;
                depth = fd;
            }
        }
        bfs(start, ordered, true, ordering != MAILLE_ORDER_MULTICOLOR_BFS, levels, qend, lastb);
        if (qend <= ordered) throw CudaFailure{"device ordering: a search placed no node"};
        ordered = qend;
    }
    // visit order = the reversed search order; colours (multicolour) or dependency levels (RCM)
    Buf<int32_t> visit(nk), rpos(nk), value(nk), fail(1);
    counted(2);
    k_reverse<<<grid_of(nk), kT, 0, st>>>(nk, queue.p, visit.p, rpos.p);
    k_fill_i32<<<grid_of(nk), kT, 0, st>>>(nk, -1, value.p);
    CK(cudaMemsetAsync(fail.p, 0, sizeof(int32_t), st));
    // every co-resident warp: a warp's node spends most of its time in dependent loads and polls,
    // so the colouring is paced by the nodes in flight (Tet10 40^3: 19 ms with one block of 8 warps
    // per SM, 6.7 ms with 64 warps per SM; without the pause between polls the full grid took 88 ms)
    const int greedy_grid = coop_grid((const void*)k_greedy, kT);
    Buf<int32_t> claim(1);
    auto colour = [&](const int32_t* vis, const int32_t* rp, int mode) {
        int32_t nk_ = nk;
        const int64_t* o = off.p;
        const int32_t* ad = adj;
        int32_t* va = value.p;
        int32_t* fl = fail.p;
        int32_t* nx = claim.p;
        CK(cudaMemsetAsync(claim.p, 0, sizeof(int32_t), st));
        unsigned int p0 = kGreedyPause0, pc = kGreedyPauseCap;
        void* args[] = {&nk_, &o, &ad, &vis, &rp, &va, &mode, &fl, &nx, &p0, &pc};
        counted();
        CK(cudaLaunchCooperativeKernel((const void*)k_greedy, dim3(greedy_grid), dim3(kT), args, 0, st));
    };
    colour(visit.p, rpos.p, ordering == MAILLE_ORDER_RCM ? 1 : 0);
    tmark("greedy", greedy_grid);
    Buf<uint64_t> k0(nk), k1(nk);
    Buf<int32_t> i0(nk), i1(nk);
    if (ordering == MAILLE_ORDER_MULTICOLOR_ITERATED) {
        // iterated greedy: recolour visiting the classes from the last to the first (RCM order
        // inside a class), twice; the node dependencies now span at most the class count
        Buf<int32_t> rpos2(nk);
        for (int pass = 0; pass < 2; ++pass) {
            std::vector<int32_t> hv(nk);
            CK(cudaMemcpyAsync(hv.data(), value.p, (size_t)nk * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            const int32_t top = *std::max_element(hv.begin(), hv.end());
            counted();
            k_class_keys<<<grid_of(nk), kT, 0, st>>>(nk, top, value.p, rpos.p, k0.p, i0.p);
            size_t b2 = 0;
            CK(cub::DeviceRadixSort::SortPairs(nullptr, b2, k0.p, k1.p, i0.p, i1.p, nk, 0, 64, st));
            temp.reserve(b2);
            CK(cub::DeviceRadixSort::SortPairs(temp.p, b2, k0.p, k1.p, i0.p, i1.p, nk, 0, 64, st));
            counted(3);
            k_inverse<<<grid_of(nk), kT, 0, st>>>(nk, i1.p, rpos2.p);
            k_fill_i32<<<grid_of(nk), kT, 0, st>>>(nk, -1, value.p);
            colour(i1.p, rpos2.p, 0);
        }
    }
    int32_t h_fail = 0;
    CK(cudaMemcpyAsync(&h_fail, fail.p, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    // rows by (colour or level, RCM visit position)
    counted();
    k_order_keys<<<grid_of(nk), kT, 0, st>>>(nk, value.p, rpos.p, k0.p, i0.p);
    size_t bytes = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, k0.p, k1.p, i0.p, i1.p, nk, 0, 64, st));
    temp.reserve(bytes);
    CK(cub::DeviceRadixSort::SortPairs(temp.p, bytes, k0.p, k1.p, i0.p, i1.p, nk, 0, 64, st));
    counted();
    order.resize(nk);
    level.resize(nk);
    CK(cudaMemcpyAsync(order.data(), i1.p, (size_t)nk * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(level.data(), value.p, (size_t)nk * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    tmark("sort and copies", bfs_grid);
    if (h_fail) throw CudaFailure{"device ordering: a colouring wait ran out or a node needs 1024 colours or more"};
}


void gpu_narrow(const int64_t* in, int64_t n, int32_t* out, cudaStream_t st) {
    if (n <= 0) return;
    counted();
    k_narrow<<<grid_of(n), kT, 0, st>>>(n, in, out);
    CK(cudaGetLastError());
}

void gpu_zero_free(int64_t n, const uint8_t* fixed, double* v, cudaStream_t st) {
    if (n <= 0) return;
    counted();
    k_zero_free<<<grid_of(n), kT, 0, st>>>(n, fixed, v);
    CK(cudaGetLastError());
}

void gpu_incidence(const int32_t* conn, int64_t n, int64_t n_nodes, cudaStream_t st, int64_t* inc_ptr,
                   int32_t* inc) {
    if (n <= 0 || n >= (int64_t(1) << 31)) throw CudaFailure{"gpu_incidence: entry count out of range"};
    Buf<int32_t> iota(n);
    Buf<uint32_t> keys(n);
    counted();
    k_iota<<<grid_of(n), kT, 0, st>>>(n, iota.p);
    int bits = 1;
    while ((int64_t(1) << bits) <= n_nodes) ++bits;
    // node ids are non-negative, so their unsigned order is theirs; the sort is stable, so the
    // positions of one node stay ascending
    const uint32_t* k_in = reinterpret_cast<const uint32_t*>(conn);
    size_t bytes = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, k_in, keys.p, iota.p, inc, (int)n, 0, bits, st));
    Temp temp;
    temp.reserve(bytes);
    CK(cub::DeviceRadixSort::SortPairs(temp.p, bytes, k_in, keys.p, iota.p, inc, (int)n, 0, bits, st));
    counted(3);
    k_run_starts<<<grid_of(n_nodes + 1), kT, 0, st>>>(n_nodes, keys.p, n, inc_ptr);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));  // the temporaries are freed on return
}

}  // namespace maille
