// analysis.cu -- symbolic analysis on the device (see analysis.cuh).
//
// Reference counterparts: Graph::from_elements (iterative.rs:38-76) builds the DOF graph from the
// elements, Csr::zeros (iterative.rs:91-114) lays out the lower profile, and FreeSystem::new
// (model.rs:1480-1492) adds every element matrix entry through Csr::add's binary search
// (iterative.rs:121-128). Here, on nodes and in the solver numbering the host ordering chose:
//  * pattern: every element emits the (row, column) keys of its kept node pairs, plus one
//    diagonal key per row; a radix sort and a unique pass give the full block pattern, rows in
//    order and columns ascending, and row pointers, diagonal and transpose positions follow by
//    binary search;
//  * scatter map: every element node pair (a, b) whose blocks fall in the lower triangle emits its
//    lower slot; a stable radix sort by slot keeps, inside each slot, the element order of the
//    input, which is the order the host analysis produces and the assembly reduces in.
// Radix sorts and scans are CUB's device primitives; the rest are the kernels below. Every step is
// a deterministic function of its inputs.

#include <atomic>
#include <climits>

#include <cub/cub.cuh>

#include "analysis.cuh"
#include "cuda_host.hpp"

namespace maille {

extern std::atomic<long long> g_kernel_launches;

namespace {

constexpr int kT = 256;

inline unsigned grid_of(int64_t n) {
    const int64_t g = (n + kT - 1) / kT;
    return (unsigned)(g < 1 ? 1 : (g > (1 << 20) ? (1 << 20) : g));
}
inline void counted(int n = 1) { g_kernel_launches.fetch_add(n, std::memory_order_relaxed); }

template <typename K>
__device__ __forceinline__ int64_t lower_bound_dev(const K* a, int64_t n, K key) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (a[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

#define GRID_STRIDE(t, n) \
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < (n); t += (int64_t)gridDim.x * blockDim.x)

// keys of the pattern: (I << sh) | J for every ordered pair of distinct kept nodes of an element,
// then (r << sh) | r for every row; ~0 for pairs with a dropped node
__global__ void k_pair_keys(int npe, int64_t ne, const int32_t* __restrict__ conn,
                            const int32_t* __restrict__ inv, int32_t nb, int sh, uint64_t* __restrict__ keys) {
    const int64_t per = (int64_t)npe * (npe - 1);
    GRID_STRIDE(t, ne * per + nb) {
        uint64_t key;
        if (t < ne * per) {
            const int64_t e = t / per;
            const int rem = (int)(t - e * per);
            const int a = rem / (npe - 1), bi = rem % (npe - 1), b = bi < a ? bi : bi + 1;
            const int32_t I = inv[conn[e * npe + a]], J = inv[conn[e * npe + b]];
            key = (I < 0 || J < 0) ? ~0ull : (((uint64_t)I << sh) | (uint64_t)J);
        } else {
            const uint64_t r = (uint64_t)(t - ne * per);
            key = (r << sh) | r;
        }
        keys[t] = key;
    }
}

__global__ void k_row_ptr(const uint64_t* __restrict__ keys, int64_t blocks, int32_t nb, int sh,
                          int64_t* __restrict__ row_ptr) {
    GRID_STRIDE(r, (int64_t)nb + 1) row_ptr[r] = lower_bound_dev<uint64_t>(keys, blocks, (uint64_t)r << sh);
}

__global__ void k_cols_tpos(const uint64_t* __restrict__ keys, int64_t blocks, int sh,
                            int32_t* __restrict__ col, int64_t* __restrict__ tpos) {
    const uint64_t mask = (1ull << sh) - 1;
    GRID_STRIDE(p, blocks) {
        const uint64_t k = keys[p];
        const uint64_t r = k >> sh, c = k & mask;
        col[p] = (int32_t)c;
        tpos[p] = lower_bound_dev<uint64_t>(keys, blocks, (c << sh) | r);
    }
}

// diag[r], and the number of lower slots of row r (columns <= r) in lcnt[r]; lcnt[nb] = 0
__global__ void k_diag(const uint64_t* __restrict__ keys, int64_t blocks, int32_t nb, int sh,
                       const int64_t* __restrict__ row_ptr, int64_t* __restrict__ diag,
                       int64_t* __restrict__ lcnt) {
    GRID_STRIDE(r, (int64_t)nb + 1) {
        if (r == nb) {
            lcnt[r] = 0;
        } else {
            const int64_t d = lower_bound_dev<uint64_t>(keys, blocks, ((uint64_t)r << sh) | (uint64_t)r);
            diag[r] = d;
            lcnt[r] = d - row_ptr[r] + 1;
        }
    }
}

__global__ void k_lslots(const uint64_t* __restrict__ keys, int64_t blocks, int sh,
                         const int64_t* __restrict__ row_ptr, const int64_t* __restrict__ diag,
                         const int64_t* __restrict__ lfirst, int64_t* __restrict__ lslot,
                         int32_t* __restrict__ lrow) {
    GRID_STRIDE(p, blocks) {
        const int64_t r = (int64_t)(keys[p] >> sh);
        if (p <= diag[r]) {
            const int64_t l = lfirst[r] + (p - row_ptr[r]);
            lslot[l] = p;
            lrow[l] = (int32_t)r;
        }
    }
}

// scatter keys: for element e and local nodes (a, b) with rows I = inv(a) >= J = inv(b), the lower
// slot of (I, J) and the contribution code (e * npairs + pair(min, max)) | (a > b) << 31
__global__ void k_scatter_keys(int npe, int64_t ne, const int32_t* __restrict__ conn,
                               const int32_t* __restrict__ inv, const int32_t* __restrict__ col,
                               const int64_t* __restrict__ row_ptr, const int64_t* __restrict__ diag,
                               const int64_t* __restrict__ lfirst, uint32_t* __restrict__ skey,
                               uint32_t* __restrict__ sval) {
    const int64_t per = (int64_t)npe * npe;
    const int np = npe * (npe + 1) / 2;
    GRID_STRIDE(t, ne * per) {
        const int64_t e = t / per;
        const int rem = (int)(t - e * per);
        const int a = rem / npe, b = rem % npe;
        const int32_t I = inv[conn[e * npe + a]], J = inv[conn[e * npe + b]];
        uint32_t key = 0xFFFFFFFFu, val = 0u;
        if (I >= 0 && J >= 0 && J <= I) {
            const int64_t rb = row_ptr[I];
            const int64_t p = rb + lower_bound_dev<int32_t>(col + rb, diag[I] - rb + 1, J);
            key = (uint32_t)(lfirst[I] + (p - rb));
            const int lo = a < b ? a : b, hi = a < b ? b : a;
            const int pair = lo * npe - lo * (lo - 1) / 2 + (hi - lo);
            val = (uint32_t)(e * np + pair) | (a > b ? 0x80000000u : 0u);
        }
        skey[t] = key;
        sval[t] = val;
    }
}

__global__ void k_lptr(const uint32_t* __restrict__ skey, int64_t n, int64_t nl, int64_t* __restrict__ lptr) {
    GRID_STRIDE(l, nl + 1) lptr[l] = lower_bound_dev<uint32_t>(skey, n, (uint32_t)l);
}

__global__ void k_fill_value(int64_t n, int32_t v, int32_t* __restrict__ a) {
    GRID_STRIDE(i, n) a[i] = v;
}

__device__ __forceinline__ int64_t part_start(SellKind kind, const int64_t* row_ptr, const int64_t* diag, int64_t i) {
    return kind == SELL_UPPER ? diag[i] + 1 : row_ptr[i];
}
__device__ __forceinline__ int64_t part_end(SellKind kind, const int64_t* row_ptr, const int64_t* diag, int64_t i) {
    return kind == SELL_LOWER ? diag[i] : row_ptr[i + 1];
}

__global__ void k_fill_sell(SellKind kind, int32_t lpr, int64_t nrow_slots, const int32_t* __restrict__ rowid,
                            const int64_t* __restrict__ off, const int64_t* __restrict__ row_ptr,
                            const int32_t* __restrict__ col, const int64_t* __restrict__ diag,
                            int32_t* __restrict__ slot_col, int32_t* __restrict__ slot_src) {
    const int S = 32 / lpr, per_step = 4 * lpr;
    GRID_STRIDE(t, nrow_slots) {
        const int32_t i = rowid[t];
        if (i < 0) continue;
        const int64_t s = t / S;
        const int r = (int)(t - s * S);
        const int64_t b0 = part_start(kind, row_ptr, diag, i), b1 = part_end(kind, row_ptr, diag, i);
        for (int64_t p = b0; p < b1; ++p) {
            const int64_t b = p - b0, st = b / per_step, rem = b % per_step;
            const int64_t slot = (off[s] + st) * 128 + 4 * (r * lpr + rem / 4) + rem % 4;
            slot_col[slot] = col[p];
            slot_src[slot] = (int32_t)p;
        }
    }
}

__global__ void k_fill_psell(SellKind kind, int64_t nrows, const int32_t* __restrict__ rows,
                             const int64_t* __restrict__ rstart, const int64_t* __restrict__ row_ptr,
                             const int32_t* __restrict__ col, const int64_t* __restrict__ diag,
                             int32_t* __restrict__ slot_col, int32_t* __restrict__ slot_src) {
    GRID_STRIDE(k, nrows) {
        const int32_t i = rows[k];
        const int64_t b0 = part_start(kind, row_ptr, diag, i), b1 = part_end(kind, row_ptr, diag, i);
        for (int64_t p = b0; p < b1; ++p) {
            slot_col[rstart[k] + (p - b0)] = col[p];
            slot_src[rstart[k] + (p - b0)] = (int32_t)p;
        }
    }
}

// CUB temporary storage, grown on demand
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

// frees a device buffer when it leaves scope unless released
template <typename T>
struct Owned {
    T* p = nullptr;
    explicit Owned(size_t n) : p(dalloc<T>(n)) {}
    ~Owned() { dfree(p); }
    T* release() {
        T* q = p;
        p = nullptr;
        return q;
    }
    Owned(const Owned&) = delete;
    Owned& operator=(const Owned&) = delete;
};

}  // namespace

void gpu_pattern(int npe, int64_t n_elems, const int32_t* conn, const int32_t* inv, int32_t nb,
                 cudaStream_t st, PatternDev& out, std::vector<int64_t>& h_row_ptr,
                 std::vector<int64_t>& h_diag) {
    out = PatternDev{};
    int sh = 1;
    while ((int64_t(1) << sh) <= (int64_t)nb) ++sh;  // nb < 2^sh: valid keys stay below ~0
    const int64_t nkeys = n_elems * npe * (npe - 1) + nb;
    const int64_t nscat = n_elems * npe * npe;
    if (nkeys >= INT_MAX || nscat >= INT_MAX || 2 * sh > 62)
        throw CudaFailure{"mesh too large for the device analysis"};
    Temp temp;
    Owned<uint64_t> ukeys(nkeys);
    int64_t blocks = 0;
    {
        Owned<uint64_t> ka(nkeys), kb(nkeys);
        counted();
        k_pair_keys<<<grid_of(nkeys), kT, 0, st>>>(npe, n_elems, conn, inv, nb, sh, ka.p);
        CK(cudaGetLastError());
        cub::DoubleBuffer<uint64_t> db(ka.p, kb.p);
        size_t bytes = 0;
        CK(cub::DeviceRadixSort::SortKeys(nullptr, bytes, db, (int)nkeys, 0, 2 * sh, st));
        temp.reserve(bytes);
        CK(cub::DeviceRadixSort::SortKeys(temp.p, bytes, db, (int)nkeys, 0, 2 * sh, st));
        Owned<int> nsel(1);
        bytes = 0;
        CK(cub::DeviceSelect::Unique(nullptr, bytes, db.Current(), ukeys.p, nsel.p, (int)nkeys, st));
        temp.reserve(bytes);
        CK(cub::DeviceSelect::Unique(temp.p, bytes, db.Current(), ukeys.p, nsel.p, (int)nkeys, st));
        counted(3);
        int n = 0;
        CK(cudaMemcpyAsync(&n, nsel.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        uint64_t last = 0;
        CK(cudaMemcpy(&last, ukeys.p + (n - 1), sizeof(uint64_t), cudaMemcpyDeviceToHost));
        blocks = last == ~0ull ? n - 1 : n;
    }
    if (blocks >= (int64_t(1) << 31)) throw CudaFailure{"pattern too large for 32-bit block positions"};
    Owned<int64_t> row_ptr(nb + 1), diag(nb), tpos(blocks), lcnt(nb + 1), lfirst(nb + 1);
    Owned<int32_t> col(blocks);
    counted(3);
    k_row_ptr<<<grid_of(nb + 1), kT, 0, st>>>(ukeys.p, blocks, nb, sh, row_ptr.p);
    k_cols_tpos<<<grid_of(blocks), kT, 0, st>>>(ukeys.p, blocks, sh, col.p, tpos.p);
    k_diag<<<grid_of(nb + 1), kT, 0, st>>>(ukeys.p, blocks, nb, sh, row_ptr.p, diag.p, lcnt.p);
    CK(cudaGetLastError());
    size_t bytes = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, lcnt.p, lfirst.p, (int)(nb + 1), st));
    temp.reserve(bytes);
    CK(cub::DeviceScan::ExclusiveSum(temp.p, bytes, lcnt.p, lfirst.p, (int)(nb + 1), st));
    counted();
    int64_t nl = 0;
    CK(cudaMemcpyAsync(&nl, lfirst.p + nb, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    Owned<int64_t> lslot(nl), lptr(nl + 1);
    Owned<int32_t> lrow(nl);
    counted();
    k_lslots<<<grid_of(blocks), kT, 0, st>>>(ukeys.p, blocks, sh, row_ptr.p, diag.p, lfirst.p, lslot.p, lrow.p);
    CK(cudaGetLastError());
    Owned<uint32_t> sval_sorted(nscat);
    {
        Owned<uint32_t> ska(nscat), skb(nscat), sva(nscat);
        counted();
        k_scatter_keys<<<grid_of(nscat), kT, 0, st>>>(npe, n_elems, conn, inv, col.p, row_ptr.p, diag.p,
                                                      lfirst.p, ska.p, sva.p);
        CK(cudaGetLastError());
        bytes = 0;
        CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, ska.p, skb.p, sva.p, sval_sorted.p, (int)nscat, 0, 32, st));
        temp.reserve(bytes);
        CK(cub::DeviceRadixSort::SortPairs(temp.p, bytes, ska.p, skb.p, sva.p, sval_sorted.p, (int)nscat, 0, 32, st));
        counted(2);
        k_lptr<<<grid_of(nl + 1), kT, 0, st>>>(skb.p, nscat, nl, lptr.p);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(&out.ncontrib, lptr.p + nl, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        h_row_ptr.resize((size_t)nb + 1);
        h_diag.resize((size_t)nb);
        CK(cudaMemcpyAsync(h_row_ptr.data(), row_ptr.p, ((size_t)nb + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(h_diag.data(), diag.p, (size_t)nb * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));  // the sort buffers are freed below
    }
    out.blocks = blocks;
    out.nl = nl;
    out.row_ptr = row_ptr.release();
    out.col = col.release();
    out.diag = diag.release();
    out.tpos = tpos.release();
    out.lslot = lslot.release();
    out.lrow = lrow.release();
    out.lptr = lptr.release();
    out.contrib = sval_sorted.release();
}

void fill_sell(SellKind kind, int32_t lpr, int32_t nslices, int64_t steps, const int32_t* rowid,
               const int64_t* off, const int64_t* row_ptr, const int32_t* col, const int64_t* diag,
               int32_t nb, int32_t* slot_col, int32_t* slot_src, cudaStream_t st) {
    const int64_t nslots = steps * 128, nrs = (int64_t)nslices * (32 / lpr);
    counted(2);
    k_fill_value<<<grid_of(nslots), kT, 0, st>>>(nslots, nb, slot_col);
    CK(cudaMemsetAsync(slot_src, 0xFF, (size_t)nslots * sizeof(int32_t), st));
    k_fill_sell<<<grid_of(nrs), kT, 0, st>>>(kind, lpr, nrs, rowid, off, row_ptr, col, diag, slot_col, slot_src);
    CK(cudaGetLastError());
}

void fill_psell(SellKind kind, int64_t nrows, int64_t steps, const int32_t* rows, const int64_t* rstart,
                const int64_t* row_ptr, const int32_t* col, const int64_t* diag, int32_t nb,
                int32_t* slot_col, int32_t* slot_src, cudaStream_t st) {
    const int64_t nslots = steps * 128;
    counted(2);
    k_fill_value<<<grid_of(nslots), kT, 0, st>>>(nslots, nb, slot_col);
    CK(cudaMemsetAsync(slot_src, 0xFF, (size_t)nslots * sizeof(int32_t), st));
    k_fill_psell<<<grid_of(nrows), kT, 0, st>>>(kind, nrows, rows, rstart, row_ptr, col, diag, slot_col, slot_src);
    CK(cudaGetLastError());
}

}  // namespace maille
