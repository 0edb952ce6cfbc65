// batch_kernels.cu -- the batched IC(0)-PCG: every instance and every load case in one
// persistent cooperative kernel (the loop of Pcg::solve, iterative.rs:210-248, run for each
// instance and load case at once), plus the small kernels around it.
//
// One launch runs the whole solve: the initial residual, then iterations of (forward sweep,
// backward sweep + r.z, p update, SpMV + p.Ap, x/r update + r.r [, mixed: true residual]) with
// grid-wide barriers between phases, until every instance has stopped. Each load case (column)
// of each instance has its own alpha, beta and stopping test; a column that has converged is
// frozen (its alpha and beta are 0) and an instance whose columns have all stopped is skipped by
// every phase. The matrix and factor blocks are read once per phase for all columns of a row.
//
// Reductions are per instance and deterministic: a vector task (a run of K slices of one
// instance) or a U slice writes its column partials to a fixed slot; after the phase's barrier one
// warp per instance sums the instance's slots in slot order and writes the instance's scalars
// (alpha, the stopping test, beta), which every warp reads after the next barrier. (A ticket
// counter that let the last slot's warp do the sum cost that warp an atomic round trip per slice
// or task: the batch took 757 ms against 636 ms with the extra barrier.) The initial norm and the
// mixed form's true residual, which run once or rarely, still use the ticket.
//
// Sweeps are dataflow like the single-system kernel: warps take L (U) slices in level order on a
// fixed round-robin schedule and wait (bounded, acquire) for each neighbour row's ready flag of
// their load-case group, then publish their own rows (release). A group whose columns have all
// stopped neither waits nor publishes; its neighbours belong to the same instance and group and
// skip too.

#include <atomic>
#include <cmath>

#include <cooperative_groups.h>

#include "batch.cuh"

namespace cg = cooperative_groups;

namespace maille {

extern std::atomic<long long> g_kernel_launches;

namespace {

constexpr unsigned int kBatchSpin = 1u << 22;  // polls of one flag before a timeout
constexpr unsigned FULLW = 0xffffffffu;

// ---- vector access (coherent L2 loads: vectors are written inside the launch) ----------------

template <typename T, int N, int AB>
__device__ __forceinline__ void ldx(const T* p, T* out) {
    if constexpr (sizeof(T) == 8 && AB >= 16 && N % 2 == 0) {
#pragma unroll
        for (int i = 0; i < N / 2; ++i) {
            const double2 v = __ldcg(reinterpret_cast<const double2*>(p) + i);
            out[2 * i] = v.x;
            out[2 * i + 1] = v.y;
        }
    } else if constexpr (sizeof(T) == 4 && AB >= 16 && N % 4 == 0) {
#pragma unroll
        for (int i = 0; i < N / 4; ++i) {
            const float4 v = __ldcg(reinterpret_cast<const float4*>(p) + i);
            out[4 * i] = v.x;
            out[4 * i + 1] = v.y;
            out[4 * i + 2] = v.z;
            out[4 * i + 3] = v.w;
        }
    } else if constexpr (sizeof(T) == 4 && AB >= 8 && N % 2 == 0) {
#pragma unroll
        for (int i = 0; i < N / 2; ++i) {
            const float2 v = __ldcg(reinterpret_cast<const float2*>(p) + i);
            out[2 * i] = v.x;
            out[2 * i + 1] = v.y;
        }
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) out[i] = __ldcg(p + i);
    }
}

template <typename T, int N, int AB>
__device__ __forceinline__ void stx(T* p, const T* v) {
    if constexpr (sizeof(T) == 8 && AB >= 16 && N % 2 == 0) {
#pragma unroll
        for (int i = 0; i < N / 2; ++i) reinterpret_cast<double2*>(p)[i] = make_double2(v[2 * i], v[2 * i + 1]);
    } else if constexpr (sizeof(T) == 4 && AB >= 16 && N % 4 == 0) {
#pragma unroll
        for (int i = 0; i < N / 4; ++i)
            reinterpret_cast<float4*>(p)[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
    } else if constexpr (sizeof(T) == 4 && AB >= 8 && N % 2 == 0) {
#pragma unroll
        for (int i = 0; i < N / 2; ++i) reinterpret_cast<float2*>(p)[i] = make_float2(v[2 * i], v[2 * i + 1]);
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) p[i] = v[i];
    }
}

// read-only matrix values: 2 or 4 slots of one plane
__device__ __forceinline__ void ldm2(const double* p, double v[2]) {
    const double2 q = __ldg(reinterpret_cast<const double2*>(p));
    v[0] = q.x;
    v[1] = q.y;
}
__device__ __forceinline__ void ldm4(const float* p, float v[4]) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = q.x;
    v[1] = q.y;
    v[2] = q.z;
    v[3] = q.w;
}

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned int* p, unsigned int v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ bool wait_ready(const unsigned int* f, unsigned int epoch) {
    if (ld_acquire(f) >= epoch) return true;
    for (unsigned int k = 0; k < kBatchSpin; ++k) {
        __nanosleep(64);
        if (ld_acquire(f) >= epoch) return true;
    }
    return false;
}

__device__ __forceinline__ unsigned long long gtime() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---- geometry -------------------------------------------------------------------------------

template <int R, int Q, int SUB>
struct Geo {
    static constexpr int G = R / Q;             // load-case groups per row
    static constexpr int LW = G * SUB;          // lanes per row
    static constexpr int S = 32 / LW;           // rows per slice
    static constexpr int SS = S * SUB * 4;      // slots per step
    static constexpr int N = 3 * Q;             // vector values one lane carries per row
    static constexpr unsigned QM = (1u << Q) - 1u;
};

// byte alignment of a lane's Q-column group inside a row (the row itself is 3 R T aligned)
template <typename T, int Q>
constexpr int group_align() {
    constexpr int b = 3 * Q * (int)sizeof(T);
    return (b % 16 == 0) ? 16 : (b % 8 == 0) ? 8 : (int)sizeof(T);
}

// acc[k][d] += sum over this lane's slots of step gs of V_block x[col][g Q + k][d]; with `flags`
// each column's ready flag (group g) is awaited first.
template <typename M, typename T, int R, int Q, int SUB>
__device__ __forceinline__ void step_acc(const M* __restrict__ vals, const int32_t* __restrict__ col,
                                         int64_t gs, const T* x, int slot0, int g, T (&acc)[Q][3],
                                         const unsigned int* flags, unsigned int epoch, bool& ok) {
    using Gm = Geo<R, Q, SUB>;
    constexpr int AB = group_align<T, Q>();
    const int4 c4 = __ldg(reinterpret_cast<const int4*>(col + gs * Gm::SS + slot0));
    const int32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
    if (flags) {
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (ok) ok = wait_ready(flags + (int64_t)cc[j] * Gm::G + g, epoch);
    }
    const M* V = vals + gs * 9 * Gm::SS + slot0;
    if constexpr (sizeof(M) == 8) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            M v[9][2];
#pragma unroll
            for (int k = 0; k < 9; ++k) ldm2(V + k * Gm::SS + 2 * h, v[k]);
#pragma unroll
            for (int jj = 0; jj < 2; ++jj) {
                T xv[Gm::N];
                ldx<T, Gm::N, AB>(x + ((int64_t)cc[2 * h + jj] * R + g * Q) * 3, xv);
#pragma unroll
                for (int k = 0; k < Q; ++k) {
                    acc[k][0] += (T)v[0][jj] * xv[3 * k] + (T)v[1][jj] * xv[3 * k + 1] + (T)v[2][jj] * xv[3 * k + 2];
                    acc[k][1] += (T)v[3][jj] * xv[3 * k] + (T)v[4][jj] * xv[3 * k + 1] + (T)v[5][jj] * xv[3 * k + 2];
                    acc[k][2] += (T)v[6][jj] * xv[3 * k] + (T)v[7][jj] * xv[3 * k + 1] + (T)v[8][jj] * xv[3 * k + 2];
                }
            }
        }
    } else {
        M v[9][4];
#pragma unroll
        for (int k = 0; k < 9; ++k) ldm4(V + k * Gm::SS, v[k]);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            T xv[Gm::N];
            ldx<T, Gm::N, AB>(x + ((int64_t)cc[j] * R + g * Q) * 3, xv);
#pragma unroll
            for (int k = 0; k < Q; ++k) {
                acc[k][0] += (T)v[0][j] * xv[3 * k] + (T)v[1][j] * xv[3 * k + 1] + (T)v[2][j] * xv[3 * k + 2];
                acc[k][1] += (T)v[3][j] * xv[3 * k] + (T)v[4][j] * xv[3 * k + 1] + (T)v[5][j] * xv[3 * k + 2];
                acc[k][2] += (T)v[6][j] * xv[3 * k] + (T)v[7][j] * xv[3 * k + 1] + (T)v[8][j] * xv[3 * k + 2];
            }
        }
    }
}

// sum over the SUB lanes of a (row, group)
template <typename T, int Q, int SUB>
__device__ __forceinline__ void sub_sum(T (&acc)[Q][3]) {
#pragma unroll
    for (int o = SUB / 2; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < Q; ++k)
#pragma unroll
            for (int d = 0; d < 3; ++d) acc[k][d] += __shfl_xor_sync(FULLW, acc[k][d], o);
}

// Column totals of per-lane values v[k] (column g Q + k) over the warp's rows and sub-lanes; lane
// c < R returns column c's total (fixed shuffle trees).
template <int R, int Q, int SUB>
__device__ __forceinline__ double cols_to_lanes(double (&v)[Q]) {
    using Gm = Geo<R, Q, SUB>;
#pragma unroll
    for (int o = 1; o < SUB; o <<= 1)
#pragma unroll
        for (int k = 0; k < Q; ++k) v[k] += __shfl_xor_sync(FULLW, v[k], o);
#pragma unroll
    for (int o = Gm::LW; o < 32; o <<= 1)
#pragma unroll
        for (int k = 0; k < Q; ++k) v[k] += __shfl_xor_sync(FULLW, v[k], o);
    const int lane = threadIdx.x & 31;
    const int c = lane < R ? lane : 0;
    double out = 0.0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const double t = __shfl_sync(FULLW, v[k], (c / Q) * SUB);
        if (k == c % Q) out = t;
    }
    return lane < R ? out : 0.0;
}

// Writes the warp's column partials (lane c holds column c) to slot `slot`, then takes a ticket;
// true in every lane of the warp that completed the instance's `count` slots.
template <int R>
__device__ __forceinline__ bool publish(double colval, double* part, int64_t slot, unsigned int* ticket,
                                       int count) {
    const int lane = threadIdx.x & 31;
    double vals[R];
#pragma unroll
    for (int c = 0; c < R; ++c) vals[c] = __shfl_sync(FULLW, colval, c);
    unsigned int t = 0;
    if (lane == 0) {
#pragma unroll
        for (int c = 0; c < R; ++c) part[slot * R + c] = vals[c];
        __threadfence();
        t = atomicAdd(ticket, 1u);
    }
    t = __shfl_sync(FULLW, t, 0);
    if (t + 1 != (unsigned int)count) return false;
    __threadfence();
    if (lane == 0) *ticket = 0;  // next use is after a grid barrier
    return true;
}

// The finisher's totals: lane l gets column l % R summed over slots [base, base + count) in a
// fixed order (each lane a fixed stride of slots, then a fixed shuffle tree).
template <int R>
__device__ __forceinline__ double ordered_total(const double* part, int64_t base, int count) {
    const int lane = threadIdx.x & 31;
    constexpr int W = 32 / R;
    const int c = lane % R, w = lane / R;
    double s = 0.0;
    for (int k = w; k < count; k += W) s += __ldcg(part + (base + k) * R + c);
#pragma unroll
    for (int o = R; o < 32; o <<= 1) s += __shfl_xor_sync(FULLW, s, o);
    return s;
}

// Marks instance i finished when every column has stopped (lane 0).
__device__ __forceinline__ void retire_if_done(const BatchState& st, int i, uint32_t before, uint32_t after,
                                               uint32_t full) {
    if (before != full && after == full) atomicSub(st.ctrl + 0, 1);
}

template <typename M, typename T, int R, int Q, int SUB, bool MIXED>
__global__ void __launch_bounds__(256) k_batch_pcg(BatchArgs<M, T> a, int passes) {
    using Gm = Geo<R, Q, SUB>;
    constexpr int AB = group_align<T, Q>();
    constexpr uint32_t FULL = (1u << R) - 1u;
    cg::grid_group grid = cg::this_grid();
    const BatchState& st = a.st;
    const int lane = threadIdx.x & 31;
    const int rr = lane / Gm::LW, g = (lane / SUB) % Gm::G, q = lane % SUB;
    const int slot0 = 4 * (rr * SUB + q);
    const int32_t warp = (int32_t)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int32_t nwarps = (int32_t)((gridDim.x * blockDim.x) >> 5);
    const bool timed = a.timing != nullptr && blockIdx.x == 0 && threadIdx.x == 0;
    unsigned long long t_last = timed ? gtime() : 0;
    auto mark = [&](int phase) {
        if (timed) {
            const unsigned long long t = gtime();
            a.timing[phase] += t - t_last;
            t_last = t;
        }
    };
    unsigned int epoch = (unsigned int)__ldcg(st.ctrl + 4);
    const uint32_t pad = a.n_rhs >= R ? 0u : (FULL & ~((1u << a.n_rhs) - 1u));  // columns past n_rhs

    // ---- phase 0: x = 0, r = b, ||b||^2 per column -------------------------------------------
    for (int32_t t = warp; t < a.ntasks; t += nwarps) {
        const int32_t inst = a.task_inst[t];
        double part[Q] = {};
        for (int32_t sl = a.task_off[t]; sl < a.task_off[t + 1]; ++sl) {
            const int32_t row = a.K.rowid[(int64_t)sl * Gm::S + rr];
            if (q != 0 || row < 0) continue;
            const int64_t o = ((int64_t)row * R + g * Q) * 3;
            double bv[Gm::N];
            ldx<double, Gm::N, group_align<double, Q>()>(a.b + o, bv);
            T rv[Gm::N], zero[Gm::N];
#pragma unroll
            for (int k = 0; k < Gm::N; ++k) {
                rv[k] = (T)bv[k];
                zero[k] = T(0);
                part[k / 3] += bv[k] * bv[k];
            }
            stx<T, Gm::N, AB>(a.r + o, rv);
            stx<T, Gm::N, AB>(a.x + o, zero);
            if constexpr (MIXED) {
                double dz[Gm::N] = {};
                stx<double, Gm::N, group_align<double, Q>()>(a.x64 + o, dz);
                stx<double, Gm::N, group_align<double, Q>()>(a.r64 + o, bv);
            }
        }
        const double tot = cols_to_lanes<R, Q, SUB>(part);
        const int cnt = a.inst_task[inst + 1] - a.inst_task[inst];
        if (publish<R>(tot, a.part_k, t, a.tickets + inst, cnt)) {
            const double bb = ordered_total<R>(a.part_k, a.inst_task[inst], cnt);
            const int c = lane;
            bool zero = false;
            if (c < R) {
                const int64_t s = (int64_t)inst * R + c;
                st.bb[s] = bb;
                st.maxr2[s] = bb;
                st.rr[s] = bb;
                st.rz[s] = 0.0;
                st.alpha[s] = 0.0;
                st.beta[s] = 0.0;
                zero = bb == 0.0;
                st.col_iter[s] = zero ? 0 : -1;  // iteration the column stopped at (-1: running)
            }
            const uint32_t zmask = __ballot_sync(FULLW, zero) & FULL;
            if (lane == 0) {
                const uint32_t d = zmask | pad;
                st.done[inst] = d;
                st.flagged[inst] = 0u;
                st.iter[inst] = 0;
                st.status[inst] = 0;
                st.updates[inst] = 0;
                retire_if_done(st, inst, 0u, d, FULL);
            }
        }
    }
    grid.sync();
    mark(7);

    bool first = true;
    for (int pass = 0; pass < passes; ++pass) {
        if (__ldcg(st.ctrl + 0) == 0 || __ldcg(st.ctrl + 2) != 0 || __ldcg(st.ctrl + 3) != 0) break;
        // ---- forward sweep: z = L_II^-1 (r - sum L z) (Csr::precondition forward, rows in
        // level order); mixed: flagged columns first fold x32 into x64 and take r = r64 ---------
        epoch += 1;
        {
            bool ok = true;
            const bool any_flag = MIXED && __ldcg(st.ctrl + 1) != 0;
            for (int32_t sl = warp; sl < a.L.nslices; sl += nwarps) {
                const int32_t inst = __ldg(a.L.inst + sl);
                const uint32_t dm = __ldcg(st.done + inst);
                if (dm == FULL) continue;
                // a group whose columns have all stopped neither waits nor publishes
                const bool gskip = ((dm >> (g * Q)) & Gm::QM) == Gm::QM;
                const int32_t row = __ldg(a.L.rowid + (int64_t)sl * Gm::S + rr);
                T acc[Q][3] = {};
                if (!gskip) {
                    const int64_t g1 = __ldg(a.L.off + sl + 1);
                    for (int64_t gs = __ldg(a.L.off + sl); gs < g1; ++gs)
                        step_acc<M, T, R, Q, SUB>(a.Lv, a.L.col, gs, a.z, slot0, g, acc, a.flags, epoch, ok);
                }
                sub_sum<T, Q, SUB>(acc);
                if (gskip || q != 0 || row < 0) continue;
                const int64_t o = ((int64_t)row * R + g * Q) * 3;
                T tv[Gm::N];
                ldx<T, Gm::N, AB>(a.r + o, tv);
                if constexpr (MIXED) {
                    const uint32_t fm = any_flag ? __ldcg(st.flagged + inst) : 0u;
                    if ((fm >> (g * Q)) & Gm::QM) {
                        double x6[Gm::N], r6[Gm::N];
                        T x3[Gm::N];
                        constexpr int AD = group_align<double, Q>();
                        ldx<double, Gm::N, AD>(a.x64 + o, x6);
                        ldx<double, Gm::N, AD>(a.r64 + o, r6);
                        ldx<T, Gm::N, AB>(a.x + o, x3);
#pragma unroll
                        for (int k = 0; k < Gm::N; ++k) {
                            if ((fm >> (g * Q + k / 3)) & 1u) {
                                x6[k] += (double)x3[k];
                                x3[k] = T(0);
                                tv[k] = (T)r6[k];
                            }
                        }
                        stx<double, Gm::N, AD>(a.x64 + o, x6);
                        stx<T, Gm::N, AB>(a.x + o, x3);
                        stx<T, Gm::N, AB>(a.r + o, tv);
                    }
                }
                const M* d = a.D + row;
                const int64_t nb = a.nb;
                const T d0 = (T)__ldg(d), d3 = (T)__ldg(d + 3 * nb), d4 = (T)__ldg(d + 4 * nb),
                        d6 = (T)__ldg(d + 6 * nb), d7 = (T)__ldg(d + 7 * nb), d8 = (T)__ldg(d + 8 * nb);
                T zv[Gm::N];
#pragma unroll
                for (int k = 0; k < Q; ++k) {
                    const T u0 = tv[3 * k] - acc[k][0], u1 = tv[3 * k + 1] - acc[k][1],
                            u2 = tv[3 * k + 2] - acc[k][2];
                    zv[3 * k] = d0 * u0;
                    zv[3 * k + 1] = d3 * u0 + d4 * u1;
                    zv[3 * k + 2] = d6 * u0 + d7 * u1 + d8 * u2;
                }
                stx<T, Gm::N, AB>(a.z + o, zv);
                st_release(a.flags + (int64_t)row * Gm::G + g, epoch);
            }
            if (!ok) atomicExch(st.ctrl + 2, 1);
        }
        grid.sync();
        mark(3);
        if (__ldcg(st.ctrl + 2) != 0) break;

        // ---- backward sweep: z = L_II^-T (y - sum L^T z), and r.z per column ------------------
        epoch += 1;
        {
            bool ok = true;
            for (int32_t k0 = warp; k0 < a.U.nslices; k0 += nwarps) {
                const int32_t sl = __ldg(a.bwd_seq + k0);
                const int32_t inst = __ldg(a.U.inst + sl);
                const uint32_t dm = __ldcg(st.done + inst);
                if (dm == FULL) continue;
                const bool gskip = ((dm >> (g * Q)) & Gm::QM) == Gm::QM;
                const int32_t row = __ldg(a.U.rowid + (int64_t)sl * Gm::S + rr);
                T acc[Q][3] = {};
                if (!gskip) {
                    const int64_t g1 = __ldg(a.U.off + sl + 1);
                    for (int64_t gs = __ldg(a.U.off + sl); gs < g1; ++gs)
                        step_acc<M, T, R, Q, SUB>(a.Uv, a.U.col, gs, a.z, slot0, g, acc, a.flags, epoch, ok);
                }
                sub_sum<T, Q, SUB>(acc);
                double part[Q] = {};
                if (!gskip && q == 0 && row >= 0) {
                    const int64_t o = ((int64_t)row * R + g * Q) * 3;
                    T tv[Gm::N], rv[Gm::N];
                    ldx<T, Gm::N, AB>(a.z + o, tv);
                    ldx<T, Gm::N, AB>(a.r + o, rv);
                    const M* d = a.D + row;
                    const int64_t nb = a.nb;
                    const T d0 = (T)__ldg(d), d3 = (T)__ldg(d + 3 * nb), d4 = (T)__ldg(d + 4 * nb),
                            d6 = (T)__ldg(d + 6 * nb), d7 = (T)__ldg(d + 7 * nb), d8 = (T)__ldg(d + 8 * nb);
                    T zv[Gm::N];
#pragma unroll
                    for (int k = 0; k < Q; ++k) {
                        const T u0 = tv[3 * k] - acc[k][0], u1 = tv[3 * k + 1] - acc[k][1],
                                u2 = tv[3 * k + 2] - acc[k][2];
                        zv[3 * k] = d0 * u0 + d3 * u1 + d6 * u2;
                        zv[3 * k + 1] = d4 * u1 + d7 * u2;
                        zv[3 * k + 2] = d8 * u2;
                        part[k] = (double)rv[3 * k] * (double)zv[3 * k] +
                                  (double)rv[3 * k + 1] * (double)zv[3 * k + 1] +
                                  (double)rv[3 * k + 2] * (double)zv[3 * k + 2];
                    }
                    stx<T, Gm::N, AB>(a.z + o, zv);
                    st_release(a.flags + (int64_t)row * Gm::G + g, epoch);
                }
                // the slice's column partials go to its slot; the instance totals are summed after
                // the barrier (no ticket: a warp never waits on an atomic's round trip per slice)
                const double tot = cols_to_lanes<R, Q, SUB>(part);
                const int us = __ldg(a.uslot + sl);
                if (lane < R) a.part_u[(int64_t)us * R + lane] = tot;
            }
            if (!ok) atomicExch(st.ctrl + 2, 1);
            if (MIXED && blockIdx.x == 0 && threadIdx.x == 0) st.ctrl[1] = 0;
        }
        grid.sync();
        // ---- r.z per column: one warp per instance sums its slots in slot order ---------------
        if (__ldcg(st.ctrl + 2) == 0) {
            for (int32_t inst = warp; inst < a.n_inst; inst += nwarps) {
                const uint32_t dm = __ldcg(st.done + inst);
                if (dm == FULL) continue;
                const int b0 = __ldg(a.inst_uslot + inst), cnt = __ldg(a.inst_uslot + inst + 1) - b0;
                const double rz = ordered_total<R>(a.part_u, b0, cnt);
                if (lane < R) {
                    const int64_t s = (int64_t)inst * R + lane;
                    const bool live = !((dm >> lane) & 1u);
                    // iterative.rs:237-239: beta = rz_new / rz_old (0 on the first pass)
                    st.beta[s] = (live && !first) ? rz / st.rz[s] : 0.0;
                    if (live) st.rz[s] = rz;
                }
                if (MIXED && lane == 0) st.flagged[inst] = 0u;
            }
        }
        grid.sync();
        mark(4);
        if (__ldcg(st.ctrl + 2) != 0) break;
        first = false;

        // ---- p = z + beta p (iterative.rs:240-242) --------------------------------------------
        for (int32_t t = warp; t < a.ntasks; t += nwarps) {
            const int32_t inst = a.task_inst[t];
            const uint32_t dm = __ldcg(st.done + inst);
            if (dm == FULL) continue;
            double bt[Q];
#pragma unroll
            for (int k = 0; k < Q; ++k) bt[k] = __ldcg(st.beta + (int64_t)inst * R + g * Q + k);
            for (int32_t sl = a.task_off[t]; sl < a.task_off[t + 1]; ++sl) {
                const int32_t row = a.K.rowid[(int64_t)sl * Gm::S + rr];
                if (q != 0 || row < 0) continue;
                const int64_t o = ((int64_t)row * R + g * Q) * 3;
                T zv[Gm::N], pv[Gm::N];
                ldx<T, Gm::N, AB>(a.z + o, zv);
                ldx<T, Gm::N, AB>(a.p + o, pv);
#pragma unroll
                for (int k = 0; k < Gm::N; ++k) pv[k] = (T)((double)zv[k] + bt[k / 3] * (double)pv[k]);
                stx<T, Gm::N, AB>(a.p + o, pv);
            }
        }
        if (blockIdx.x == 0 && threadIdx.x == 0 && a.cancel && *a.cancel) st.ctrl[3] = 1;
        if (blockIdx.x == 0 && threadIdx.x == 0) st.ctrl[4] = (int32_t)epoch;
        grid.sync();
        mark(5);
        if (__ldcg(st.ctrl + 3) != 0) break;

        // ---- ap = K p and p.ap per column; alpha = rz / p.ap (iterative.rs:223-228) ---------
        for (int32_t t = warp; t < a.ntasks; t += nwarps) {
            const int32_t inst = a.task_inst[t];
            const uint32_t dm = __ldcg(st.done + inst);
            if (dm == FULL) continue;
            double part[Q] = {};
            for (int32_t sl = a.task_off[t]; sl < a.task_off[t + 1]; ++sl) {
                const int32_t row = a.K.rowid[(int64_t)sl * Gm::S + rr];
                T acc[Q][3] = {};
                bool ok = true;
                const int64_t g1 = a.K.off[sl + 1];
                for (int64_t gs = a.K.off[sl]; gs < g1; ++gs)
                    step_acc<M, T, R, Q, SUB>(a.Kv, a.K.col, gs, a.p, slot0, g, acc, nullptr, 0u, ok);
                sub_sum<T, Q, SUB>(acc);
                if (q != 0 || row < 0) continue;
                const int64_t o = ((int64_t)row * R + g * Q) * 3;
                T pv[Gm::N], av[Gm::N];
                ldx<T, Gm::N, AB>(a.p + o, pv);
#pragma unroll
                for (int k = 0; k < Q; ++k)
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        av[3 * k + d] = acc[k][d];
                        part[k] += (double)pv[3 * k + d] * (double)acc[k][d];
                    }
                stx<T, Gm::N, AB>(a.ap + o, av);
            }
            const double tot = cols_to_lanes<R, Q, SUB>(part);
            if (lane < R) a.part_k[(int64_t)t * R + lane] = tot;
        }
        grid.sync();
        // ---- p.ap per column: one warp per instance sums its task slots in order -------------
        for (int32_t inst = warp; inst < a.n_inst; inst += nwarps) {
            const uint32_t dm = __ldcg(st.done + inst);
            if (dm == FULL) continue;
            const int b0 = a.inst_task[inst], cnt = a.inst_task[inst + 1] - b0;
            {
                const double pap = ordered_total<R>(a.part_k, b0, cnt);
                bool bad = false;
                if (lane < R) {
                    const int64_t s = (int64_t)inst * R + lane;
                    const bool live = !((dm >> lane) & 1u);
                    double al = 0.0;
                    if (live) {
                        if (isnan(pap) || pap <= 0.0) bad = true;  // iterative.rs:224-227
                        else al = st.rz[s] / pap;
                    }
                    st.alpha[s] = al;
                }
                const bool any_bad = __ballot_sync(FULLW, bad) != 0u;
                if (lane == 0) {
                    st.iter[inst] += 1;
                    if (any_bad) {
                        st.status[inst] = 1;  // Singular
                        st.done[inst] = FULL;
                        retire_if_done(st, inst, dm, FULL, FULL);
                    }
                }
            }
        }
        grid.sync();
        mark(0);

        // ---- x += alpha p, r -= alpha ap, ||r||^2 per column; stopping test ------------------
        for (int32_t t = warp; t < a.ntasks; t += nwarps) {
            const int32_t inst = a.task_inst[t];
            const uint32_t dm = __ldcg(st.done + inst);
            if (dm == FULL) continue;
            double al[Q];
#pragma unroll
            for (int k = 0; k < Q; ++k) al[k] = __ldcg(st.alpha + (int64_t)inst * R + g * Q + k);
            double part[Q] = {};
            for (int32_t sl = a.task_off[t]; sl < a.task_off[t + 1]; ++sl) {
                const int32_t row = a.K.rowid[(int64_t)sl * Gm::S + rr];
                if (q != 0 || row < 0) continue;
                const int64_t o = ((int64_t)row * R + g * Q) * 3;
                T xv[Gm::N], rv[Gm::N], pv[Gm::N], av[Gm::N];
                ldx<T, Gm::N, AB>(a.x + o, xv);
                ldx<T, Gm::N, AB>(a.r + o, rv);
                ldx<T, Gm::N, AB>(a.p + o, pv);
                ldx<T, Gm::N, AB>(a.ap + o, av);
#pragma unroll
                for (int k = 0; k < Gm::N; ++k) {
                    if (al[k / 3] != 0.0) {
                        xv[k] = (T)((double)xv[k] + al[k / 3] * (double)pv[k]);
                        rv[k] = (T)((double)rv[k] - al[k / 3] * (double)av[k]);
                    }
                    part[k / 3] += (double)rv[k] * (double)rv[k];
                }
                stx<T, Gm::N, AB>(a.x + o, xv);
                stx<T, Gm::N, AB>(a.r + o, rv);
            }
            const double tot = cols_to_lanes<R, Q, SUB>(part);
            if (lane < R) a.part_k[(int64_t)t * R + lane] = tot;
        }
        grid.sync();
        // ---- ||r||^2 per column and the stopping test: one warp per instance -----------------
        for (int32_t inst = warp; inst < a.n_inst; inst += nwarps) {
            const uint32_t dm = __ldcg(st.done + inst);
            if (dm == FULL) continue;
            const int b0 = a.inst_task[inst], cnt = a.inst_task[inst + 1] - b0;
            {
                const double rrv = ordered_total<R>(a.part_k, b0, cnt);
                const int it = __ldcg(st.iter + inst);
                const bool capped = it >= a.max_iter;
                bool conv = false, flag = false;
                if (lane < R) {
                    const int64_t s = (int64_t)inst * R + lane;
                    const bool live = !((dm >> lane) & 1u);
                    if (live) {
                        st.rr[s] = rrv;
                        const bool small = rrv <= a.tol2 * st.bb[s];  // iterative.rs:233
                        if (!MIXED) {
                            conv = small;
                            if (conv) st.col_iter[s] = it;
                        } else {
                            // reliable update when converged by the recurrence, when the residual
                            // fell by delta since the last update, or at the cap
                            flag = small || rrv < a.delta2 * st.maxr2[s] || capped;
                        }
                    }
                }
                const uint32_t cm = __ballot_sync(FULLW, conv) & FULL;
                const uint32_t fm = __ballot_sync(FULLW, flag) & FULL;
                if (lane == 0) {
                    uint32_t nd = dm | cm;
                    if (!MIXED && capped && nd != FULL) {
                        st.status[inst] = 2;  // IterativeNotConverged
                        nd = FULL;
                    }
                    if (nd != dm) {
                        st.done[inst] = nd;
                        retire_if_done(st, inst, dm, nd, FULL);
                    }
                    if (MIXED && fm) {
                        st.flagged[inst] = fm;
                        atomicExch(st.ctrl + 1, 1);
                    }
                }
            }
        }
        grid.sync();
        mark(1);

        // ---- mixed: r64 = b - K64 (x64 + x32) for flagged instances; true stopping test -------
        if constexpr (MIXED) {
            if (__ldcg(st.ctrl + 1) != 0) {
                for (int32_t t = warp; t < a.ntasks; t += nwarps) {
                    const int32_t inst = a.task_inst[t];
                    const uint32_t fm = __ldcg(st.flagged + inst);
                    if (fm == 0u) continue;
                    const uint32_t dm = __ldcg(st.done + inst);
                    double part[Q] = {};
                    for (int32_t sl = a.task_off[t]; sl < a.task_off[t + 1]; ++sl) {
                        const int32_t row = a.K.rowid[(int64_t)sl * Gm::S + rr];
                        double acc[Q][3] = {};
                        bool ok = true;
                        const int64_t g1 = a.K.off[sl + 1];
                        for (int64_t gs = a.K.off[sl]; gs < g1; ++gs)
                            step_acc<double, double, R, Q, SUB>(a.K64, a.K.col, gs, a.x64, slot0, g, acc,
                                                                nullptr, 0u, ok);
                        // plus the x32 part against the same FP64 blocks
                        for (int64_t gs = a.K.off[sl]; gs < g1; ++gs) {
                            const int4 c4 = __ldg(reinterpret_cast<const int4*>(a.K.col + gs * Gm::SS + slot0));
                            const int32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
                            const double* V = a.K64 + gs * 9 * Gm::SS + slot0;
#pragma unroll
                            for (int j = 0; j < 4; ++j) {
                                T xv[Gm::N];
                                ldx<T, Gm::N, AB>(a.x + ((int64_t)cc[j] * R + g * Q) * 3, xv);
#pragma unroll
                                for (int k = 0; k < Q; ++k) {
                                    const double x0 = xv[3 * k], x1 = xv[3 * k + 1], x2 = xv[3 * k + 2];
                                    acc[k][0] += __ldg(V + j) * x0 + __ldg(V + Gm::SS + j) * x1 + __ldg(V + 2 * Gm::SS + j) * x2;
                                    acc[k][1] += __ldg(V + 3 * Gm::SS + j) * x0 + __ldg(V + 4 * Gm::SS + j) * x1 + __ldg(V + 5 * Gm::SS + j) * x2;
                                    acc[k][2] += __ldg(V + 6 * Gm::SS + j) * x0 + __ldg(V + 7 * Gm::SS + j) * x1 + __ldg(V + 8 * Gm::SS + j) * x2;
                                }
                            }
                        }
                        sub_sum<double, Q, SUB>(acc);
                        if (q != 0 || row < 0) continue;
                        const int64_t o = ((int64_t)row * R + g * Q) * 3;
                        constexpr int AD = group_align<double, Q>();
                        double bv[Gm::N], rv[Gm::N];
                        ldx<double, Gm::N, AD>(a.b + o, bv);
                        ldx<double, Gm::N, AD>(a.r64 + o, rv);
#pragma unroll
                        for (int k = 0; k < Q; ++k)
#pragma unroll
                            for (int d = 0; d < 3; ++d) {
                                const double v = bv[3 * k + d] - acc[k][d];
                                if ((fm >> (g * Q + k)) & 1u) rv[3 * k + d] = v;
                                part[k] += v * v;
                            }
                        stx<double, Gm::N, AD>(a.r64 + o, rv);
                    }
                    const double tot = cols_to_lanes<R, Q, SUB>(part);
                    const int b0 = a.inst_task[inst], cnt = a.inst_task[inst + 1] - b0;
                    if (publish<R>(tot, a.part_k, t, a.tickets + 2 * a.n_inst + inst, cnt)) {
                        const double rt = ordered_total<R>(a.part_k, b0, cnt);
                        const int it = __ldcg(st.iter + inst);
                        bool conv = false;
                        if (lane < R && ((fm >> lane) & 1u)) {
                            const int64_t s = (int64_t)inst * R + lane;
                            st.maxr2[s] = rt;
                            st.rr[s] = rt;
                            conv = rt <= a.tol2 * st.bb[s];
                            if (conv) st.col_iter[s] = it;
                        }
                        const uint32_t cm = __ballot_sync(FULLW, conv) & FULL;
                        if (lane == 0) {
                            uint32_t nd = dm | cm;
                            st.updates[inst] += 1;
                            if (it >= a.max_iter && nd != FULL) {
                                st.status[inst] = 2;
                                nd = FULL;
                            }
                            if (nd != dm) {
                                st.done[inst] = nd;
                                retire_if_done(st, inst, dm, nd, FULL);
                            }
                        }
                    }
                }
                grid.sync();
                mark(2);
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) st.ctrl[4] = (int32_t)epoch;
    if (timed) a.timing[6] += 1;
}

// ---- small kernels ----------------------------------------------------------------------------

template <typename T>
__global__ void k_bsell_fill(int64_t n, int slots, const int32_t* __restrict__ src,
                             const double* __restrict__ csr, T* __restrict__ vals) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int64_t g = t / slots, j = t - g * slots;
    const int32_t p = src[t];
    const double* m = csr + 9 * (int64_t)(p < 0 ? 0 : p);
#pragma unroll
    for (int k = 0; k < 9; ++k) vals[(g * 9 + k) * slots + j] = p < 0 ? T(0) : (T)m[k];
}

__global__ void k_batch_rhs(int32_t nb, int R, int n_rhs, int64_t n3, const int32_t* __restrict__ perm,
                            const uint8_t* __restrict__ fixmask, const double* __restrict__ f,
                            const double* __restrict__ coupling, double* __restrict__ b) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = ((int64_t)nb + 1) * R * 3;
    if (t >= total) return;
    const int64_t I = t / (3 * R);
    const int rem = (int)(t - I * 3 * R);
    const int c = rem / 3, d = rem % 3;
    double v = 0.0;
    if (I < nb && c < n_rhs && !((fixmask[I] >> d) & 1)) {
        const int64_t gdof = 3 * (int64_t)perm[I] + d;
        v = (f ? f[(int64_t)c * n3 + gdof] : 0.0) - (coupling ? coupling[gdof] : 0.0);
    }
    b[t] = v;
}

__global__ void k_batch_gather(int64_t n_nodes, int R, int n_rhs, const int32_t* __restrict__ inv,
                               const uint8_t* __restrict__ fixed, const double* __restrict__ imposed,
                               const double* __restrict__ x64, const float* __restrict__ x32,
                               double* __restrict__ u) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n3 = 3 * n_nodes;
    if (t >= n3 * n_rhs) return;
    const int64_t c = t / n3, gdof = t - c * n3;
    const int64_t v = gdof / 3;
    const int d = (int)(gdof - 3 * v);
    const int32_t I = inv[v];
    double val = 0.0;
    if (fixed && fixed[gdof]) val = imposed ? imposed[gdof] : 0.0;
    else if (I >= 0) {
        const int64_t o = ((int64_t)I * R + c) * 3 + d;
        val = x64[o] + (x32 ? (double)x32[o] : 0.0);
    }
    u[t] = val;
}

// ctrl[0] = active instances, ctrl[1..3] = 0 (ctrl[4], the epoch, is kept); tickets = 0
__global__ void k_batch_reset(int32_t* ctrl, int32_t n_inst, unsigned int* tickets, int64_t nt) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < 4) ctrl[t] = t == 0 ? n_inst : 0;
    if (t < nt) tickets[t] = 0u;
}

// ---- kernel table -----------------------------------------------------------------------------

template <typename M, typename T, bool MIXED>
void* pick(const BatchShape& s) {
#define MAILLE_BPICK(R_, Q_, S_) \
    if (s.R == R_ && s.Q == Q_ && s.SUB == S_) return (void*)k_batch_pcg<M, T, R_, Q_, S_, MIXED>;
    MAILLE_BPICK(8, 8, 1) MAILLE_BPICK(8, 8, 2) MAILLE_BPICK(8, 4, 1) MAILLE_BPICK(8, 4, 2)
    MAILLE_BPICK(8, 2, 1)
    MAILLE_BPICK(4, 4, 1) MAILLE_BPICK(4, 4, 2) MAILLE_BPICK(4, 2, 1)
    MAILLE_BPICK(2, 2, 1) MAILLE_BPICK(2, 2, 2) MAILLE_BPICK(2, 1, 1)
#undef MAILLE_BPICK
    return nullptr;
}

}  // namespace

bool batch_shape_supported(const BatchShape& s) { return pick<double, double, false>(s) != nullptr; }

template <typename M, typename T, bool MIXED>
int batch_grid(const BatchShape& s, int threads) {
    void* f = pick<M, T, MIXED>(s);
    if (!f) return 0;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, threads, 0);
    return sms * per_sm;
}

template <typename M, typename T, bool MIXED>
cudaError_t launch_batch_pcg(const BatchShape& s, const BatchArgs<M, T>& a, int grid, int threads,
                             int passes, cudaStream_t st) {
    void* f = pick<M, T, MIXED>(s);
    if (!f || grid <= 0) return cudaErrorInvalidValue;
    BatchArgs<M, T> copy = a;
    int ps = passes;
    void* args[] = {&copy, &ps};
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    return cudaLaunchCooperativeKernel(f, dim3(grid), dim3(threads), args, 0, st);
}

template int batch_grid<double, double, false>(const BatchShape&, int);
template int batch_grid<float, float, true>(const BatchShape&, int);
template cudaError_t launch_batch_pcg<double, double, false>(const BatchShape&, const BatchArgs<double, double>&,
                                                             int, int, int, cudaStream_t);
template cudaError_t launch_batch_pcg<float, float, true>(const BatchShape&, const BatchArgs<float, float>&,
                                                          int, int, int, cudaStream_t);

template <typename T>
void launch_bsell_fill(int64_t steps, int slots, const int32_t* src, const double* csr, T* vals,
                       cudaStream_t st) {
    const int64_t n = steps * slots;
    if (n <= 0) return;
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    k_bsell_fill<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, slots, src, csr, vals);
}
template void launch_bsell_fill<double>(int64_t, int, const int32_t*, const double*, double*, cudaStream_t);
template void launch_bsell_fill<float>(int64_t, int, const int32_t*, const double*, float*, cudaStream_t);

void launch_batch_reset(int32_t* ctrl, int32_t n_inst, unsigned int* tickets, int64_t nt,
                        cudaStream_t st) {
    const int64_t n = nt > 4 ? nt : 4;
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    k_batch_reset<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(ctrl, n_inst, tickets, nt);
}

void launch_batch_rhs(int32_t nb, int R, int n_rhs, int64_t n3, const int32_t* perm,
                      const uint8_t* fixmask, const double* f, const double* coupling, double* b,
                      cudaStream_t st) {
    const int64_t n = ((int64_t)nb + 1) * R * 3;
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    k_batch_rhs<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(nb, R, n_rhs, n3, perm, fixmask, f, coupling, b);
}

void launch_batch_gather(int64_t n_nodes, int R, int n_rhs, const int32_t* inv, const uint8_t* fixed,
                         const double* imposed, const double* x64, const float* x32, double* u,
                         cudaStream_t st) {
    const int64_t n = 3 * n_nodes * n_rhs;
    if (n <= 0) return;
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    k_batch_gather<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n_nodes, R, n_rhs, inv, fixed, imposed, x64,
                                                                 x32, u);
}

}  // namespace maille
