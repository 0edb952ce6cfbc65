// persist.cu -- the whole IC(0)-PCG iteration in one persistent cooperative kernel.
//
// One launch runs up to `chunk` iterations of Pcg::solve (iterative.rs:222-243): the SpMV, the
// x/r update with the stopping test, the IC(0) forward and backward sweeps and the p update.
// Phases are separated by grid-wide barriers; every block sums the per-block partials of a
// reduction in the same fixed order, so alpha, beta and the stopping decisions are bit-identical
// in every block and the whole grid takes the same branches. The mixed form adds the reliable
// update (x64 += x32, r64 = b - K64 x64 against the FP64 matrix, r32 = r64) on the iterations
// whose FP32 residual fell by `delta` since the last one.
//
// Sweeps are dataflow instead of one barrier per level: warps take slices in level order on a
// fixed round-robin schedule; before gathering a neighbour's value a lane waits for that row's
// ready flag to reach the current sweep epoch (acquire), and after writing a row the lane
// publishes its flag (release). A slice only depends on slices of earlier levels, which come
// earlier in every warp's schedule, and all warps are co-resident (cooperative launch), so every
// wait ends; each wait is also bounded and reports a timeout status instead of spinning forever.
//
// Vectors written inside the launch are read with ld.global.cg (L2, coherent after a barrier or
// an acquire); matrix data, which no phase writes, through the read-only path.

#include <atomic>
#include <cmath>

#include <cooperative_groups.h>

#include "reduce.cuh"
#include "sparse.cuh"

namespace cg = cooperative_groups;

namespace maille {

extern std::atomic<long long> g_kernel_launches;

namespace {

constexpr int kPW = 8;                        // warps per block
constexpr unsigned int kSpinLimit = 1u << 22;  // polls of one flag before a timeout (~0.3 s)

template <typename T>
__device__ __forceinline__ void node3_cg(const T* x, int64_t c, T& a, T& b, T& d);
template <>
__device__ __forceinline__ void node3_cg<float>(const float* x, int64_t c, float& a, float& b, float& d) {
    const float4 q = __ldcg(reinterpret_cast<const float4*>(x + 4 * c));
    a = q.x; b = q.y; d = q.z;
}
template <>
__device__ __forceinline__ void node3_cg<double>(const double* x, int64_t c, double& a, double& b, double& d) {
    const double2 q = __ldcg(reinterpret_cast<const double2*>(x + 4 * c));
    a = q.x; b = q.y; d = __ldcg(x + 4 * c + 2);
}

__device__ __forceinline__ void ldv4(const float* p, float v[4]) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void ldv4(const double* p, double v[4]) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p + 2));
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

// node i of a padded vector as 4 doubles (coherent L2 loads) and back
__device__ __forceinline__ void get4(const float* x, int64_t i, double v[4]) {
    const float4 q = __ldcg(reinterpret_cast<const float4*>(x + 4 * i));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void get4(const double* x, int64_t i, double v[4]) {
    const double2 a = __ldcg(reinterpret_cast<const double2*>(x + 4 * i));
    const double2 b = __ldcg(reinterpret_cast<const double2*>(x + 4 * i + 2));
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void set4(float* x, int64_t i, const double v[4]) {
    *reinterpret_cast<float4*>(x + 4 * i) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
}
__device__ __forceinline__ void set4(double* x, int64_t i, const double v[4]) {
    *reinterpret_cast<double2*>(x + 4 * i) = make_double2(v[0], v[1]);
    *reinterpret_cast<double2*>(x + 4 * i + 2) = make_double2(v[2], v[3]);
}

template <typename T>
__device__ __forceinline__ void put3(T* x, int64_t i, T a, T b, T d) {
    const double v[4] = {(double)a, (double)b, (double)d, 0.0};
    set4(x, i, v);
}

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned int* p, unsigned int v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Waits (acquire loads) until row c is ready for sweep `epoch`; false after the spin limit.
__device__ __forceinline__ bool wait_ready(const unsigned int* flags, int32_t c, unsigned int epoch) {
    if (ld_acquire(flags + c) >= epoch) return true;
    for (unsigned int k = 0; k < kSpinLimit; ++k) {
        __nanosleep(64);
        if (ld_acquire(flags + c) >= epoch) return true;
    }
    return false;
}

// this lane's 4 slots of step g: acc += V_b x[col_b] (x read coherently through L2). With
// `flags`, each column's ready flag is awaited first (dataflow sweeps).
template <typename M, typename T>
__device__ __forceinline__ bool step(const M* __restrict__ vals, const int32_t* __restrict__ col,
                                     int64_t g, const T* x, int lane, T& a0, T& a1, T& a2,
                                     const unsigned int* flags = nullptr, unsigned int epoch = 0) {
    const int4 c4 = __ldg(reinterpret_cast<const int4*>(col + g * kStepSlots + 4 * lane));
    const M* V = vals + g * 9 * kStepSlots + 4 * lane;
    M v[9][4];
#pragma unroll
    for (int k = 0; k < 9; ++k) ldv4(V + k * kStepSlots, v[k]);
    const int32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
    bool ok = true;
    if (flags) {
#pragma unroll
        for (int j = 0; j < 4; ++j) ok = wait_ready(flags, cc[j], epoch) && ok;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        T x0, x1, x2;
        node3_cg<T>(x, cc[j], x0, x1, x2);
        a0 += (T)v[0][j] * x0 + (T)v[1][j] * x1 + (T)v[2][j] * x2;
        a1 += (T)v[3][j] * x0 + (T)v[4][j] * x1 + (T)v[5][j] * x2;
        a2 += (T)v[6][j] * x0 + (T)v[7][j] * x1 + (T)v[8][j] * x2;
    }
    return ok;
}

template <typename T, int LPR>
__device__ __forceinline__ void lanes_sum(T& a0, T& a1, T& a2) {
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
}

// block partial of a grid reduction into partials[slot * G + block]
__device__ __forceinline__ void publish(double v, double* partials, int slot, double* sh) {
    const double t = block_sum(v, sh);
    if (threadIdx.x == 0) partials[slot * gridDim.x + blockIdx.x] = t;
}

// after a grid barrier: the ordered total of slot `slot`, identical in every block and thread
__device__ __forceinline__ double grid_total(const double* partials, int slot) {
    const int lane = threadIdx.x & 31;
    double t = 0.0;
    for (int k = lane; k < (int)gridDim.x; k += 32) t += __ldcg(partials + slot * gridDim.x + k);
    return warp_sum(t);
}

// y = K x over the full layout, one warp per slice; returns this thread's share of x . y. With
// b, writes the residual y = b - K x instead and returns its share of ||y||^2.
template <typename M, typename T, int LPR>
__device__ __forceinline__ double spmv_phase(const SellDev& A, const M* vals, const T* x, T* y,
                                             const double* b = nullptr) {
    const int lane = threadIdx.x & 31, r = lane / LPR, q = lane % LPR;
    constexpr int S = 32 / LPR;
    const int32_t nw = (int32_t)(gridDim.x * kPW);
    double loc = 0.0;
    for (int32_t sl = (int32_t)(blockIdx.x * kPW + (threadIdx.x >> 5)); sl < A.nslices; sl += nw) {
        const int32_t row = A.rowid[(int64_t)sl * S + r];
        T a0 = 0, a1 = 0, a2 = 0;
        const int64_t g1 = A.off[sl + 1];
        for (int64_t g = A.off[sl]; g < g1; ++g) step<M, T>(vals, A.col, g, x, lane, a0, a1, a2);
        lanes_sum<T, LPR>(a0, a1, a2);
        if (q == 0 && row >= 0) {
            if (b) {
                double bv[4];
                get4(b, row, bv);
                a0 = (T)(bv[0] - (double)a0);
                a1 = (T)(bv[1] - (double)a1);
                a2 = (T)(bv[2] - (double)a2);
                loc += (double)a0 * (double)a0 + (double)a1 * (double)a1 + (double)a2 * (double)a2;
            } else {
                T x0, x1, x2;
                node3_cg<T>(x, row, x0, x1, x2);
                loc += (double)x0 * (double)a0 + (double)x1 * (double)a1 + (double)x2 * (double)a2;
            }
            put3(y, row, a0, a1, a2);
        }
    }
    return loc;
}

// One dataflow sweep, one warp per slice. Warp w of the grid takes slices k = w, w + W, ... of
// `seq` (slice ids in dependency order: levels ascending forward, descending backward), a fixed
// round-robin schedule: the smallest unfinished slice always belongs to a warp that has finished
// all its earlier slices, and everything it depends on comes earlier in `seq`, so the sweep
// always progresses; the schedule is also fixed from run to run, which keeps the r . z partial
// sums deterministic. Before gathering a neighbour a lane waits for its ready flag (acquire);
// after writing a row it publishes the row's flag (release). Returns this thread's share of
// r . z (backward); `ok` turns false when a wait hit the spin limit.
template <typename T, int LPR, bool FWD>
__device__ __forceinline__ double sweep(const SellDev& A, int32_t nslices, const int32_t* seq,
                                        unsigned int* flags, unsigned int epoch, const T* vals,
                                        const T* D, int32_t nb, const T* r, T* z, bool& ok) {
    const int lane = threadIdx.x & 31, rr = lane / LPR, q = lane % LPR;
    constexpr int S = 32 / LPR;
    const int32_t nw = (int32_t)(gridDim.x * kPW);
    double loc = 0.0;
    for (int32_t k = (int32_t)(blockIdx.x * kPW + (threadIdx.x >> 5)); k < nslices; k += nw) {
        const int32_t sl = seq ? __ldg(seq + k) : k;
        const int32_t row = __ldg(A.rowid + (int64_t)sl * S + rr);
        // the row's right-hand side and diagonal block, loaded while the steps run
        T t0 = 0, t1 = 0, t2 = 0, d0 = 0, d3 = 0, d4 = 0, d6 = 0, d7 = 0, d8 = 0;
        if (q == 0 && row >= 0) {
            node3_cg<T>(FWD ? r : z, row, t0, t1, t2);
            const T* d = D + row;
            d0 = __ldg(d);
            d3 = __ldg(d + 3 * (int64_t)nb);
            d4 = __ldg(d + 4 * (int64_t)nb);
            d6 = __ldg(d + 6 * (int64_t)nb);
            d7 = __ldg(d + 7 * (int64_t)nb);
            d8 = __ldg(d + 8 * (int64_t)nb);
        }
        T a0 = 0, a1 = 0, a2 = 0;
        const int64_t g1 = __ldg(A.off + sl + 1);
        for (int64_t g = __ldg(A.off + sl); g < g1; ++g)
            ok = step<T, T>(vals, A.col, g, z, lane, a0, a1, a2, flags, epoch) && ok;
        lanes_sum<T, LPR>(a0, a1, a2);
        if (q == 0 && row >= 0) {
            const T u0 = t0 - a0, u1 = t1 - a1, u2 = t2 - a2;
            if (FWD) {
                // y = L_II^-1 (r - sum L y)
                put3(z, row, d0 * u0, d3 * u0 + d4 * u1, d6 * u0 + d7 * u1 + d8 * u2);
            } else {
                // z = L_II^-T (y - sum L^T z), and r . z
                const T z0 = d0 * u0 + d3 * u1 + d6 * u2, z1 = d4 * u1 + d7 * u2, z2 = d8 * u2;
                put3(z, row, z0, z1, z2);
                T r0, r1, r2;
                node3_cg<T>(r, row, r0, r1, r2);
                loc += (double)r0 * (double)z0 + (double)r1 * (double)z1 + (double)r2 * (double)z2;
            }
            st_release(flags + row, epoch);  // orders the row's stores before its flag
        }
    }
    return loc;
}

struct Local {
    double alpha, beta, rz, rr, bb, tol, maxr, delta, rr_true;
    int32_t iter, max_iter, done, status, updates;
    unsigned int epoch;
};

__device__ __forceinline__ unsigned long long gtime() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <typename T, int LPRK, int LPRLU, bool MIXED>
__global__ void __launch_bounds__(kPW * 32, sizeof(T) == 4 ? 4 : 2) k_pcg(PcgArgs<T> a, int init) {
    __shared__ double sh[kPW];
    cg::grid_group grid = cg::this_grid();
    PcgScalars* s = a.s;
    Local v{s->alpha, s->beta, s->rz, s->rr, s->bb, s->tol, s->maxr, s->delta, s->rr_true,
            s->iter, s->max_iter, s->done, s->status, s->updates, s->epoch};
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
    const bool timed = a.timing != nullptr && blockIdx.x == 0 && threadIdx.x == 0;
    unsigned long long t_last = timed ? gtime() : 0;
    auto mark = [&](int phase) {
        if (timed) {
            const unsigned long long t = gtime();
            a.timing[phase] += t - t_last;
            t_last = t;
        }
    };
    int* timeout = reinterpret_cast<int*>(a.claim + 2);
    int it = 0;
    while (!v.done && (init ? it < 1 : it < a.chunk)) {
        double loc;
        if (!init) {
            // ap = K p, alpha = rz / p.ap (iterative.rs:223-228)
            loc = spmv_phase<T, T, LPRK>(a.K, a.Kv, a.p, a.ap);
            publish(loc, a.partials, 0, sh);
            grid.sync();
            mark(0);
            const double pap = grid_total(a.partials, 0);
            v.iter += 1;
            if (isnan(pap) || pap <= 0.0) {
                v.done = 1;
                v.status = 1;
                break;
            }
            v.alpha = v.rz / pap;
            // x += alpha p, r -= alpha ap, ||r||^2 (iterative.rs:229-233)
            loc = 0.0;
            for (int64_t i = tid; i < a.nb; i += nthreads) {
                double xv[4], rv[4], pv[4], av[4];
                get4(a.x, i, xv);
                get4(a.r, i, rv);
                get4(a.p, i, pv);
                get4(a.ap, i, av);
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    xv[c] = (double)(T)(xv[c] + v.alpha * pv[c]);
                    rv[c] = (double)(T)(rv[c] - v.alpha * av[c]);
                    loc += rv[c] * rv[c];
                }
                set4(a.x, i, xv);
                set4(a.r, i, rv);
            }
            publish(loc, a.partials, 1, sh);
            grid.sync();
            mark(1);
            v.rr = grid_total(a.partials, 1);
            const bool small = sqrt(v.rr) <= v.tol * sqrt(v.bb);
            if (!MIXED) {
                if (small) {
                    v.done = 1;
                    break;
                }
                if (v.iter >= v.max_iter) {
                    v.done = 1;
                    v.status = 2;
                    break;
                }
            } else if (small || sqrt(v.rr) < v.delta * v.maxr || v.iter >= v.max_iter) {
                // reliable update: fold x32 into x64, true residual against the FP64 matrix
                for (int64_t i = tid; i < a.nb; i += nthreads) {
                    double xs[4], xd[4];
                    get4(a.x64, i, xd);
                    get4(a.x, i, xs);
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        xd[c] += xs[c];
                        xs[c] = 0.0;
                    }
                    set4(a.x64, i, xd);
                    set4(a.x, i, xs);
                }
                grid.sync();
                loc = spmv_phase<double, double, LPRK>(a.K, a.K64, a.x64, a.r64, a.b64);
                publish(loc, a.partials, 2, sh);
                grid.sync();
                v.rr_true = grid_total(a.partials, 2);
                v.maxr = sqrt(v.rr_true);
                v.updates += 1;
                if (sqrt(v.rr_true) <= v.tol * sqrt(v.bb)) {
                    v.done = 1;
                    break;
                }
                if (v.iter >= v.max_iter) {
                    v.done = 1;
                    v.status = 2;
                    break;
                }
                for (int64_t i = tid; i < a.nb; i += nthreads) {
                    double rv[4];
                    get4(a.r64, i, rv);
                    set4(a.r, i, rv);
                }
                grid.sync();
                mark(2);
            }
        }
        // z = (L L^T)^-1 r (Csr::precondition, iterative.rs:173-188): dataflow sweeps
        bool ok = true;
        v.epoch += 1;
        sweep<T, LPRLU, true>(a.L, a.L.nslices, nullptr, a.flags, v.epoch, a.Lv, a.D, a.nb, a.r,
                              a.z, ok);
        grid.sync();
        mark(3);
        v.epoch += 1;
        loc = sweep<T, LPRLU, false>(a.U, a.U.nslices, a.bwd_seq, a.flags, v.epoch, a.Uv, a.D,
                                     a.nb, a.r, a.z, ok);
        if (!ok) atomicExch(timeout, 1);
        publish(loc, a.partials, 3, sh);
        grid.sync();
        mark(4);
        if (__ldcg(timeout)) {
            v.done = 1;
            v.status = 3;
            break;
        }
        const double rz = grid_total(a.partials, 3);
        v.beta = init ? 0.0 : rz / v.rz;  // iterative.rs:237-239
        v.rz = rz;
        // p = z + beta p (iterative.rs:240-242)
        for (int64_t i = tid; i < a.nb; i += nthreads) {
            double zv[4], pv[4];
            get4(a.z, i, zv);
            get4(a.p, i, pv);
#pragma unroll
            for (int c = 0; c < 4; ++c) pv[c] = (double)(T)(zv[c] + v.beta * pv[c]);
            set4(a.p, i, pv);
        }
        grid.sync();
        mark(5);
        ++it;
    }
    if (timed) a.timing[6] += 1;  // launches
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        s->alpha = v.alpha;
        s->beta = v.beta;
        s->rz = v.rz;
        s->rr = v.rr;
        s->maxr = v.maxr;
        s->rr_true = v.rr_true;
        s->iter = v.iter;
        s->done = v.done;
        s->status = v.status;
        s->updates = v.updates;
        s->epoch = v.epoch;
    }
}

template <typename T, bool MIXED>
void* pick(int lprk, int lprlu) {
#define MAILLE_PICK(K, LU) \
    if (lprk == K && lprlu == LU) return (void*)k_pcg<T, K, LU, MIXED>;
    MAILLE_PICK(1, 1) MAILLE_PICK(1, 2) MAILLE_PICK(1, 4) MAILLE_PICK(2, 1) MAILLE_PICK(2, 2)
    MAILLE_PICK(2, 4) MAILLE_PICK(4, 1) MAILLE_PICK(4, 2) MAILLE_PICK(4, 4)
#undef MAILLE_PICK
    return nullptr;
}

}  // namespace

// Grid size of the persistent kernel: every block co-resident (0 when the layout's lanes-per-
// row combination has no instance).
template <typename T, bool MIXED>
int pcg_persistent_grid(int lprk, int lprlu) {
    void* f = pick<T, MIXED>(lprk, lprlu);
    if (!f) return 0;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, kPW * 32, 0);
    return sms * per_sm;
}

template <typename T, bool MIXED>
cudaError_t launch_pcg_persistent(const PcgArgs<T>& a, int grid, bool init, cudaStream_t st) {
    void* f = pick<T, MIXED>(a.K.lpr, a.L.lpr);
    if (!f) return cudaErrorInvalidValue;
    PcgArgs<T> copy = a;
    int in = init ? 1 : 0;
    void* args[] = {&copy, &in};
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    return cudaLaunchCooperativeKernel(f, dim3(grid), dim3(kPW * 32), args, 0, st);
}

template int pcg_persistent_grid<double, false>(int, int);
template int pcg_persistent_grid<float, true>(int, int);
template cudaError_t launch_pcg_persistent<double, false>(const PcgArgs<double>&, int, bool, cudaStream_t);
template cudaError_t launch_pcg_persistent<float, true>(const PcgArgs<float>&, int, bool, cudaStream_t);

}  // namespace maille
