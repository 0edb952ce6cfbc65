// persist.cu -- the whole IC(0)-PCG iteration in one persistent cooperative kernel.
//
// One launch runs up to `chunk` iterations of Pcg::solve (iterative.rs:222-243): the SpMV, the
// x/r update with the stopping test (fused into the IC(0) forward sweep in the mixed form: each
// row takes x += alpha p, r -= alpha ap right before it is swept), the forward and backward
// sweeps and the p update.
// Phases are separated by grid-wide barriers; every block sums the per-block partials of a
// reduction in the same fixed order, so alpha, beta and the stopping decisions are bit-identical
// in every block and the whole grid takes the same branches. The mixed form adds the reliable
// update (x64 += x32, r64 = b - K64 x64 against the FP64 matrix, r32 = r64) on the iterations
// whose FP32 residual fell by `delta` since the last one.
//
// Sweeps are dataflow instead of one barrier per level: warps take slices in level order on a
// fixed round-robin schedule; before gathering a neighbour's value a lane waits until that row
// has been written in the current sweep (epoch): while any record of the warp is stale, one lane
// polls the one likely written last and the warp then re-reads its stale records together (a
// poll by every lane is up to 128 scattered L2 requests per warp, and the waiting warps' polls
// delayed the working warps' own instructions). A slice only depends on slices of earlier
// levels, which come earlier in every warp's schedule, and all warps are co-resident
// (cooperative launch), so every wait ends; each wait is also bounded and reports a timeout
// status instead of spinning forever. How a lane knows a row is ready depends on the precision:
//  * FP32: the sweep vector holds one 16-byte record per node, (z0, z1, z2, tag), written and
//    read as single 128-bit accesses; the tag is the epoch of the sweep that wrote the record.
//    A gather that sees the current tag has the row's values in the same access (the
//    single-transaction property of aligned 16-byte accesses that CUB's decoupled look-back
//    also relies on), so one round trip per gather and no fence.
//  * FP64: (z0, z1, z2, tag) in one 32-byte word, read and written as single 256-bit accesses
//    (sm_100 vector width), aligned to one L2 sector, so the same single-access argument holds.
// The factors use the packed layout (PsellDev): one-step slices of whole rows, a segmented scan
// over the warp instead of a fixed number of lanes per row, so neither padding to a row-length
// multiple nor a chain of steps per row sits on the sweep's critical path.
//
// Vectors written inside the launch are read with ld.global.cg (L2, coherent after a barrier or
// an acquire); matrix data, which no phase writes, through the read-only path.

#include <atomic>
#include <cmath>
#include <cstring>

#include <cooperative_groups.h>

#include "cuda_host.hpp"
#include "reduce.cuh"
#include "sparse.cuh"

namespace cg = cooperative_groups;

namespace maille {

extern std::atomic<long long> g_kernel_launches;

namespace {

constexpr int kPW = 8;                        // warps per block
constexpr unsigned int kSpinLimit = 1u << 22;  // rounds of a wait before a timeout (seconds)

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



// FP32 sweep record of node c: (z0, z1, z2, tag) in one 128-bit access
__device__ __forceinline__ float4 ld_rec(const float* z, int32_t c) {
    float4 v;
    asm volatile("ld.relaxed.gpu.global.v4.f32 {%0,%1,%2,%3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(z + 4 * (int64_t)c)
                 : "memory");
    return v;
}
__device__ __forceinline__ void st_rec(float* z, int32_t c, float a, float b, float d, unsigned int tag) {
    asm volatile("st.relaxed.gpu.global.v4.f32 [%0], {%1,%2,%3,%4};" ::"l"(z + 4 * (int64_t)c), "f"(a),
                 "f"(b), "f"(d), "f"(__uint_as_float(tag))
                 : "memory");
}


// this lane's 4 slots of step g with columns c4: acc += V_b x[col_b] (x read coherently through L2)
template <typename M, typename T>
__device__ __forceinline__ void step(const M* __restrict__ vals, int4 c4, int64_t g, const T* x, int lane,
                                     int32_t pad, T& a0, T& a1, T& a2) {
    const M* V = vals + g * 9 * kStepSlots + 4 * lane;
    M v[9][4];
#pragma unroll
    for (int k = 0; k < 9; ++k) ldv4(V + k * kStepSlots, v[k]);
    const int32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        T x0 = 0, x1 = 0, x2 = 0;
        if (cc[j] != pad) node3_cg<T>(x, cc[j], x0, x1, x2);  // padding slots: zero values, no load
        a0 += (T)v[0][j] * x0 + (T)v[1][j] * x1 + (T)v[2][j] * x2;
        a1 += (T)v[3][j] * x0 + (T)v[4][j] * x1 + (T)v[5][j] * x2;
        a2 += (T)v[6][j] * x0 + (T)v[7][j] * x1 + (T)v[8][j] * x2;
    }
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
        const int64_t g0 = A.off[sl], g1 = A.off[sl + 1];
        // each step's columns are fetched one step ahead, so its gathers wait on L2 only
        int4 cnext = __ldg(reinterpret_cast<const int4*>(A.col + g0 * kStepSlots + 4 * lane));
        for (int64_t g = g0; g < g1; ++g) {
            const int4 c4 = cnext;
            if (g + 1 < g1) cnext = __ldg(reinterpret_cast<const int4*>(A.col + (g + 1) * kStepSlots + 4 * lane));
            step<M, T>(vals, c4, g, x, lane, A.pad, a0, a1, a2);
        }
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

// ---- dataflow sweeps on the packed layout -------------------------------------------------

// Sweep records: (z0, z1, z2, tag) per node, 16 bytes in FP32 and 32 bytes in FP64, each
// written and read as one vector access and carrying the epoch of the sweep that wrote it, so a
// reader that sees the current tag has the row's current values.
struct Rec32 {
    float4 q;
};
struct Rec64 {
    double x, y, z, w;
};
__device__ __forceinline__ Rec32 ld_record(const float* z, int32_t c) { return Rec32{ld_rec(z, c)}; }
__device__ __forceinline__ Rec64 ld_record(const double* z, int32_t c) {
    Rec64 v;
    asm volatile("ld.relaxed.gpu.global.v4.f64 {%0,%1,%2,%3}, [%4];"
                 : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w)
                 : "l"(z + 4 * (int64_t)c)
                 : "memory");
    return v;
}
__device__ __forceinline__ bool ready(const Rec32& r, unsigned int epoch) {
    return __float_as_uint(r.q.w) >= epoch;
}
__device__ __forceinline__ bool ready(const Rec64& r, unsigned int epoch) {
    return (unsigned long long)__double_as_longlong(r.w) >= epoch;
}
__device__ __forceinline__ void values(const Rec32& r, float& a, float& b, float& d) {
    a = r.q.x; b = r.q.y; d = r.q.z;
}
__device__ __forceinline__ void values(const Rec64& r, double& a, double& b, double& d) {
    a = r.x; b = r.y; d = r.z;
}
template <typename T>
struct RecOf;
template <>
struct RecOf<float> { using type = Rec32; };
template <>
struct RecOf<double> { using type = Rec64; };
// the record of a padding slot: zero values, always current (padding needs no load)
template <typename T>
__device__ __forceinline__ typename RecOf<T>::type pad_record();
template <>
__device__ __forceinline__ Rec32 pad_record<float>() {
    return Rec32{make_float4(0.f, 0.f, 0.f, __uint_as_float(0xFFFFFFFFu))};
}
template <>
__device__ __forceinline__ Rec64 pad_record<double>() {
    return Rec64{0.0, 0.0, 0.0, __longlong_as_double(-1ll)};
}

// Waits until the 4 records q (read from z at columns cc) carry `epoch`; called by the whole warp.
// While any lane has a record that is not current, one lane polls the warp's pending record that
// is usually written last (rows are numbered by level: the largest column in a forward sweep, the
// smallest in a backward one), then every lane re-reads its pending records together (one L2
// round trip), and so on; at most `limit` polls in all; false when the limit ran out. Polling with one lane instead of every lane's
// records matters: a warp-wide poll of 128 scattered records is 128 L2 requests, and the waiting
// warps' polls queued ahead of the working warps' own loads and shuffles (Tet4 20^3 FP64: the
// sweeps' per-level time fell from 9 us to 4 us; Tet10 40^3: the mixed step 11 % shorter).
template <typename T>
__device__ __forceinline__ bool await_records(const T* z, const int32_t cc[4], unsigned int epoch,
                                              typename RecOf<T>::type q[4], unsigned int limit, bool fwd) {
    bool pending = false;
#pragma unroll
    for (int j = 0; j < 4; ++j) pending = pending || !ready(q[j], epoch);
    unsigned int k = 0;
    while (__any_sync(0xffffffffu, pending) && k < limit) {
        // the pending column to poll: largest (forward) or smallest (backward), as an unsigned
        // maximum of c or of ~c
        uint32_t key = 0u;
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (!ready(q[j], epoch)) key = max(key, fwd ? (uint32_t)cc[j] + 1u : ~(uint32_t)cc[j]);
        key = __reduce_max_sync(0xffffffffu, key);
        const int32_t mc = fwd ? (int32_t)(key - 1u) : (int32_t)~key;
        if ((threadIdx.x & 31) == 0) {
            typename RecOf<T>::type w = ld_record(z, mc);
            while (!ready(w, epoch) && k < limit) {
                w = ld_record(z, mc);
                ++k;
            }
        }
        k = __shfl_sync(0xffffffffu, k, 0) + 1;
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (!ready(q[j], epoch)) q[j] = ld_record(z, cc[j]);
        pending = false;
#pragma unroll
        for (int j = 0; j < 4; ++j) pending = pending || !ready(q[j], epoch);
    }
    return !pending;
}

// Self-test of the bounded wait: one warp awaits records 0..3 of z for `epoch` with at most `limit`
// rounds and lane 0 writes 1 to *timed_out when the wait ran out, 0 when every record was
// current. Nothing else writes z meanwhile, so a record whose tag is below `epoch` stays stale.
__global__ void k_wait_selftest(const float* z, unsigned int epoch, unsigned int limit, int32_t* timed_out) {
    const int32_t cc[4] = {0, 1, 2, 3};
    Rec32 q[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) q[j] = ld_record(z, cc[j]);
    const bool ok = await_records<float>(z, cc, epoch, q, limit, true);
    if ((threadIdx.x & 31) == 0) *timed_out = ok ? 0 : 1;
}

// publishes row `row` of the sweep output for sweep `epoch`
__device__ __forceinline__ void publish_row(float* z, int32_t row, float a, float b, float d, unsigned int epoch) {
    st_rec(z, row, a, b, d, epoch);
}
__device__ __forceinline__ void publish_row(double* z, int32_t row, double a, double b, double d, unsigned int epoch) {
    asm volatile("st.relaxed.gpu.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(z + 4 * (int64_t)row), "d"(a),
                 "d"(b), "d"(d), "d"(__longlong_as_double((long long)epoch))
                 : "memory");
}
// values of row i of a sweep record vector (plain loads: callers read after a grid barrier)
__device__ __forceinline__ void rec_get(const float* z, int64_t i, double v[3]) {
    const float4 q = __ldcg(reinterpret_cast<const float4*>(z + 4 * i));
    v[0] = q.x; v[1] = q.y; v[2] = q.z;
}
__device__ __forceinline__ void rec_get(const double* z, int64_t i, double v[3]) {
    const double2 q = __ldcg(reinterpret_cast<const double2*>(z + 4 * i));
    v[0] = q.x; v[1] = q.y; v[2] = __ldcg(z + 4 * i + 2);
}

// ---- staging of the factor values: TMA bulk copies into a per-warp shared buffer ------------

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// one 1-D bulk copy global -> shared (16-byte aligned addresses, size a multiple of 16) that
// completes on `bar`; the issuing lane also arrives on `bar`, announcing the bytes
__device__ __forceinline__ void bulk_stage(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// Waits for phase `parity` of `bar` to complete; false after the spin limit. A bulk copy from
// global memory depends on nothing else, so the wait ends; the bound only guards against a hang.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (unsigned int k = 0; k < kSpinLimit; ++k)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void lds4(const float* p, float v[4]) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void lds4(const double* p, double v[4]) {
    const double2 a = *reinterpret_cast<const double2*>(p);
    const double2 b = *reinterpret_cast<const double2*>(p + 2);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

// Per-warp staging state of a sweep: the warp's shared buffer (one step: 9 planes x 128 slots),
// its mbarrier and the phase parity the next wait expects.
template <typename T>
struct Stage {
    T* buf;
    uint64_t* bar;
    uint32_t phase;
};
// starts the bulk copy of step g's values (9 planes x 128 slots) into the warp's buffer
template <typename T>
__device__ __forceinline__ void stage_step(const T* vals, int64_t g, Stage<T>& st) {
    constexpr uint32_t kBytes = 9 * kStepSlots * sizeof(T);
    bulk_stage(st.buf, vals + g * 9 * kStepSlots, kBytes, st.bar);
}

// The first read of this lane's 4 records of a step (columns c4; padding slots need none).
template <typename T>
__device__ __forceinline__ void issue_records(int4 c4, const T* z, int32_t pad, typename RecOf<T>::type q[4]) {
    const int32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) q[j] = cc[j] == pad ? pad_record<T>() : ld_record(z, cc[j]);
}

// One step of a packed slice for this lane's 4 slots: P[j] = V_j z[col_j], every column first
// awaited for sweep `epoch`; false when a wait hit the spin limit. The step's values are already on
// their way into the warp's buffer (a bulk copy started when the buffer last became free), the
// lane's columns were fetched ahead and its records q requested by issue_records, so their L2
// round trip is the step's only wait. Once every lane has read the buffer, lane 0 starts the copy
// of step `next` (the next step of this slice or the first of the warp's next slice; < 0: none).
// `fwd`: the sweep's direction, which tells the wait which pending record to poll.
template <typename T>
__device__ __forceinline__ bool slot_products(const T* __restrict__ vals, int4 c4, const T* z,
                                              unsigned int epoch, int lane, Stage<T>& st,
                                              int64_t next, typename RecOf<T>::type q[4], T P[4][3], bool fwd) {
    const int32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
    bool ok = await_records<T>(z, cc, epoch, q, kSpinLimit, fwd);
    ok = mbar_wait(st.bar, st.phase) && ok;
    st.phase ^= 1u;
    const T* V = st.buf + 4 * lane;
#pragma unroll
    for (int j = 0; j < 4; ++j) P[j][0] = P[j][1] = P[j][2] = 0;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        T v[4];
        lds4(V + k * kStepSlots, v);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            T x0, x1, x2;
            values(q[j], x0, x1, x2);
            const T x = k % 3 == 0 ? x0 : (k % 3 == 1 ? x1 : x2);
            P[j][k / 3] += v[j] * x;
        }
    }
    __syncwarp();  // every lane has read the buffer before lane 0 refills it
    if (lane == 0 && next >= 0) stage_step(vals, next, st);
    return ok;
}

// position of the n-th (0-based) set bit of m (m has more than n bits set)
__device__ __forceinline__ int nth_set(uint32_t m, int n) {
    int pos = 0, c = __popc(m & 0xFFFFu);
    if (n >= c) { n -= c; m >>= 16; pos += 16; }
    c = __popc(m & 0xFFu);
    if (n >= c) { n -= c; m >>= 8; pos += 8; }
    c = __popc(m & 0xFu);
    if (n >= c) { n -= c; m >>= 4; pos += 4; }
    c = __popc(m & 0x3u);
    if (n >= c) { n -= c; m >>= 2; pos += 2; }
    if (n >= (int)(m & 1u)) pos += 1;
    return pos;
}
__device__ __forceinline__ int nth_set(uint4 h, int n) {
    int c = __popc(h.x);
    if (n < c) return nth_set(h.x, n);
    n -= c;
    c = __popc(h.y);
    if (n < c) return 32 + nth_set(h.y, n);
    n -= c;
    c = __popc(h.z);
    if (n < c) return 64 + nth_set(h.z, n);
    return 96 + nth_set(h.w, n - c);
}
__device__ __forceinline__ uint32_t head_bits(uint4 h, int lane) {
    const int w = lane >> 3;
    const uint32_t word = w == 0 ? h.x : w == 1 ? h.y : w == 2 ? h.z : h.w;
    return (word >> ((lane & 7) * 4)) & 0xFu;
}

// The right-hand side and diagonal inverse of one sweep row: t = (FWD ? r : y) at the row; D is
// 9 planes of nb entries, lower triangular (entries 0, 3, 4, 6, 7, 8).
// The PCG update a fused forward sweep applies to each row before sweeping it.
template <typename T>
struct XrUpdate {
    double alpha;
    T *x, *r;
    const T *p, *ap;
};

template <typename T, bool FWD, bool FUSED = false>
struct RowIn {
    T t0, t1, t2, d0, d3, d4, d6, d7, d8;
    T q0, q1, q2;  // backward: r at the row, for r . z; fused forward: x at the row
    T w0, w1, w2;  // fused forward: ap at the row
    T s0, s1, s2;  // fused forward: p at the row
    __device__ __forceinline__ void load(int32_t row, const T* D, int32_t nb, const T* r, const T* z,
                                         const XrUpdate<T>& upd) {
        if (FWD) {
            node3_cg<T>(r, row, t0, t1, t2);
            if (FUSED) {
                node3_cg<T>(upd.x, row, q0, q1, q2);
                node3_cg<T>(upd.ap, row, w0, w1, w2);
                node3_cg<T>(upd.p, row, s0, s1, s2);
            }
        } else {
            double v[3];
            rec_get(z, row, v);
            t0 = (T)v[0]; t1 = (T)v[1]; t2 = (T)v[2];
            node3_cg<T>(r, row, q0, q1, q2);
        }
        const T* d = D + row;
        d0 = __ldg(d);
        d3 = __ldg(d + 3 * (int64_t)nb);
        d4 = __ldg(d + 4 * (int64_t)nb);
        d6 = __ldg(d + 6 * (int64_t)nb);
        d7 = __ldg(d + 7 * (int64_t)nb);
        d8 = __ldg(d + 8 * (int64_t)nb);
    }
    // forward: y = L_II^-1 (r - sum L y); backward: z = L_II^-T (y - sum L^T z) and r . z.
    // Fused forward: the row first takes its PCG update x += alpha p, r -= alpha ap (rounded to T
    // like the separate update phase, iterative.rs:229-232), writes x and r, sweeps with the new r
    // and returns its ||r||^2 share.
    __device__ __forceinline__ double finish(int32_t row, T a0, T a1, T a2, const T* r, T* z,
                                             unsigned int epoch, const XrUpdate<T>& upd) const {
        if (FWD && FUSED) {
            const double al = upd.alpha;
            const T r0 = (T)((double)t0 - al * (double)w0), r1 = (T)((double)t1 - al * (double)w1),
                    r2 = (T)((double)t2 - al * (double)w2);
            put3(upd.x, row, (T)((double)q0 + al * (double)s0), (T)((double)q1 + al * (double)s1),
                 (T)((double)q2 + al * (double)s2));
            put3(upd.r, row, r0, r1, r2);
            const T u0 = r0 - a0, u1 = r1 - a1, u2 = r2 - a2;
            publish_row(z, row, d0 * u0, d3 * u0 + d4 * u1, d6 * u0 + d7 * u1 + d8 * u2, epoch);
            return (double)r0 * (double)r0 + (double)r1 * (double)r1 + (double)r2 * (double)r2;
        }
        const T u0 = t0 - a0, u1 = t1 - a1, u2 = t2 - a2;
        if (FWD) {
            publish_row(z, row, d0 * u0, d3 * u0 + d4 * u1, d6 * u0 + d7 * u1 + d8 * u2, epoch);
            return 0.0;
        }
        const T z0 = d0 * u0 + d3 * u1 + d6 * u2, z1 = d4 * u1 + d7 * u2, z2 = d8 * u2;
        publish_row(z, row, z0, z1, z2, epoch);
        return (double)q0 * (double)z0 + (double)q1 * (double)z1 + (double)q2 * (double)z2;
    }
};

// Slice bookkeeping a warp fetches ahead: the slice's steps [g0, g1), its packed rows [r0, r1)
// and its row-start bits. Out-of-range slices read as empty.
struct SliceMeta {
    int64_t g0, g1;
    int32_t r0, r1;
    uint4 head;
};
__device__ __forceinline__ SliceMeta slice_meta(const PsellDev& A, int32_t sl) {
    SliceMeta m{0, 0, 0, 0, make_uint4(0u, 0u, 0u, 0u)};
    if (sl < A.nslices) {
        m.g0 = __ldg(A.off + sl);
        m.g1 = __ldg(A.off + sl + 1);
        m.r0 = __ldg(A.row0 + sl);
        m.r1 = __ldg(A.row0 + sl + 1);
        m.head = __ldg(A.head + sl);
    }
    return m;
}
__device__ __forceinline__ int4 lane_cols(const PsellDev& A, int64_t g, int lane) {
    return __ldg(reinterpret_cast<const int4*>(A.col + g * kStepSlots + 4 * lane));
}

// One dataflow sweep over a packed layout whose slices are stored in sweep order, one warp per
// slice. Warp w of the grid takes slices w, w + W, ...: a fixed round-robin schedule in which the
// smallest unfinished slice always belongs to a warp that has finished all its earlier slices, and
// everything it depends on comes earlier, so the sweep always progresses; the schedule is also
// fixed from run to run, which keeps the r . z partial sums deterministic.
// The warp's slice loop is software-pipelined so that a slice's critical path is the L2 round
// trip of its records: the bookkeeping of the slice after next, the columns and owned rows of the
// next slice, the next slice's right-hand sides and diagonal blocks, and (once the buffer frees)
// the next step's values are all requested while the current slice runs, and the slice's own row
// inputs (right-hand sides, diagonal blocks, the update's operands) are requested right after its
// records, so they travel during the records' round trip instead of being carried in registers
// from the previous slice (whose register copy waited for them at the loop's end).
// In a one-step slice (at most 32 rows) lane k owns row k. Each lane forms the products of its 4
// slots and sums them per row inside the lane; a segmented scan over the warp (fixed order)
// carries the partial sums across lanes, and the owner of each row fetches the row's total from
// the lane that holds its last slot. A multi-step slice holds one long row, summed over the warp.
// Returns this thread's share of r . z (backward), or of ||r||^2 for a FUSED forward sweep, in
// which each row first takes the PCG update of `upd` (x += alpha p, r -= alpha ap) and is swept
// with the new r; `ok` turns false when a wait hit the spin limit.
template <typename T, bool FWD, bool FUSED = false>
__device__ __forceinline__ double sweep(const PsellDev& A, unsigned int epoch, const T* vals,
                                        const T* D, int32_t nb, const T* r, T* z, Stage<T>& st,
                                        bool& ok, const XrUpdate<T>& upd = XrUpdate<T>{}) {
    const int lane = threadIdx.x & 31;
    const int32_t nw = (int32_t)(gridDim.x * kPW), n = A.nslices;
    double loc = 0.0;
    int32_t k = (int32_t)(blockIdx.x * kPW + (threadIdx.x >> 5));
    if (k >= n) return loc;
    SliceMeta m0 = slice_meta(A, k), m1 = slice_meta(A, k + nw);
    int4 c0 = lane_cols(A, m0.g0, lane);
    int32_t row0 = lane < m0.r1 - m0.r0 ? __ldg(A.rows + m0.r0 + lane) : -1;
    if (lane == 0) stage_step(vals, m0.g0, st);
    using R = typename RecOf<T>::type;
    for (; k < n; k += nw) {
        const bool more = k + nw < n;
        const SliceMeta m2 = slice_meta(A, k + 2 * nw);
        int4 c1 = make_int4(nb, nb, nb, nb);
        int32_t row1 = -1;
        if (more) {
            c1 = lane_cols(A, m1.g0, lane);
            if (lane < m1.r1 - m1.r0) row1 = __ldg(A.rows + m1.r0 + lane);
        }
        const int64_t next_slice = more ? m1.g0 : -1;
        T a0 = 0, a1 = 0, a2 = 0;
        RowIn<T, FWD, FUSED> in{};
        if (m0.g1 - m0.g0 == 1) {
            R q[4];
            issue_records<T>(c0, z, A.pad, q);
            if (row0 >= 0) in.load(row0, D, nb, r, z, upd);
            const int32_t nrows = m0.r1 - m0.r0;
            const uint32_t mine = head_bits(m0.head, lane);
            const int last = lane + 1 < nrows ? nth_set(m0.head, lane + 1) - 1 : 127;
            T P[4][3];
            ok = slot_products(vals, c0, z, epoch, lane, st, next_slice, q, P, FWD) && ok;
            // in-lane running sums, restarted at each row start; the lane's carry-out is the sum
            // of its slots after its last row start (all 4 when none starts here)
            T s0 = 0, s1 = 0, s2 = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if ((mine >> j) & 1u) s0 = s1 = s2 = 0;
                s0 += P[j][0]; s1 += P[j][1]; s2 += P[j][2];
                P[j][0] = s0; P[j][1] = s1; P[j][2] = s2;
            }
            // segmented inclusive scan of the carry-outs over the warp
            int f = mine != 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const T u0 = __shfl_up_sync(0xffffffffu, s0, o);
                const T u1 = __shfl_up_sync(0xffffffffu, s1, o);
                const T u2 = __shfl_up_sync(0xffffffffu, s2, o);
                const int fu = __shfl_up_sync(0xffffffffu, f, o);
                if (lane >= o) {
                    if (!f) { s0 += u0; s1 += u1; s2 += u2; }
                    f |= fu;
                }
            }
            // the open row's sum over the lanes before this one completes the slots before the
            // lane's first row start
            T i0 = __shfl_up_sync(0xffffffffu, s0, 1), i1 = __shfl_up_sync(0xffffffffu, s1, 1),
              i2 = __shfl_up_sync(0xffffffffu, s2, 1);
            if (lane == 0) i0 = i1 = i2 = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if ((mine & ((2u << j) - 1u)) == 0) {
                    P[j][0] += i0; P[j][1] += i1; P[j][2] += i2;
                }
            // the owner of each row takes the sum at the row's last slot
            const int src = last >> 2, js = last & 3;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const T v0 = __shfl_sync(0xffffffffu, P[j][0], src);
                const T v1 = __shfl_sync(0xffffffffu, P[j][1], src);
                const T v2 = __shfl_sync(0xffffffffu, P[j][2], src);
                if (j == js) { a0 = v0; a1 = v1; a2 = v2; }
            }
        } else {
            if (row0 >= 0) in.load(row0, D, nb, r, z, upd);
            for (int64_t g = m0.g0; g < m0.g1; ++g) {
                const int4 cg4 = g == m0.g0 ? c0 : lane_cols(A, g, lane);
                R q[4];
                issue_records<T>(cg4, z, A.pad, q);
                T P[4][3];
                ok = slot_products(vals, cg4, z, epoch, lane, st, g + 1 < m0.g1 ? g + 1 : next_slice, q, P, FWD) && ok;
#pragma unroll
                for (int j = 0; j < 4; ++j) { a0 += P[j][0]; a1 += P[j][1]; a2 += P[j][2]; }
            }
            lanes_sum<T, 32>(a0, a1, a2);
        }
        if (row0 >= 0) loc += in.finish(row0, a0, a1, a2, r, z, epoch, upd);
        m0 = m1;
        m1 = m2;
        c0 = c1;
        row0 = row1;
    }
    return loc;
}

// The FP32 SpMV of the mixed form with its values staged through shared memory: the warp's steps
// (slice after slice, in its round-robin order) stream through two buffers by TMA bulk copies,
// the copy of step k + 2 starting as soon as step k's buffer has been read, so two steps (9 KB)
// per warp are in flight without holding registers. Columns are fetched one step ahead and the
// gathers of a step are requested before its values are awaited. Same arithmetic and summation
// order as spmv_phase; returns this thread's share of x . y.
template <int LPR>
__device__ __forceinline__ double spmv_staged(const SellDev& A, const float* __restrict__ vals,
                                              const float* x, float* y, float* buf, uint64_t* bars,
                                              uint32_t& phases) {
    const int lane = threadIdx.x & 31, r = lane / LPR, q = lane % LPR;
    constexpr int S = 32 / LPR;
    constexpr uint32_t kBytes = 9 * kStepSlots * sizeof(float);
    const int32_t nw = (int32_t)(gridDim.x * kPW), n = A.nslices;
    int32_t sl = (int32_t)(blockIdx.x * kPW + (threadIdx.x >> 5));
    double loc = 0.0;
    if (sl >= n) return loc;
    // staging cursor of lane 0: the next step to copy, walking the warp's slices
    int32_t cs = sl;
    int64_t cg = __ldg(A.off + sl), cg1 = __ldg(A.off + sl + 1);
    auto stage_next = [&](int b) {
        if (cs >= n) return;
        bulk_stage(buf + b * 9 * kStepSlots, vals + cg * 9 * kStepSlots, kBytes, &bars[b]);
        if (++cg == cg1) {
            cs += nw;
            if (cs < n) {
                cg = __ldg(A.off + cs);
                cg1 = __ldg(A.off + cs + 1);
            }
        }
    };
    if (lane == 0) {
        stage_next(0);
        stage_next(1);
    }
    int b = 0;
    for (; sl < n; sl += nw) {
        const int32_t row = A.rowid[(int64_t)sl * S + r];
        float a0 = 0, a1 = 0, a2 = 0;
        const int64_t g0 = A.off[sl], g1 = A.off[sl + 1];
        int4 cnext = __ldg(reinterpret_cast<const int4*>(A.col + g0 * kStepSlots + 4 * lane));
        for (int64_t g = g0; g < g1; ++g) {
            const int4 c4 = cnext;
            if (g + 1 < g1) cnext = __ldg(reinterpret_cast<const int4*>(A.col + (g + 1) * kStepSlots + 4 * lane));
            const int32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
            float xv[4][3];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                xv[j][0] = xv[j][1] = xv[j][2] = 0.f;
                if (cc[j] != A.pad) node3_cg<float>(x, cc[j], xv[j][0], xv[j][1], xv[j][2]);
            }
            mbar_wait(&bars[b], (phases >> b) & 1u);
            phases ^= 1u << b;
            const float* V = buf + b * 9 * kStepSlots + 4 * lane;
            float v[9][4];
#pragma unroll
            for (int k = 0; k < 9; ++k) lds4(V + k * kStepSlots, v[k]);
            __syncwarp();  // every lane has read the buffer before lane 0 refills it
            if (lane == 0) stage_next(b);
            b ^= 1;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                a0 += v[0][j] * xv[j][0] + v[1][j] * xv[j][1] + v[2][j] * xv[j][2];
                a1 += v[3][j] * xv[j][0] + v[4][j] * xv[j][1] + v[5][j] * xv[j][2];
                a2 += v[6][j] * xv[j][0] + v[7][j] * xv[j][1] + v[8][j] * xv[j][2];
            }
        }
        lanes_sum<float, LPR>(a0, a1, a2);
        if (q == 0 && row >= 0) {
            float x0, x1, x2;
            node3_cg<float>(x, row, x0, x1, x2);
            loc += (double)x0 * (double)a0 + (double)x1 * (double)a1 + (double)x2 * (double)a2;
            put3(y, row, a0, a1, a2);
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

template <typename T, int LPRK, bool MIXED>
__global__ void __launch_bounds__(kPW * 32, 2) k_pcg(PcgArgs<T> a, int init) {
    __shared__ double sh[kPW];
    __shared__ uint64_t bars[kPW];
    __shared__ uint64_t spmv_bars[2 * kPW];  // the two staging buffers of the mixed form's SpMV
    extern __shared__ __align__(128) unsigned char stage_mem[];  // kPW x one step of factor values
    cg::grid_group grid = cg::this_grid();
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        mbar_init(&bars[warp]);
        mbar_init(&spmv_bars[2 * warp]);
        mbar_init(&spmv_bars[2 * warp + 1]);
    }
    uint32_t spmv_phases = 0;
    mbar_init_fence();
    __syncthreads();
    // each warp's buffer: 9 KB (one FP64 step, or two FP32 steps for the staged SpMV)
    Stage<T> stage{reinterpret_cast<T*>(stage_mem + (size_t)warp * 9 * kStepSlots * 8), &bars[warp], 0u};
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
        bool ok = true;
        bool need_fwd = true;  // the plain forward sweep below (not fused with the update)
        if (!init) {
            // ap = K p, alpha = rz / p.ap (iterative.rs:223-228)
            if constexpr (MIXED)
                loc = spmv_staged<LPRK>(a.K, a.Kv, a.p, a.ap, stage.buf, &spmv_bars[2 * warp], spmv_phases);
            else
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
            // x += alpha p, r -= alpha ap and ||r||^2 (iterative.rs:229-233). Mixed form: fused into
            // the forward sweep, each row taking its update right before it is swept with the new
            // r (one grid pass and one barrier less per iteration). Plain form: a separate pass (the
            // FP64 sweep's extra registers cost more than the pass; measured both ways).
            if constexpr (MIXED) {
                v.epoch += 1;
                loc = sweep<T, true, true>(a.L, v.epoch, a.Lv, a.D, a.nb, a.r, a.z, stage, ok,
                                           XrUpdate<T>{v.alpha, a.x, a.r, a.p, a.ap});
                if (!ok) atomicExch(timeout, 1);
                publish(loc, a.partials, 1, sh);
                grid.sync();
                mark(3);
                if (__ldcg(timeout)) {
                    v.done = 1;
                    v.status = 3;
                    break;
                }
                need_fwd = false;
            } else {
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
            }
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
                need_fwd = true;  // the fused sweep ran on the recurrence residual: again on the true one
            }
        }
        // z = (L L^T)^-1 r (Csr::precondition, iterative.rs:173-188): dataflow sweeps
        if (need_fwd) {
            v.epoch += 1;
            sweep<T, true>(a.L, v.epoch, a.Lv, a.D, a.nb, a.r, a.z, stage, ok);
            grid.sync();
            mark(3);
        }
        v.epoch += 1;
        loc = sweep<T, false>(a.U, v.epoch, a.Uv, a.D, a.nb, a.r, a.z, stage, ok);
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
            double zv[3], pv[4];
            rec_get(a.z, i, zv);
            get4(a.p, i, pv);
#pragma unroll
            for (int c = 0; c < 3; ++c) pv[c] = (double)(T)(zv[c] + v.beta * pv[c]);
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

// dynamic shared memory of the persistent kernel: one staged step of factor values per warp
template <typename T>
constexpr size_t stage_bytes() {
    // one step of FP64 values (9 KB) per warp; two FP32 steps in the mixed form's staged SpMV
    return (size_t)kPW * 9 * kStepSlots * 8;
}

template <typename T, bool MIXED>
void* pick(int lprk) {
    if (lprk == 1) return (void*)k_pcg<T, 1, MIXED>;
    if (lprk == 2) return (void*)k_pcg<T, 2, MIXED>;
    if (lprk == 4) return (void*)k_pcg<T, 4, MIXED>;
    return nullptr;
}

}  // namespace

// Runs k_wait_selftest on 4 FP32 records whose tags are `tags` for `epoch` with at most `limit`
// rounds; *timed_out tells whether the wait ran out. Throws CudaFailure on a CUDA error.
void wait_selftest(const unsigned int tags[4], unsigned int epoch, unsigned int limit, int32_t* timed_out) {
    float host[16] = {};
    for (int j = 0; j < 4; ++j) std::memcpy(&host[4 * j + 3], &tags[j], sizeof(unsigned int));
    float* z = dalloc<float>(16);
    int32_t* flag = dalloc<int32_t>(1);
    CK(cudaMemcpy(z, host, sizeof(host), cudaMemcpyHostToDevice));
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    k_wait_selftest<<<1, 32>>>(z, epoch, limit, flag);
    CK(cudaGetLastError());
    CK(cudaMemcpy(timed_out, flag, sizeof(int32_t), cudaMemcpyDeviceToHost));
    dfree(z);
    dfree(flag);
}

// Grid size of the persistent kernel: every block co-resident (0 when the layout's lanes-per-
// row combination has no instance).
template <typename T, bool MIXED>
int pcg_persistent_grid(int lprk) {
    void* f = pick<T, MIXED>(lprk);
    if (!f) return 0;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t smem = stage_bytes<T>();
    if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, kPW * 32, smem);
    return sms * per_sm;
}

template <typename T, bool MIXED>
cudaError_t launch_pcg_persistent(const PcgArgs<T>& a, int grid, bool init, cudaStream_t st) {
    void* f = pick<T, MIXED>(a.K.lpr);
    if (!f) return cudaErrorInvalidValue;
    PcgArgs<T> copy = a;
    int in = init ? 1 : 0;
    void* args[] = {&copy, &in};
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    return cudaLaunchCooperativeKernel(f, dim3(grid), dim3(kPW * 32), args, stage_bytes<T>(), st);
}

template int pcg_persistent_grid<double, false>(int);
template int pcg_persistent_grid<float, true>(int);
template cudaError_t launch_pcg_persistent<double, false>(const PcgArgs<double>&, int, bool, cudaStream_t);
template cudaError_t launch_pcg_persistent<float, true>(const PcgArgs<float>&, int, bool, cudaStream_t);

}  // namespace maille
