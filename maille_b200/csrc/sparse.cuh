// sparse.cuh -- sliced 3x3-block layouts (SELL for K, packed for the factor) and the PCG kernels.
//
// Layout. Rows of one level are cut into warp slices of 32/lpr rows (lpr = lanes per row); in a
// slice every step holds 128 slots, 4 consecutive slots per lane, so a lane reads the 9 values
// of its 4 blocks as 9 128-bit loads (float4, or two double2) and their 4 node columns as one
// int4. Value plane k of step g is vals[(g * 9 + k) * 128 + slot]: every load instruction of the
// warp reads 512 (FP32) or 1024 (FP64) contiguous bytes. A row's blocks are spread over its lpr
// lanes; the lanes of a row are summed with shuffles. Rows inside a level are sorted by length
// (descending) per layout, which keeps the padding of a slice small; rowid maps slice rows to
// matrix rows. Vectors are padded to 4 entries per node, so the x of one block is one 16-byte
// gather (FP32) or a 16 + 8-byte gather (FP64). Vectors hold nb + 1 nodes: node nb is a dummy
// that stays 0 and that padding slots point at.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace maille {

constexpr int kLaneSlots = 4;    // slots (blocks) per lane per step
constexpr int kStepSlots = 128;  // 32 lanes x kLaneSlots

struct SellDev {
    int32_t lpr;            // lanes per row: 1, 2, 4 or 8
    int32_t nslices;
    const int32_t* rowid;   // [nslices * 32 / lpr] matrix row of each slice row, -1 when empty
    const int64_t* off;     // [nslices + 1] first step of each slice
    const int32_t* col;     // [steps * 128] node column of each slot
    int32_t pad;            // column of the padding slots (the dummy node nb, zero values)
};

// Packed layout of a strictly lower or upper factor (PsellHost in common.hpp): one-step slices of
// whole rows (a row may span lanes), row starts marked in a 128-bit mask per slice.
struct PsellDev {
    int32_t nslices;
    const int64_t* off;    // [nslices + 1] first step of each slice
    const int32_t* col;    // [steps * 128] node column of each slot
    const uint4* head;     // [nslices] row-start bits of the 128 slots
    const int32_t* row0;   // [nslices + 1] first packed row of each slice
    const int32_t* rows;   // [nb] matrix row of each packed row
    int32_t pad;           // column of the padding slots (the dummy node nb, zero values)
};

// Device-resident scalars of one PCG run.
struct PcgScalars {
    double alpha, beta, rz, rr, bb, tol, pap;
    double maxr, delta, rr_true;  // reliable updates (mixed form)
    int32_t iter, max_iter, done, status;  // status: 0 ok, 1 singular (also NaN), 2 cap reached
    int32_t update, updates;
    unsigned int ticket[4];
    unsigned int epoch;  // sweep counter of the row-ready flags; never reset (monotonic)
};

// ap = K p on its own (the persistent kernel has its own SpMV phase)
template <typename T>
void launch_spmv(const SellDev& A, const T* vals, const T* p, T* ap, int grid, cudaStream_t st);
void launch_pcg_init(PcgScalars* s, double tol, int32_t max_iter, double delta, cudaStream_t st);
template <typename T>
void launch_norm2(int64_t n, const T* v, double* partials, unsigned int* ticket, double* out,
                  cudaStream_t st);
// vals[slot layout] = csr[src[slot]] (9 entries per block, 0 for padding)
template <typename T>
void launch_sell_fill(int64_t steps, const int32_t* src, const double* csr, T* vals, cudaStream_t st);
// D[k * nb + i] = F[diag[i] * 9 + k]
template <typename T>
void launch_diag_fill(int32_t nb, const int64_t* diag, const double* F, T* D, cudaStream_t st);
void launch_cast(int64_t n, const double* a, float* b, cudaStream_t st);

// The persistent cooperative PCG kernel (persist.cu): arguments, co-resident grid size and launch.
template <typename T>
struct PcgArgs {
    int32_t nb, levels, chunk;
    SellDev K;
    PsellDev L, U;
    const T *Kv, *Lv, *Uv, *D;
    // padded vectors (4 entries per node); z holds the sweep records (z0, z1, z2, tag)
    T *x, *r, *z, *p, *ap;
    const double* K64;  // mixed form: FP64 matrix, right-hand side, solution, true residual
    const double* b64;
    double *x64, *r64;
    PcgScalars* s;
    int32_t* claim;  // claim[2]: the sweeps' timeout flag
    double* partials;       // [4 * grid]
    unsigned long long* timing;  // optional [8] ns per phase (block 0): spmv, axpy, update, fwd, bwd, p
};
template <typename T, bool MIXED>
int pcg_persistent_grid(int lprk);
// Self-test of the sweeps' bounded wait (persist.cu): awaits 4 FP32 records with tags `tags` for
// `epoch` within `limit` rounds; *timed_out = 1 when the wait ran out. Throws CudaFailure.
void wait_selftest(const unsigned int tags[4], unsigned int epoch, unsigned int limit, int32_t* timed_out);
template <typename T, bool MIXED>
cudaError_t launch_pcg_persistent(const PcgArgs<T>& a, int grid, bool init, cudaStream_t st);

}  // namespace maille
