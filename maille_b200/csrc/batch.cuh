// batch.cuh -- device data of the batched solver: many independent instances packed as one
// block-diagonal 3x3-block system, R right-hand sides (load cases) per instance.
//
// Layout in HBM:
//   * Rows are the kept nodes of all instances in the union analysis (setup.cpp on the packed
//     mesh); an instance's rows never couple to another instance's rows.
//   * K, L (strictly lower factor blocks) and U (L^T) in the batched sliced layout of
//     common.hpp (BSellHost): `rows` rows of one instance per slice, 4 slots per lane and step.
//   * Vectors are [(nb + 1) rows][R][3]: the 3 DOFs of load case c of row I at (I R + c) 3;
//     row nb is the dummy zero node that padding slots point at. R is 2, 4 or 8.
//   * Lanes of a warp map to (row, load-case group, sub-lane): G = R / Q groups of Q load cases
//     per row and SUB lanes splitting a row's slots, so a warp holds 32 / (G SUB) rows.
//   * Per-instance reductions are deterministic: each vector task or U slice writes its column
//     partials into a fixed slot, and the last task of an instance to finish (ticket counter)
//     sums the instance's slots in slot order.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace maille {

struct BSellDev {
    int32_t nslices;
    const int32_t* rowid;  // [nslices * rows]
    const int64_t* off;    // [nslices + 1]
    const int32_t* col;    // [steps * slots]
    const int32_t* inst;   // [nslices]
};

// Per-instance solver state; column c of instance i at [i * R + c].
struct BatchState {
    double *alpha, *beta, *rz, *rr, *bb, *maxr2;
    int32_t *iter, *col_iter, *status, *updates;
    uint32_t *done, *flagged;  // [n_inst] bit c: load case c finished / due a reliable update
    int32_t* ctrl;             // [0] active instances [1] any reliable update pending
                               // [2] sweep wait timed out [3] cancelled [4] last sweep epoch
                               // (row-ready flags only grow, across launches too)
};

template <typename M, typename T>
struct BatchArgs {
    int32_t nb, n_inst, n_rhs, max_iter;
    double tol2, delta2;
    BSellDev K, L, U;
    int32_t ntasks;
    const int32_t* task_off;    // [ntasks + 1] K slices of each vector task
    const int32_t* task_inst;   // [ntasks]
    const int32_t* inst_task;   // [n_inst + 1] tasks of each instance (instance-major)
    const int32_t* uslot;       // [U slices] reduction slot of each U slice
    const int32_t* inst_uslot;  // [n_inst + 1]
    const int32_t* bwd_seq;     // U slices by level, descending
    const M *Kv, *Lv, *Uv;
    const M* D;                 // [9 nb], entry k of row I at k nb + I
    T *x, *r, *z, *p, *ap;      // [(nb + 1) R 3]
    const double* K64;          // mixed: FP64 K in the K layout
    const double* b;            // right-hand sides [(nb + 1) R 3]
    double *x64, *r64;          // mixed: FP64 solution and true residual
    BatchState st;
    double *part_k, *part_u;    // [ntasks R], [U slices R]
    unsigned int* tickets;      // [3 n_inst]
    unsigned int* flags;        // [(nb + 1) G] row-ready epochs per load-case group
    const volatile int32_t* cancel;  // host-mapped cancel flag
    unsigned long long* timing;      // optional [8] ns per phase
};

// Lane geometry of one kernel instance.
struct BatchShape {
    int R, Q, SUB;
    int groups() const { return R / Q; }
    int rows() const { return 32 / (groups() * SUB); }
    int slots() const { return rows() * SUB * 4; }
};

// Instances compiled: R in {2, 4, 8}; (Q, SUB) per R as listed in batch_kernels.cu.
bool batch_shape_supported(const BatchShape& s);

template <typename M, typename T, bool MIXED>
int batch_grid(const BatchShape& s, int threads);
template <typename M, typename T, bool MIXED>
cudaError_t launch_batch_pcg(const BatchShape& s, const BatchArgs<M, T>& a, int grid, int threads,
                             int passes, cudaStream_t st);

// K, L, U values of the batched layout from the CSR K / factor F (src: slot -> CSR block).
template <typename T>
void launch_bsell_fill(int64_t steps, int slots, const int32_t* src, const double* csr, T* vals,
                       cudaStream_t st);
// ctrl[0] = n_inst, ctrl[1..3] = 0, tickets[0..nt) = 0 (before every solve)
void launch_batch_reset(int32_t* ctrl, int32_t n_inst, unsigned int* tickets, int64_t nt,
                        cudaStream_t st);
// b [(nb+1) R 3] = f_j - coupling at free DOFs (0 at fixed DOFs, rows past n_rhs and the dummy)
void launch_batch_rhs(int32_t nb, int R, int n_rhs, int64_t n3, const int32_t* perm,
                      const uint8_t* fixmask, const double* f, const double* coupling, double* b,
                      cudaStream_t st);
// u [n_rhs][3 N] = imposed at fixed DOFs, x64 (+ x32) elsewhere
void launch_batch_gather(int64_t n_nodes, int R, int n_rhs, const int32_t* inv, const uint8_t* fixed,
                         const double* imposed, const double* x64, const float* x32, double* u,
                         cudaStream_t st);

}  // namespace maille
