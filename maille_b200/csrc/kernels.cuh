// kernels.cuh -- sm_100a kernels of the linear-elastic solve path.
//
// Data layout in HBM (new = solver numbering of the kept nodes, see setup.cpp):
//   * K and F (the IC(0) factor) are assembled and factorised on one full 3x3-block CSR pattern:
//     row_ptr (int64), col (int32), 9 consecutive entries per block, row-major. F holds L below
//     the diagonal, L^T above it and D = L_II^-1 on the diagonal. The iteration kernels read
//     copies of K, L, L^T and D in the sliced layout of sparse.cuh.
//   * Solver vectors are padded, [4 nb] in new numbering: DOF c of row I at 4 I + c, 4th = 0.
//   * Element matrices are kept as their node-pair blocks a <= b: Ke[(e * NP + pair) * 9 + 3 i + j]
//     = K_e[3 a + i][3 b + j].
// Every reduction is deterministic: fixed per-warp shuffle trees, per-block partials in fixed
// slots, and a final sum in slot order by the last block to finish (ticket counter).
#pragma once

#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

namespace maille {

constexpr int kThreads = 256;       // threads per block of the row kernels
constexpr int kWarps = kThreads / 32;
constexpr int kMaxLevels = 65536;

// kernels launched by this library since load (a graph launch adds its kernel nodes)
extern std::atomic<long long> g_kernel_launches;

// Element geometry / material inputs (old numbering).
struct ElemIn {
    int64_t ne;
    const double* coords;
    const int32_t* conn;
    const double* young;
    const double* poisson;
};

struct Pattern {
    int32_t nb;
    const int64_t* row_ptr;
    const int32_t* col;
    const int64_t* diag;
    const int64_t* tpos;
    const uint8_t* fixmask;
};

// ---- launchers (defined in kernels.cu) -------------------------------------------------------
void launch_elem_stiffness(int npe, const ElemIn& in, double* ke_up, cudaStream_t st);
void launch_assemble(const Pattern& pt, int64_t nl, const int64_t* lslot, const int32_t* lrow,
                     const int64_t* lptr,
                     const uint32_t* contrib, const double* ke_up, double* K, cudaStream_t st);
void launch_factor_level(const Pattern& pt, int32_t r0, int32_t r1, const double* K, double* F,
                        double shift, int32_t* fail, cudaStream_t st);
// b (padded solver numbering, 4 per node) = F_f - K_fc u_c, 0 at fixed DOFs
void launch_build_rhs(int32_t nb, const int32_t* perm, const uint8_t* fixmask, const double* f,
                      const double* coupling, double* b, cudaStream_t st);
// u (caller numbering) = imposed at fixed DOFs, x (padded solver numbering) elsewhere
void launch_gather_u(int64_t n_nodes, const int32_t* inv, const uint8_t* fixed,
                     const double* imposed, const double* x, double* u, cudaStream_t st);
void launch_elem_apply(int npe, int64_t nlist, const int32_t* list, const int32_t* conn,
                       const double* ke_up, const double* u, double* ye, cudaStream_t st);
void launch_node_gather(int npe, int64_t nnodes, const int32_t* nodes, const int64_t* inc_ptr,
                        const int32_t* inc, const int32_t* elem_slot, const double* ye,
                        double* y, cudaStream_t st);
void launch_reactions(int64_t n_nodes, const int32_t* nodes, int64_t nnodes,
                      const uint8_t* fixed, const double* y, const double* f, double* react,
                      cudaStream_t st);
void launch_stresses(int npe, const ElemIn& in, const double* u, double* gauss, double* vm,
                     cudaStream_t st);
// smoothed nodal stresses [n * 6] and their von Mises values [n] from the Gauss stresses
void launch_nodal_stresses(int npe, int64_t n_nodes, const int64_t* inc_ptr, const int32_t* inc,
                           const double* gauss, double* stress, double* vm, cudaStream_t st);
void launch_adjoint_grad(int npe, int64_t ne, const int32_t* conn, const double* ke_up,
                         const double* young, const double* lambda, const double* u,
                         double* grad, cudaStream_t st);

}  // namespace maille
