// thermal.cu -- transient heat conduction (the theta-method of Model::solve_step, model.rs:621-706)
// on the device: element conduction / capacity / convection matrices, deterministic assembly of
// the left (C/dt + theta K) and right (C/dt - (1 - theta) K) matrices on the free-node pattern,
// scalar IC(0) with the reference's shift ladder, and one persistent cooperative IC(0)-PCG kernel
// per increment; right-hand sides, reactions and heat fluxes stay on the device, so a whole step
// of many increments is enqueued without a host synchronisation.
//
// Data layout in HBM (solver numbering = the multicolour order of the free nodes, setup.cpp):
//   * element matrices as node pairs a <= b, pair-major: left[pair * n_elems + e], the element
//     index fastest so that the element kernel's stores and the assembly's loads coalesce;
//   * the left matrix A, the right matrix R (free-free part) and the factor F on the full
//     scalar CSR pattern of the free nodes (gpu_pattern: the node graph is the pattern of a
//     one-DOF-per-node problem); F holds l_ij below the diagonal, l_ij again at the transposed
//     position above it, and l_ii on the diagonal;
//   * the iteration operands in the sliced layout of sparse.cuh with one scalar per slot: A and R
//     in the full-row layout (SpMV), F's strictly lower and upper parts in per-level slices (the
//     triangular sweeps), so each lane reads 4 consecutive slots (32 bytes of values, one int4 of
//     columns) and a warp 1 KB per step;
//   * vectors [nb + 1] in solver numbering; entry nb is the dummy node the padding slots point
//     at (always 0);
//   * the history [(increments + 1) n_nodes] of temperatures and reactions, and of Gauss-point
//     heat fluxes when asked for, in the caller's numbering, copied to the host once at the end.
//
// Roofline: every iteration kernel here is HBM-bandwidth bound (FP64 values streamed once per
// SpMV / sweep; vectors stay in L2). The element kernel is FP64 arithmetic, once per step.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "analysis.cuh"
#include "common.hpp"
#include "cuda_host.hpp"
#include "kernels.cuh"
#include "ordering.cuh"
#include "reduce.cuh"
#include "sparse.cuh"
#include "tet.cuh"

namespace cg = cooperative_groups;

namespace maille {
namespace {

constexpr int kT = 256;  // threads per block of every kernel here

inline void counted() { g_kernel_launches.fetch_add(1, std::memory_order_relaxed); }
inline int grid_of(int64_t n) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + kT - 1) / kT, 64 * (int64_t)device_sms()));
}

// ---- quadrature (quadrature.rs) and faces (shape.rs:129-135, mesh.rs:184-198) --------------

// Barycentric (l0, l1, l2, l3) and weight of point g of the element rule (TETRA_1 for Tet4,
// TETRA_4 for Tet10, quadrature.rs:100-138) or the capacity rule (TETRA_4 for Tet4, TETRA_14
// for Tet10, assembly.rs:413-433).
struct Rules {
    double elem[2][4][5];   // [tet10][g] l0..l3, w
    double cap[2][14][5];
};
__constant__ Rules c_rules;

// TETRA_14, quadrature.rs:140-177: the published 14-point degree-5 rule (weights sum to 1/6);
// two orbits of 4 points (a, a, a) with their moves to 1 - 3a, one orbit of 6 points (b, b, d),
// d = 1/2 - b, kept in the reference's point order.
constexpr double kT14A1 = 0.09273525031089142, kT14W1 = 0.01224884051939372;
constexpr double kT14A2 = 0.3108859192633008, kT14W2 = 0.01878132095300283;
constexpr double kT14B = 0.04550370412564851, kT14W3 = 0.00709100346284674;

Rules make_rules() {
    Rules r{};
    auto put = [](double* o, double xi, double eta, double zeta, double w) {
        o[0] = 1.0 - xi - eta - zeta;
        o[1] = xi;
        o[2] = eta;
        o[3] = zeta;
        o[4] = w;
    };
    const double A = 0.5854101966249685, B = 0.1381966011250105;  // TET_A, TET_B (quadrature.rs:108)
    const double t4[4][3] = {{B, B, B}, {A, B, B}, {B, A, B}, {B, B, A}};
    put(r.elem[0][0], 0.25, 0.25, 0.25, 1.0 / 6.0);
    for (int g = 0; g < 4; ++g) {
        put(r.elem[1][g], t4[g][0], t4[g][1], t4[g][2], 1.0 / 24.0);
        put(r.cap[0][g], t4[g][0], t4[g][1], t4[g][2], 1.0 / 24.0);
    }
    int k = 0;
    for (int o = 0; o < 2; ++o) {
        const double a = o == 0 ? kT14A1 : kT14A2, w = o == 0 ? kT14W1 : kT14W2, c = 1.0 - 3.0 * a;
        put(r.cap[1][k++], a, a, a, w);
        put(r.cap[1][k++], c, a, a, w);
        put(r.cap[1][k++], a, c, a, w);
        put(r.cap[1][k++], a, a, c, w);
    }
    const double b = kT14B, d = 0.5 - kT14B;
    const double six[6][3] = {{b, b, d}, {b, d, b}, {d, b, b}, {d, d, b}, {d, b, d}, {b, d, d}};
    for (auto& p : six) put(r.cap[1][k++], p[0], p[1], p[2], kT14W3);
    return r;
}

bool g_rules_ready[64] = {false};
void ensure_rules() {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && g_rules_ready[dev]) return;
    const Rules r = make_rules();
    CK(cudaMemcpyToSymbol(c_rules, &r, sizeof(r)));
    if (dev >= 0 && dev < 64) g_rules_ready[dev] = true;
}

// Face `face` (0..3) of a Tet4/Tet10: element positions of its nodes (vertices, then for Tet10
// the mid-edge nodes of its edges a-b, b-c, c-a: Element::face_positions, mesh.rs:184-198).
__host__ __device__ __forceinline__ int face_nodes(int npe, int face, int pos[6]) {
    const int F[4][3] = {{0, 1, 2}, {0, 3, 1}, {1, 3, 2}, {2, 3, 0}};
    const int E[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
    if (face < 0 || face > 3) return 0;
    for (int q = 0; q < 3; ++q) pos[q] = F[face][q];
    if (npe == 4) return 3;
    for (int q = 0; q < 3; ++q) {
        const int p0 = pos[q], p1 = pos[(q + 1) % 3];
        int m = 4;
        for (int k = 0; k < 6; ++k)
            if ((E[k][0] == p0 && E[k][1] == p1) || (E[k][0] == p1 && E[k][1] == p0)) m = 4 + k;
        pos[3 + q] = m;
    }
    return 6;
}

// Point g of the face rule (TRIANGLE_3 on Tet4 faces, TRIANGLE_6 on Tet10 faces,
// quadrature.rs:19-54): (xi, eta, w) and the face shape values (tri3 / tri6, shape.rs:11-48).
__host__ __device__ __forceinline__ double face_point(int nn, int g, double nv[6]) {
    double xi, eta, w;
    if (nn == 3) {
        xi = g == 1 ? 2.0 / 3.0 : 1.0 / 6.0;
        eta = g == 2 ? 2.0 / 3.0 : 1.0 / 6.0;
        w = 1.0 / 6.0;
    } else {
        const double A = 0.445948490915965, WA = 0.223381589678011 / 2.0;
        const double B = 0.091576213509771, WB = 0.109951743655322 / 2.0;
        const double a = g < 3 ? A : B;
        const int k = g % 3;
        xi = k == 1 ? 1.0 - 2.0 * a : a;
        eta = k == 2 ? 1.0 - 2.0 * a : a;
        w = g < 3 ? WA : WB;
    }
    const double l1 = 1.0 - xi - eta, l2 = xi, l3 = eta;
    if (nn == 3) {
        nv[0] = l1;
        nv[1] = l2;
        nv[2] = l3;
    } else {
        nv[0] = l1 * (2.0 * l1 - 1.0);
        nv[1] = l2 * (2.0 * l2 - 1.0);
        nv[2] = l3 * (2.0 * l3 - 1.0);
        nv[3] = 4.0 * l1 * l2;
        nv[4] = 4.0 * l2 * l3;
        nv[5] = 4.0 * l3 * l1;
    }
    return w;
}

// |(x1 - x0) x (x2 - x0)| of the face's vertices (twice its area, face_rule assembly.rs:556-585)
__host__ __device__ __forceinline__ double twice_area(const double* x0, const double* x1, const double* x2) {
    double u[3], v[3];
    for (int k = 0; k < 3; ++k) {
        u[k] = x1[k] - x0[k];
        v[k] = x2[k] - x0[k];
    }
    const double c0 = u[1] * v[2] - u[2] * v[1], c1 = u[2] * v[0] - u[0] * v[2], c2 = u[0] * v[1] - u[1] * v[0];
    double sq = c0 * c0;
    sq = sq + c1 * c1;
    sq = sq + c2 * c2;
    return sqrt(sq);
}

// ---- element matrices ----------------------------------------------------------------------

struct HeatElemIn {
    int64_t ne;
    const double* coords;
    const int32_t* conn;
    const double* k;
    const double* rho_c;
    const int32_t* face_ptr;   // [ne + 1] convection faces of each element, in the model's order
    const int32_t* face_id;    // [faces] 0..3
    const double* face_film;   // [faces]
    double dt, theta, theta_m1;  // theta - 1 (the right matrix's factor of K)
};

template <int NPE>
struct HeatTet {
    static constexpr int NG = NPE == 4 ? 1 : 4;    // element rule
    static constexpr int NC = NPE == 4 ? 4 : 14;   // capacity rule
    static constexpr int NP = NPE * (NPE + 1) / 2;
    static constexpr int G = NPE == 4 ? 32 : 8;    // elements per block
};

// One block integrates G elements: coordinates staged in shared memory, then w |det J| k and the
// gradients dN/dx at the element rule's points (conduction, element.rs:451-463), w |det J| rho_c
// and N at the capacity rule's points (capacity, element.rs:465-477), then one thread per node
// pair: K_ab = sum_g (w k) (grad N_a . grad N_b), plus h int N_a N_b dS of every convection face
// of the element holding both nodes (FaceConvection::add_matrix, in the model's face order),
// C_ab = sum_g ((w rho_c) N_a) N_b, and the pair's entries of C/dt + theta K and
// C/dt + (theta - 1) K (model.rs:646-663).
template <int NPE>
__global__ void __launch_bounds__(kT) k_heat_elem(HeatElemIn in, double* __restrict__ left,
                                                   double* __restrict__ right) {
    using TT = HeatTet<NPE>;
    constexpr int G = TT::G, NG = TT::NG, NC = TT::NC, NP = TT::NP;
    constexpr int Q = NPE == 4 ? 0 : 1;
    __shared__ double xyz[G][NPE][3];
    __shared__ double wk[G][NG];
    __shared__ double inv[G][NG][9];
    __shared__ double grad[G][NG][NPE][3];
    __shared__ double wc[G][NC];
    __shared__ double nval[G][NC][NPE];
    const int64_t e0 = (int64_t)blockIdx.x * G;
    for (int t = threadIdx.x; t < G * NPE; t += blockDim.x) {
        const int e = t / NPE, a = t - e * NPE;
        if (e0 + e < in.ne) {
            const int64_t v = in.conn[(e0 + e) * NPE + a];
            for (int c = 0; c < 3; ++c) xyz[e][a][c] = in.coords[3 * v + c];
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < G * (NG + NC); t += blockDim.x) {
        const int e = t / (NG + NC), g = t - e * (NG + NC);
        if (e0 + e >= in.ne) continue;
        if (g < NG) {
            const double* r = c_rules.elem[Q][g];
            wk[e][g] = r[4] * fabs(jacobian<NPE>(xyz[e], r, inv[e][g])) * in.k[e0 + e];
        } else {
            const double* r = c_rules.cap[Q][g - NG];
            double scratch[9];
            wc[e][g - NG] = r[4] * fabs(jacobian<NPE>(xyz[e], r, scratch)) * in.rho_c[e0 + e];
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < G * (NG + NC) * NPE; t += blockDim.x) {
        const int e = t / ((NG + NC) * NPE), g = (t / NPE) % (NG + NC), a = t % NPE;
        if (e0 + e >= in.ne) continue;
        if (g < NG) {
            double d[3];
            dshape<NPE>(c_rules.elem[Q][g], a, d);
            const double* iv = inv[e][g];
            for (int r = 0; r < 3; ++r) grad[e][g][a][r] = iv[3 * r] * d[0] + iv[3 * r + 1] * d[1] + iv[3 * r + 2] * d[2];
        } else {
            nval[e][g - NG][a] = shape_value<NPE>(c_rules.cap[Q][g - NG], a);
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < G * NP; t += blockDim.x) {
        const int e = t % G, p = t / G;  // element fastest: coalesced pair-major stores
        const int64_t ge = e0 + e;
        if (ge >= in.ne) continue;
        int a = 0, rem = p;
        while (rem >= NPE - a) {
            rem -= NPE - a;
            ++a;
        }
        const int b = a + rem;
        double kab = 0.0;
#pragma unroll
        for (int g = 0; g < NG; ++g) {
            const double* ga = grad[e][g][a];
            const double* gb = grad[e][g][b];
            double s = ga[0] * gb[0];
            s = s + ga[1] * gb[1];
            s = s + ga[2] * gb[2];
            kab += wk[e][g] * s;
        }
        for (int32_t f = in.face_ptr[ge]; f < in.face_ptr[ge + 1]; ++f) {
            int pos[6];
            const int nn = face_nodes(NPE, in.face_id[f], pos);
            int la = -1, lb = -1;
            for (int q = 0; q < nn; ++q) {
                if (pos[q] == a) la = q;
                if (pos[q] == b) lb = q;
            }
            if (la < 0 || lb < 0) continue;
            const double area2 = twice_area(xyz[e][pos[0]], xyz[e][pos[1]], xyz[e][pos[2]]);
            const double film = in.face_film[f];
            double m = 0.0;
            for (int g = 0; g < nn; ++g) {
                double nv[6];
                const double w = face_point(nn, g, nv) * area2;
                m += film * w * nv[la] * nv[lb];
            }
            kab += m;
        }
        double cab = 0.0;
#pragma unroll
        for (int g = 0; g < NC; ++g) cab += wc[e][g] * nval[e][g][a] * nval[e][g][b];
        const double cdt = cab / in.dt;
        left[(int64_t)p * in.ne + ge] = cdt + in.theta * kab;
        right[(int64_t)p * in.ne + ge] = cdt + in.theta_m1 * kab;
    }
}

// ---- assembly and factorisation --------------------------------------------------------------

// One thread per lower slot (I, J), J <= I: the left and right entries summed over the slot's
// element pairs in element order (the scatter map of gpu_pattern), written at the slot and at
// its transposed position.
__global__ void k_heat_assemble(int64_t nl, int64_t ne, int np, const int64_t* __restrict__ lslot,
                                const int64_t* __restrict__ lptr, const uint32_t* __restrict__ contrib,
                                const int64_t* __restrict__ tpos, const double* __restrict__ left,
                                const double* __restrict__ right, double* __restrict__ A,
                                double* __restrict__ R) {
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < nl; l += (int64_t)gridDim.x * blockDim.x) {
        double sa = 0.0, sr = 0.0;
        for (int64_t k = lptr[l]; k < lptr[l + 1]; ++k) {
            const uint32_t c = contrib[k] & 0x7fffffffu;
            const int64_t e = c / (uint32_t)np, pair = c - e * np;
            sa += left[pair * ne + e];
            sr += right[pair * ne + e];
        }
        const int64_t pos = lslot[l], tp = tpos[pos];
        A[pos] = sa;
        R[pos] = sr;
        A[tp] = sa;
        R[tp] = sr;
    }
}

// Scalar IC(0) of rows r0..r1 (one level; their lower neighbours are in earlier levels), one warp
// per row, the row-oriented IC(0) of Csr::incomplete_cholesky (iterative.rs:146-170):
//   l_IJ = (a_IJ - sum_{K < J in rows I and J} l_IK l_JK) / l_JJ for each lower J ascending,
//   l_II = sqrt(a_II (1 + shift) - sum_K l_IK^2), failing the shift on NaN or <= 1e-12 a_II.
__global__ void k_heat_factor(const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
                              const int64_t* __restrict__ diag, const int64_t* __restrict__ tpos,
                              int32_t r0, int32_t r1, const double* __restrict__ A, double* F,
                              double shift, int32_t* fail) {
    const int lane = threadIdx.x & 31;
    const int32_t I = r0 + (int32_t)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (I >= r1) return;
    if (*(volatile int32_t*)fail) return;
    const int64_t rb = row_ptr[I], rd = diag[I];
    for (int64_t p = rb; p < rd; ++p) {
        const int32_t J = col[p];
        const int64_t jb = row_ptr[J], jd = diag[J];
        double s = 0.0;
        for (int64_t q = rb + lane; q < p; q += 32) {
            const int32_t kc = col[q];
            int64_t lo = jb, hi = jd;
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                if (col[mid] < kc) lo = mid + 1; else hi = mid;
            }
            if (lo < jd && col[lo] == kc) s += F[q] * F[lo];
        }
        s = warp_sum(s);
        if (lane == 0) {
            const double l = (A[p] - s) / F[jd];
            F[p] = l;
            F[tpos[p]] = l;
        }
        __syncwarp();
    }
    double s = 0.0;
    for (int64_t q = rb + lane; q < rd; q += 32) s += F[q] * F[q];
    s = warp_sum(s);
    if (lane == 0) {
        const double a = A[rd];
        const double pivot = a * (1.0 + shift) - s;
        if (isnan(pivot) || pivot <= 1e-12 * a) atomicExch(fail, 1);
        else F[rd] = sqrt(pivot);
    }
}

// out[slot] = M[src[slot]] (0 for padding), D[i] = M[diag[i]]
__global__ void k_gather_slots(int64_t n, const int32_t* __restrict__ src, const double* __restrict__ M,
                               double* __restrict__ out) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int32_t s = src[t];
        out[t] = s >= 0 ? M[s] : 0.0;
    }
}
__global__ void k_to_float(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        b[t] = (float)a[t];
}
__global__ void k_gather_diag(int32_t nb, const int64_t* __restrict__ diag, const double* __restrict__ M,
                              double* __restrict__ D) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += (int64_t)gridDim.x * blockDim.x)
        D[i] = M[diag[i]];
}

// ---- increments --------------------------------------------------------------------------------

// The constant part of every increment's right-hand side on free row I (node v = perm[I]):
//   g_I = F_v + sum_{e at v} sum_{b fixed} (right_e[a][b] - left_e[a][b]) T_b
// (the fixed columns of the carried product R T_n, model.rs:687-688, less the coupling of
// FreeSystem::new, model.rs:1487-1495; imposed temperatures do not change during the step).
__global__ void k_heat_const(int32_t nb, int npe, int64_t ne, const int32_t* __restrict__ perm,
                             const int64_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc,
                             const int32_t* __restrict__ conn, const uint8_t* __restrict__ fixed,
                             const double* __restrict__ imposed, const double* __restrict__ f,
                             const double* __restrict__ left, const double* __restrict__ right,
                             double* __restrict__ g) {
    for (int64_t I = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; I <= nb; I += (int64_t)gridDim.x * blockDim.x) {
        if (I == nb) {  // the dummy node
            g[I] = 0.0;
            continue;
        }
        const int32_t v = perm[I];
        double s = f ? f[v] : 0.0;
        for (int64_t q = inc_ptr[v]; q < inc_ptr[v + 1]; ++q) {
            const int32_t ea = inc[q];
            const int64_t e = ea / npe;
            const int a = ea - (int)(e * npe);
            for (int b = 0; b < npe; ++b) {
                const int32_t w = conn[e * npe + b];
                if (!fixed[w]) continue;
                const int lo = a < b ? a : b, hi = a < b ? b : a;
                const int64_t pair = lo * npe - lo * (lo - 1) / 2 + (hi - lo);
                s += (right[pair * ne + e] - left[pair * ne + e]) * imposed[w];
            }
        }
        g[I] = s;
    }
}


// Lane share of sum over a slice row's slots of vals * x[col] (the sliced layout of sparse.cuh,
// one scalar per slot), reduced over the row's lpr lanes: every lane of the row returns the sum.
// The columns and values of up to kChunk steps are loaded before their gathers are issued, so a
// chunk costs two memory round trips however many steps it holds.
template <int kChunk>
__device__ __forceinline__ double slice_row_dot(const SellDev& S, const double* __restrict__ vals, int32_t sl,
                                                const double* x, int lane) {
    double acc = 0.0;
    const int64_t g0 = S.off[sl], g1 = S.off[sl + 1];
    for (int64_t g = g0; g < g1; g += kChunk) {
        int4 c[kChunk];
        double2 v01[kChunk], v23[kChunk];
#pragma unroll
        for (int j = 0; j < kChunk; ++j)
            if (g + j < g1) {
                const int64_t base = (g + j) * kStepSlots + 4 * lane;
                c[j] = __ldg(reinterpret_cast<const int4*>(S.col + base));
                v01[j] = __ldg(reinterpret_cast<const double2*>(vals + base));
                v23[j] = __ldg(reinterpret_cast<const double2*>(vals + base + 2));
            }
        double xv[kChunk][4];
#pragma unroll
        for (int j = 0; j < kChunk; ++j)
            if (g + j < g1) {
                xv[j][0] = __ldcg(x + c[j].x);
                xv[j][1] = __ldcg(x + c[j].y);
                xv[j][2] = __ldcg(x + c[j].z);
                xv[j][3] = __ldcg(x + c[j].w);
            }
#pragma unroll
        for (int j = 0; j < kChunk; ++j)
            if (g + j < g1) {
                acc += v01[j].x * xv[j][0];
                acc += v01[j].y * xv[j][1];
                acc += v23[j].x * xv[j][2];
                acc += v23[j].y * xv[j][3];
            }
    }
    for (int o = S.lpr >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return acc;
}

// b = R x + g on the free rows (the carried product plus the constant part), x = T_n in solver
// numbering; one warp per slice of R's full-row layout.
__global__ void __launch_bounds__(kT) k_heat_rhs(SellDev R, const double* __restrict__ Rv,
                                                  const double* __restrict__ x, const double* __restrict__ g,
                                                  double* __restrict__ b) {
    const int lane = threadIdx.x & 31, S = 32 / R.lpr, r = lane / R.lpr, q = lane % R.lpr;
    for (int32_t sl = (int32_t)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5); sl < R.nslices;
         sl += (int32_t)(((int64_t)gridDim.x * blockDim.x) >> 5)) {
        const double acc = slice_row_dot<4>(R, Rv, sl, x, lane);
        const int32_t row = R.rowid[(int64_t)sl * S + r];
        if (q == 0 && row >= 0) b[row] = acc + g[row];
    }
}

// Arguments of the persistent PCG kernel of one increment. T is the storage type of the
// iteration's matrices and vectors: double in the plain form, float in the mixed form, whose
// solution accumulates in x64 (FP64) through reliable updates against the FP64 matrix A64v.
template <typename T>
struct HeatPcg {
    using Rec = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
    int32_t nb;
    SellDev A, Lo, Up;
    const int32_t* bwd_slice;        // [Up.nslices] slices of Up in backward sweep order
    const T *Av, *Lv, *Uv, *D;
    const double* b;                 // FP64 right-hand side
    T *x, *r, *p, *ap;               // [nb + 1]; the plain form's x is the solution
    Rec *yrec, *zrec;                // [nb + 1] sweep records (value, tag); entry nb always ready
    double* partials;                // [4 * grid]
    int32_t* timeout;                // set when a record wait ran out
    unsigned long long epoch0;       // the launch's sweeps tag their records epoch0 + 1, + 2, ...
    double tol;
    int32_t max_iter;
    int32_t* status;                 // this increment: 0 ok, 1 singular, 2 cap reached, 3 wait
                                     // timeout; set before the launch by k_heat_gate to 5 (skipped
                                     // after an earlier failure) or 6 (cancelled), else 0
    int32_t* iterations;
    double* rel;
    unsigned long long* timing;      // optional [4] ns per phase (block 0): spmv, update, sweeps, p
    // mixed form only
    const double* A64v;              // A's FP64 values in the same sliced layout
    double* x64;                     // [nb + 1] the FP64 solution
    double* r64;                     // [nb + 1] the true residual b - A x64
    double delta;                    // reliable update when ||r|| fell below delta x its last true value
};

__device__ __forceinline__ unsigned long long heat_clock() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

constexpr unsigned int kSpinLimit = 1u << 22;  // re-reads of a record before a wait gives up
// mixed form: a reliable update whenever the FP32 residual fell below this fraction of the last
// true one (the elastic mixed form's threshold)
constexpr double kHeatDelta = 0.3;

__device__ __forceinline__ void heat_publish(double v, double* partials, int slot, double* sh) {
    const double t = block_sum(v, sh);
    if (threadIdx.x == 0) partials[slot * gridDim.x + blockIdx.x] = t;
}
__device__ __forceinline__ double heat_total(const double* partials, int slot) {
    const int lane = threadIdx.x & 31;
    double t = 0.0;
    for (int k = lane; k < (int)gridDim.x; k += 32) t += __ldcg(partials + slot * gridDim.x + k);
    return warp_sum(t);
}

// A sweep record: the row's value and the epoch of the sweep that wrote it, in one access (16
// bytes in FP64, the tag a 64-bit word; 8 bytes in FP32, the tag the low 32 bits of the epoch), so
// the tag never arrives without its value.
__device__ __forceinline__ double2 ld_rec(const double2* q) {
    double2 v;
    asm volatile("ld.relaxed.gpu.global.v2.f64 {%0,%1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(q) : "memory");
    return v;
}
__device__ __forceinline__ float2 ld_rec(const float2* q) {
    float2 v;
    asm volatile("ld.relaxed.gpu.global.v2.f32 {%0,%1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(q) : "memory");
    return v;
}
__device__ __forceinline__ void st_rec(double2* q, double v, unsigned long long tag) {
    asm volatile("st.relaxed.gpu.global.v2.f64 [%0], {%1,%2};" ::"l"(q), "d"(v),
                 "d"(__longlong_as_double((long long)tag))
                 : "memory");
}
__device__ __forceinline__ void st_rec(float2* q, float v, unsigned long long tag) {
    asm volatile("st.relaxed.gpu.global.v2.f32 [%0], {%1,%2};" ::"l"(q), "f"(v),
                 "f"(__uint_as_float((unsigned int)tag))
                 : "memory");
}
__device__ __forceinline__ bool rec_ready(double2 v, unsigned long long epoch) {
    return (unsigned long long)__double_as_longlong(v.y) >= epoch;
}
__device__ __forceinline__ bool rec_ready(float2 v, unsigned long long epoch) {
    return __float_as_uint(v.y) >= (unsigned int)epoch;
}

// Waits (bounded) until the four records v (read once already from rec at the columns c) carry
// `epoch`, re-reading the stale ones; false when the wait gave up (its own limit, or another
// warp's timeout flag).
template <typename R>
__device__ __forceinline__ bool await4(const R* rec, int4 c, unsigned long long epoch, R v[4],
                                       const int32_t* timeout) {
    for (unsigned int k = 0; k < kSpinLimit; ++k) {
        const bool r0 = rec_ready(v[0], epoch), r1 = rec_ready(v[1], epoch), r2 = rec_ready(v[2], epoch),
                   r3 = rec_ready(v[3], epoch);
        if (r0 && r1 && r2 && r3) return true;
        if ((k & 1023u) == 1023u && *(volatile const int32_t*)timeout) return false;
        if (!r0) v[0] = ld_rec(rec + c.x);
        if (!r1) v[1] = ld_rec(rec + c.y);
        if (!r2) v[2] = ld_rec(rec + c.z);
        if (!r3) v[3] = ld_rec(rec + c.w);
    }
    return false;
}
template <typename R>
__device__ __forceinline__ bool await1(const R* rec, unsigned long long epoch, R& v, const int32_t* timeout) {
    v = ld_rec(rec);
    for (unsigned int k = 0; k < kSpinLimit; ++k) {
        if (rec_ready(v, epoch)) return true;
        if ((k & 1023u) == 1023u && *(volatile const int32_t*)timeout) return false;
        v = ld_rec(rec);
    }
    return false;
}

// 4 consecutive slot values of a lane (16-byte aligned)
__device__ __forceinline__ void lane4(const double* p, double v[4]) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p + 2));
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void lane4(const float* p, float v[4]) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}

// Lane share of sum over a slice row's slots of vals * rec[col].value once every record carries
// `epoch`, reduced over the row's lanes. The columns and values of step g + 1 are requested
// before the records of step g are awaited, so a step costs about one round trip.
template <typename T, typename R>
__device__ __forceinline__ T slice_row_dot_rec(const SellDev& S, const T* __restrict__ vals, int64_t g0, int64_t g1,
                                               const R* rec, unsigned long long epoch, int lane,
                                               const int32_t* timeout, bool& ok) {
    T acc = 0;
    int4 cn = make_int4(0, 0, 0, 0);
    T vn[4] = {0, 0, 0, 0};
    if (g0 < g1) {
        const int64_t base = g0 * kStepSlots + 4 * lane;
        cn = __ldg(reinterpret_cast<const int4*>(S.col + base));
        lane4(vals + base, vn);
    }
    for (int64_t g = g0; g < g1; ++g) {
        const int4 c = cn;
        const T v0 = vn[0], v1 = vn[1], v2 = vn[2], v3 = vn[3];
        if (g + 1 < g1) {
            const int64_t base = (g + 1) * kStepSlots + 4 * lane;
            cn = __ldg(reinterpret_cast<const int4*>(S.col + base));
            lane4(vals + base, vn);
        }
        R v[4];
        v[0] = ld_rec(rec + c.x);
        v[1] = ld_rec(rec + c.y);
        v[2] = ld_rec(rec + c.z);
        v[3] = ld_rec(rec + c.w);
        if (!await4(rec, c, epoch, v, timeout)) ok = false;
        acc += v0 * (T)v[0].x;
        acc += v1 * (T)v[1].x;
        acc += v2 * (T)v[2].x;
        acc += v3 * (T)v[3].x;
    }
    __syncwarp();
    for (int o = S.lpr >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return acc;
}

// Lane share of a sliced SpMV row (vals * x[col]) in the precision of x, reduced over the row's
// lanes; kChunk steps' columns and values are requested before their gathers.
template <int kChunk, typename M, typename X>
__device__ __forceinline__ X slice_row_dot_t(const SellDev& S, const M* __restrict__ vals, int32_t sl, const X* x,
                                             int lane) {
    X acc = 0;
    const int64_t g0 = S.off[sl], g1 = S.off[sl + 1];
    for (int64_t g = g0; g < g1; g += kChunk) {
        int4 c[kChunk];
        M v[kChunk][4];
#pragma unroll
        for (int j = 0; j < kChunk; ++j)
            if (g + j < g1) {
                const int64_t base = (g + j) * kStepSlots + 4 * lane;
                c[j] = __ldg(reinterpret_cast<const int4*>(S.col + base));
                lane4(vals + base, v[j]);
            }
        X xv[kChunk][4];
#pragma unroll
        for (int j = 0; j < kChunk; ++j)
            if (g + j < g1) {
                xv[j][0] = __ldcg(x + c[j].x);
                xv[j][1] = __ldcg(x + c[j].y);
                xv[j][2] = __ldcg(x + c[j].z);
                xv[j][3] = __ldcg(x + c[j].w);
            }
#pragma unroll
        for (int j = 0; j < kChunk; ++j)
            if (g + j < g1) {
                acc += (X)v[j][0] * xv[j][0];
                acc += (X)v[j][1] * xv[j][1];
                acc += (X)v[j][2] * xv[j][2];
                acc += (X)v[j][3] * xv[j][3];
            }
    }
    for (int o = S.lpr >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return acc;
}

// z = M^-1 r with M = L L^T (Csr::precondition, iterative.rs:173-188) as one dataflow pass: the
// forward sweep y_i = (r_i - sum_{j<i} l_ij y_j) / l_ii over L's slices (levels ascending), then
// the backward sweep z_i = (y_i - sum_{j>i} l_ji z_j) / l_ii over U's slices (levels
// descending); warp w takes the slices w, w + warps, ... of that sequence. A row waits only for
// the records it reads, tagged with this pass's epoch, so no barrier separates the levels; every
// dependency lies earlier in the sequence and every warp is resident, so the earliest unfinished
// slice can always proceed. The next slice's metadata is fetched while this one is swept (going
// further, with the next slice's columns and values too, measured slower: more registers on the
// critical path). Returns this thread's share of r . z.
template <typename T>
__device__ __forceinline__ double heat_sweeps(const HeatPcg<T>& a, unsigned long long epoch) {
    const int lane = threadIdx.x & 31;
    const int32_t w0 = (int32_t)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int32_t nw = (int32_t)(((int64_t)gridDim.x * blockDim.x) >> 5);
    const int32_t nl = a.Lo.nslices, nt = a.Lo.nslices + a.Up.nslices;
    bool ok = true;
    double rz = 0.0;
    // the slice's place in L or U, its step range and this lane's row
    auto meta = [&](int32_t k, int32_t& sl, int64_t& g0, int64_t& g1, int32_t& row) {
        const bool fwd = k < nl;
        const SellDev& S = fwd ? a.Lo : a.Up;
        sl = fwd ? k : __ldg(a.bwd_slice + (k - nl));
        g0 = __ldg(S.off + sl);
        g1 = __ldg(S.off + sl + 1);
        row = __ldg(S.rowid + (int64_t)sl * (32 / S.lpr) + lane / S.lpr);
    };
    int32_t sl_n = 0, row_n = -1;
    int64_t g0_n = 0, g1_n = 0;
    if (w0 < nt) meta(w0, sl_n, g0_n, g1_n, row_n);
    for (int32_t k = w0; k < nt; k += nw) {
        const int32_t row = row_n;
        const int64_t g0 = g0_n, g1 = g1_n;
        if (k + nw < nt) meta(k + nw, sl_n, g0_n, g1_n, row_n);
        const bool fwd = k < nl;
        const SellDev& S = fwd ? a.Lo : a.Up;
        const bool owner = (lane % S.lpr) == 0 && row >= 0;
        // the row's own operands, requested before the wait
        const T d = owner ? __ldg(a.D + row) : (T)1;
        const T ri = owner ? __ldcg(a.r + row) : (T)0;
        const T acc = slice_row_dot_rec<T>(S, fwd ? a.Lv : a.Uv, g0, g1, fwd ? a.yrec : a.zrec, epoch, lane,
                                           a.timeout, ok);
        if (owner) {
            if (fwd) {
                st_rec(a.yrec + row, (ri - acc) / d, epoch);
            } else {
                typename HeatPcg<T>::Rec y;
                if (!await1(a.yrec + row, epoch, y, a.timeout)) ok = false;
                const T z = (y.x - acc) / d;
                st_rec(a.zrec + row, z, epoch);
                rz += (double)ri * (double)z;
            }
        }
    }
    if (!ok) atomicExch(a.timeout, 1);
    return rz;
}

// Decides, before increment s's PCG launch, whether it runs: 5 when an earlier increment failed or
// was cancelled, 6 when the cancel flag (mapped host memory) is raised, 0 otherwise. One thread
// reads the flag once, so every block of the cooperative launch that follows sees one decision.
__global__ void k_heat_gate(const volatile int32_t* cancel, const int32_t* prev_status, int32_t* status) {
    int32_t g = 0;
    if (prev_status && *prev_status != 0)
        g = 5;
    else if (cancel && *cancel != 0)
        g = 6;
    *status = g;
}

// two consecutive entries of a vector (16-byte FP64 / 8-byte FP32 access) and back
__device__ __forceinline__ double2 ld2(const double* p) { return __ldcg(reinterpret_cast<const double2*>(p)); }
__device__ __forceinline__ double2 ld2(const float* p) {
    const float2 v = __ldcg(reinterpret_cast<const float2*>(p));
    return make_double2(v.x, v.y);
}
__device__ __forceinline__ void st2(double* p, double a, double b) {
    *reinterpret_cast<double2*>(p) = make_double2(a, b);
}
__device__ __forceinline__ void st2(float* p, double a, double b) {
    *reinterpret_cast<float2*>(p) = make_float2((float)a, (float)b);
}

// IC(0)-PCG of one increment from x = 0 (Pcg::solve, iterative.rs:210-248) in one cooperative
// launch: SpMV, the x / r update, the dataflow preconditioner and the p update, each closed by a
// grid barrier (four per iteration). (Fusing the two updates into the SpMV and the sweeps saves
// two barriers but puts more loads on the sweeps' critical path; measured slower.) Every
// reduction is per-block partials in fixed slots summed in slot order by every block.
// MIXED: FP32 matrices and vectors with FP64 scalars and reductions; whenever the FP32 residual
// fell by delta since the last true one (and at the end), x64 += x, x = 0 and r64 = b - A64 x64 in
// FP64, r = r64 (the reliable update of the elastic mixed form); the stopping test is on r64.
template <typename T, bool MIXED>
__global__ void __launch_bounds__(kT, 2) k_heat_pcg(HeatPcg<T> a) {
    __shared__ double sh[kT / 32];
    cg::grid_group grid = cg::this_grid();
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    if (*a.status != 0) {  // gated off before the launch (an earlier failure, or cancelled)
        if (lead) {
            *a.iterations = 0;
            *a.rel = 0.0;
        }
        return;
    }
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nth = (int64_t)gridDim.x * blockDim.x;
    const bool timed = a.timing != nullptr && lead;
    unsigned long long t_last = timed ? heat_clock() : 0;
    auto mark = [&](int phase) {
        if (timed) {
            const unsigned long long t = heat_clock();
            a.timing[phase] += t - t_last;
            t_last = t;
        }
    };
    unsigned long long epoch = a.epoch0;
    double loc = 0.0;
    for (int64_t i = tid; i < a.nb; i += nth) {
        const double bi = a.b[i];
        a.x[i] = (T)0;
        a.r[i] = (T)bi;
        if constexpr (MIXED) {
            a.x64[i] = 0.0;
            a.r64[i] = bi;
        }
        loc += bi * bi;
    }
    heat_publish(loc, a.partials, 3, sh);
    grid.sync();
    const double bnorm = sqrt(heat_total(a.partials, 3));
    double maxr = bnorm;  // mixed: the last true residual norm
    int32_t status = 0, it = 0;
    double rel = 0.0;
    if (bnorm > 0.0) {
        loc = heat_sweeps(a, ++epoch);
        heat_publish(loc, a.partials, 2, sh);
        grid.sync();
        double rz = heat_total(a.partials, 2);
        for (int64_t i = tid; i < a.nb; i += nth) a.p[i] = (T)__ldcg(&a.zrec[i].x);
        grid.sync();
        for (;;) {
            if (__ldcg(a.timeout)) {
                status = 3;
                break;
            }
            // ap = A p, curvature p . ap
            {
                const int lane = threadIdx.x & 31, S = 32 / a.A.lpr, r = lane / a.A.lpr, q = lane % a.A.lpr;
                const int32_t w0 = (int32_t)(tid >> 5), nw = (int32_t)(nth >> 5);
                loc = 0.0;
                for (int32_t sl = w0; sl < a.A.nslices; sl += nw) {
                    const T acc = slice_row_dot_t<2>(a.A, a.Av, sl, (const T*)a.p, lane);
                    const int32_t row = a.A.rowid[(int64_t)sl * S + r];
                    if (q == 0 && row >= 0) {
                        a.ap[row] = acc;
                        loc += (double)__ldcg(a.p + row) * (double)acc;
                    }
                }
            }
            heat_publish(loc, a.partials, 0, sh);
            grid.sync();
            mark(0);
            const double pap = heat_total(a.partials, 0);
            it += 1;
            if (isnan(pap) || pap <= 0.0) {
                status = 1;
                break;
            }
            const double alpha = rz / pap;
            loc = 0.0;
            // two entries per thread and pass (16-byte FP64 / 8-byte FP32 accesses; the vectors
            // hold nb + 1 >= 2 entries and start 256-byte aligned); an odd last entry alone
            for (int64_t i2 = tid; 2 * i2 < a.nb; i2 += nth) {
                const int64_t i = 2 * i2;
                if (i + 1 < a.nb) {
                    const double2 xv = ld2(a.x + i), pv = ld2(a.p + i), rv = ld2(a.r + i), av = ld2(a.ap + i);
                    const T r0 = (T)(rv.x - alpha * av.x), r1 = (T)(rv.y - alpha * av.y);
                    st2(a.x + i, xv.x + alpha * pv.x, xv.y + alpha * pv.y);
                    st2(a.r + i, r0, r1);
                    loc += (double)r0 * (double)r0;
                    loc += (double)r1 * (double)r1;
                } else {
                    a.x[i] = (T)((double)__ldcg(a.x + i) + alpha * (double)__ldcg(a.p + i));
                    const T ri = (T)((double)__ldcg(a.r + i) - alpha * (double)__ldcg(a.ap + i));
                    a.r[i] = ri;
                    loc += (double)ri * (double)ri;
                }
            }
            heat_publish(loc, a.partials, 1, sh);
            grid.sync();
            mark(1);
            double rn = sqrt(heat_total(a.partials, 1));
            if constexpr (MIXED) {
                if (rn <= a.tol * bnorm || rn < a.delta * maxr || it >= a.max_iter) {
                    // reliable update: fold x into x64, the true residual against the FP64 matrix
                    for (int64_t i = tid; i < a.nb; i += nth) {
                        a.x64[i] += (double)__ldcg(a.x + i);
                        a.x[i] = (T)0;
                    }
                    grid.sync();
                    {
                        const int lane = threadIdx.x & 31, S = 32 / a.A.lpr, r = lane / a.A.lpr,
                                  q = lane % a.A.lpr;
                        const int32_t w0 = (int32_t)(tid >> 5), nw = (int32_t)(nth >> 5);
                        loc = 0.0;
                        for (int32_t sl = w0; sl < a.A.nslices; sl += nw) {
                            const double acc = slice_row_dot_t<2>(a.A, a.A64v, sl, (const double*)a.x64, lane);
                            const int32_t row = a.A.rowid[(int64_t)sl * S + r];
                            if (q == 0 && row >= 0) {
                                const double rv = a.b[row] - acc;
                                a.r64[row] = rv;
                                loc += rv * rv;
                            }
                        }
                    }
                    heat_publish(loc, a.partials, 1, sh);
                    grid.sync();
                    rn = sqrt(heat_total(a.partials, 1));
                    maxr = rn;
                    rel = rn / bnorm;
                    if (rn <= a.tol * bnorm) break;
                    if (it >= a.max_iter) {
                        status = 2;
                        break;
                    }
                    for (int64_t i = tid; i < a.nb; i += nth) a.r[i] = (T)__ldcg(a.r64 + i);
                    grid.sync();
                }
            } else {
                rel = rn / bnorm;
                if (rn <= a.tol * bnorm) break;
                if (it >= a.max_iter) {
                    status = 2;
                    break;
                }
            }
            loc = heat_sweeps(a, ++epoch);
            heat_publish(loc, a.partials, 2, sh);
            grid.sync();
            mark(2);
            if (__ldcg(a.timeout)) {
                status = 3;
                break;
            }
            const double rz_next = heat_total(a.partials, 2);
            const double beta = rz_next / rz;
            rz = rz_next;
            for (int64_t i2 = tid; 2 * i2 < a.nb; i2 += nth) {
                const int64_t i = 2 * i2;
                if (i + 1 < a.nb) {
                    const double z0 = (double)__ldcg(&a.zrec[i].x), z1 = (double)__ldcg(&a.zrec[i + 1].x);
                    const double2 pv = ld2(a.p + i);
                    st2(a.p + i, z0 + beta * pv.x, z1 + beta * pv.y);
                } else {
                    a.p[i] = (T)((double)__ldcg(&a.zrec[i].x) + beta * (double)__ldcg(a.p + i));
                }
            }
            grid.sync();
            mark(3);
        }
    }
    if (lead) {
        *a.status = status;
        *a.iterations = it;
        *a.rel = rel;
    }
}

// T (caller numbering) = imposed at fixed nodes, x[inv[v]] at free ones; and x from T
__global__ void k_heat_scatter(int64_t n, const int32_t* __restrict__ inv, const uint8_t* __restrict__ fixed,
                               const double* __restrict__ imposed, const double* __restrict__ x,
                               double* __restrict__ T) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        T[v] = fixed[v] ? imposed[v] : x[inv[v]];
}
__global__ void k_heat_initial(int64_t n, const int32_t* __restrict__ inv, const uint8_t* __restrict__ fixed,
                               const double* __restrict__ imposed, const double* __restrict__ initial,
                               double* __restrict__ T, double* __restrict__ x) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const double t = fixed[v] ? imposed[v] : initial[v];
        T[v] = t;
        if (!fixed[v]) x[inv[v]] = t;
    }
}

// Reactions on the imposed nodes (model.rs:690-697 with product, model.rs:1353-1369):
//   R_v = sum_{e at v} left_e[a] . T_new  -  (sum_{e at v} right_e[a] . T_old + F_v)
// one thread per imposed node, elements in order; other entries were zeroed.
__global__ void k_heat_react(int64_t nfix, const int32_t* __restrict__ nodes, int npe, int64_t ne,
                             const int64_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc,
                             const int32_t* __restrict__ conn, const double* __restrict__ left,
                             const double* __restrict__ right, const double* __restrict__ f,
                             const double* __restrict__ t_new, const double* __restrict__ t_old,
                             double* __restrict__ react) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nfix; k += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = nodes[k];
        double y = 0.0, c = 0.0;
        for (int64_t q = inc_ptr[v]; q < inc_ptr[v + 1]; ++q) {
            const int32_t ea = inc[q];
            const int64_t e = ea / npe;
            const int a = ea - (int)(e * npe);
            double sy = 0.0, sc = 0.0;
            for (int b = 0; b < npe; ++b) {
                const int lo = a < b ? a : b, hi = a < b ? b : a;
                const int64_t pair = lo * npe - lo * (lo - 1) / 2 + (hi - lo);
                const int32_t w = conn[e * npe + b];
                sy += left[pair * ne + e] * t_new[w];
                sc += right[pair * ne + e] * t_old[w];
            }
            y += sy;
            c += sc;
        }
        react[v] = y - (c + (f ? f[v] : 0.0));
    }
}

// Heat fluxes q = -k grad T and the point position at every element-rule point (heat_fluxes,
// element.rs:480-506); one thread per (element, point); out: x, y, z, qx, qy, qz.
template <int NPE>
__global__ void k_heat_flux(int64_t ne, const double* __restrict__ coords, const int32_t* __restrict__ conn,
                            const double* __restrict__ k, const double* __restrict__ T, double* __restrict__ out) {
    constexpr int NG = NPE == 4 ? 1 : 4, Q = NPE == 4 ? 0 : 1;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ne * NG; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = t / NG;
        const int g = (int)(t - e * NG);
        double xyz[NPE][3], te[NPE];
        for (int a = 0; a < NPE; ++a) {
            const int64_t v = conn[e * NPE + a];
            for (int c = 0; c < 3; ++c) xyz[a][c] = coords[3 * v + c];
            te[a] = T[v];
        }
        const double* l = c_rules.elem[Q][g];
        double iv[9];
        jacobian<NPE>(xyz, l, iv);
        double q[3] = {0.0, 0.0, 0.0}, at[3] = {0.0, 0.0, 0.0};
        for (int a = 0; a < NPE; ++a) {
            double d[3];
            dshape<NPE>(l, a, d);
            const double n = shape_value<NPE>(l, a);
            for (int c = 0; c < 3; ++c) {
                q[c] += (iv[3 * c] * d[0] + iv[3 * c + 1] * d[1] + iv[3 * c + 2] * d[2]) * te[a];
                at[c] += n * xyz[a][c];
            }
        }
        double* o = out + t * 6;
        for (int c = 0; c < 3; ++c) {
            o[c] = at[c];
            o[3 + c] = -k[e] * q[c];
        }
    }
}

// ---- host driver -----------------------------------------------------------------------------

// Cancel flags of the thermal step, one per device, in mapped pinned host memory: the host raises
// one with maille_gpu_thermal_cancel and k_heat_gate reads it on the device before every
// increment, so the whole step stays enqueued at once without a host synchronisation per
// increment.
constexpr int kMaxCancelDevices = 64;
std::mutex g_cancel_mutex;
int32_t* g_cancel_host = nullptr;

int32_t* cancel_flags() {
    std::lock_guard<std::mutex> lock(g_cancel_mutex);
    if (!g_cancel_host) {
        void* p = nullptr;
        CK(cudaHostAlloc(&p, kMaxCancelDevices * sizeof(int32_t), cudaHostAllocMapped | cudaHostAllocPortable));
        std::memset(p, 0, kMaxCancelDevices * sizeof(int32_t));
        g_cancel_host = static_cast<int32_t*>(p);
    }
    return g_cancel_host;
}

// The device's flag as the current device addresses it (nullptr past kMaxCancelDevices: such a
// device's steps cannot be cancelled).
const int32_t* cancel_flag_device(int device) {
    if (device < 0 || device >= kMaxCancelDevices) return nullptr;
    int32_t* h = cancel_flags() + device;
    void* d = nullptr;
    CK(cudaHostGetDevicePointer(&d, h, 0));
    return static_cast<const int32_t*>(d);
}

int32_t th_fail(int32_t status, const std::string& m) {
    set_last_error(m);
    return status;
}

// A sliced layout of one part (full rows, strictly lower, strictly upper) of the scalar pattern.
struct Slices {
    SellHost h;
    SellKind kind = SELL_FULL;
    int32_t *rowid = nullptr, *col = nullptr, *src = nullptr, *level = nullptr;
    int64_t* off = nullptr;
    int32_t pad = 0;
    SellDev dev() const { return SellDev{h.lpr, h.nslices(), rowid, off, col, pad}; }
    void upload(const PatternDev& pt, int32_t nb, cudaStream_t st) {
        pad = nb;
        rowid = dupload(h.rowid.data(), h.rowid.size(), st);
        off = dupload(h.off.data(), h.off.size(), st);
        level = dupload(h.level_slices.data(), h.level_slices.size(), st);
        col = dalloc<int32_t>((size_t)h.steps() * kStepSlots);
        src = dalloc<int32_t>((size_t)h.steps() * kStepSlots);
        fill_sell(kind, h.lpr, h.nslices(), h.steps(), rowid, off, pt.row_ptr, pt.col, pt.diag, nb, col, src, st);
    }
    void release() {
        for (void* p : {(void*)rowid, (void*)col, (void*)src, (void*)level, (void*)off}) dfree(p);
    }
};

struct DevBufs {
    std::vector<void*> all;
    template <typename T>
    T* take(T* p) {
        all.push_back((void*)p);
        return p;
    }
    ~DevBufs() {
        for (void* p : all) dfree(p);
    }
};

bool finite_all(const double* v, int64_t n) {
    for (int64_t i = 0; i < n; ++i)
        if (!std::isfinite(v[i])) return false;
    return true;
}

int32_t check_thermal(const MailleThermalProblem* p, std::string& why) {
    auto bad = [&](const std::string& m) {
        why = m;
        return MAILLE_INVALID_INPUT;
    };
    if (!p->coords || !p->conn || !p->conductivity || !p->rho_c || !p->fixed || !p->initial)
        return bad("null argument");
    if (p->nodes_per_elem != 4 && p->nodes_per_elem != 10) return bad("nodes_per_elem must be 4 or 10");
    if (p->n_nodes <= 0 || p->n_elems <= 0) return bad("empty mesh");
    if (!(p->time_step > 0.0) || !std::isfinite(p->time_step)) return bad("time_step must be finite and > 0");
    if (!(p->theta >= 0.5 && p->theta <= 1.0)) return bad("theta must lie in [0.5, 1] (ThetaOutOfRange)");
    if (p->increments <= 0) return bad("increments must be > 0 (NoIncrements)");
    if (p->ordering < MAILLE_ORDER_AUTO || p->ordering > MAILLE_ORDER_MULTICOLOR_ITERATED) return bad("unknown ordering");
    if (p->precision != MAILLE_FP64 && p->precision != MAILLE_MIXED) return bad("unknown precision");
    if (p->precision == MAILLE_MIXED) {
        // FP32 sweep records carry 32-bit tags: every sweep of the step needs its own
        const int64_t span = (int64_t)(p->max_iter > 0 ? p->max_iter : kDefaultMaxIter) + 2;
        if ((int64_t)p->increments * span >= (int64_t)UINT32_MAX - 1)
            return bad("too many increments x iterations for the mixed form's 32-bit sweep tags");
    }
    if (p->n_convection < 0 || (p->n_convection > 0 && (!p->conv_elem || !p->conv_face || !p->conv_film)))
        return bad("null convection arrays");
    const int64_t n = p->n_nodes;
    for (int64_t k = 0; k < p->n_elems * p->nodes_per_elem; ++k)
        if (p->conn[k] < 0 || p->conn[k] >= n)
            return bad("element " + std::to_string(k / p->nodes_per_elem) + " refers to unknown node " +
                       std::to_string(p->conn[k]));
    if (!finite_all(p->coords, 3 * n)) return bad("non-finite coordinate");
    if (!finite_all(p->conductivity, p->n_elems) || !finite_all(p->rho_c, p->n_elems))
        return bad("non-finite conductivity or heat capacity");
    for (int64_t v = 0; v < n; ++v)
        if (!std::isfinite(p->initial[v])) return bad("NonFiniteTemperature at node " + std::to_string(v));
    if (p->imposed)
        for (int64_t v = 0; v < n; ++v)
            if (p->fixed[v] && !std::isfinite(p->imposed[v])) return bad("non-finite imposed temperature");
    if (p->f && !finite_all(p->f, n)) return bad("non-finite heat load");
    if (p->n_convection > 0 && !finite_all(p->conv_film, p->n_convection)) return bad("non-finite film");
    int64_t nfree = 0;
    for (int64_t v = 0; v < n; ++v) nfree += p->fixed[v] ? 0 : 1;
    if (nfree == 0) return bad("every DOF is fixed");
    return MAILLE_OK;
}

int32_t thermal_transient(const MailleThermalProblem* p, MailleThermalResult* res) {
    NvtxRange nvtx("maille thermal transient");
    std::string why;
    if (const int32_t s = check_thermal(p, why); s != MAILLE_OK) return th_fail(s, why);
    const int npe = p->nodes_per_elem;
    const int64_t n = p->n_nodes, ne = p->n_elems;
    const int np = node_pairs(npe), ng = gauss_points(npe);
    const int32_t steps = p->increments;
    const double tol = p->rel_tol > 0.0 ? p->rel_tol : kDefaultTol;
    const int32_t max_iter = p->max_iter > 0 ? p->max_iter : kDefaultMaxIter;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || p->device < 0 || p->device >= ndev)
        return th_fail(MAILLE_CUDA_ERROR, "no CUDA device " + std::to_string(p->device));

    // host: ordering of the free nodes (one DOF per node: a node is kept when free) on a thread
    // of its own while the device takes the inputs and integrates the element matrices
    std::vector<uint8_t> fixed3(3 * n);
    for (int64_t v = 0; v < n; ++v) fixed3[3 * v] = fixed3[3 * v + 1] = fixed3[3 * v + 2] = p->fixed[v] ? 1 : 0;
    Symbolic sym;
    Error err{MAILLE_OK, ""};
    bool analysed = false;
    const double t_setup0 = now_ms();
    double t_setup1 = t_setup0;
    // AUTO: MULTICOLOR_BFS (on Tet10 40^3: 17 levels against 18 and 12 % fewer iterations than
    // MULTICOLOR, the step 21 % shorter). The ordering runs on the device (ordering.cu) once the
    // connectivity is there, the node incidence on this thread meanwhile; MAILLE_HOST_ORDERING=1
    // orders on the thread instead (the same permutation).
    const int ordering = p->ordering == MAILLE_ORDER_AUTO ? MAILLE_ORDER_MULTICOLOR_BFS : p->ordering;
    const char* host_env = std::getenv("MAILLE_HOST_ORDERING");
    const bool host_ordering = host_env && std::atoi(host_env) != 0;
    std::vector<int32_t> kept, kept_of;
    std::thread analysis([&] {
        if (host_ordering)
            analysed = analyse(n, npe, ne, p->conn, fixed3.data(), ordering, sym, err, /*pattern=*/false,
                               /*boundary_lists=*/false);
        else
            analysed = analyse_topology(n, npe, ne, p->conn, fixed3.data(), sym, kept, kept_of, err,
                                        /*boundary_lists=*/false, /*incidence=*/false);
        t_setup1 = now_ms();
    });
    struct Joiner {
        std::thread& t;
        ~Joiner() {
            if (t.joinable()) t.join();
        }
    } joiner{analysis};

    cudaStream_t st = nullptr;
    cudaEvent_t ev[7] = {};
    DevBufs mem;
    Slices sk, sl, su;
    sk.kind = SELL_FULL;
    sl.kind = SELL_LOWER;
    su.kind = SELL_UPPER;
    struct Cleanup {
        cudaStream_t& st;
        cudaEvent_t* ev;
        Slices *a, *b, *c;
        ~Cleanup() {
            if (st) cudaStreamSynchronize(st);
            a->release();
            b->release();
            c->release();
            for (int k = 0; k < 7; ++k)
                if (ev[k]) cudaEventDestroy(ev[k]);
            if (st) cudaStreamDestroy(st);
        }
    };
    try {
        CK(cudaSetDevice(p->device));
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        Cleanup cleanup{st, ev, &sk, &sl, &su};
        for (auto& e : ev) CK(cudaEventCreate(&e));
        ensure_rules();
        CK(cudaEventRecord(ev[0], st));
        // inputs (the connectivity is narrowed to 32 bits on the device)
        // convection faces grouped by element, the model's order kept inside an element
        std::vector<int32_t> face_ptr(ne + 1, 0), face_id;
        std::vector<double> face_film;
        {
            std::vector<int64_t> keep;
            for (int64_t k = 0; k < p->n_convection; ++k)
                if (p->conv_elem[k] >= 0 && p->conv_elem[k] < ne && p->conv_face[k] >= 0 && p->conv_face[k] <= 3) {
                    keep.push_back(k);
                    face_ptr[p->conv_elem[k] + 1]++;
                }
            for (int64_t e = 0; e < ne; ++e) face_ptr[e + 1] += face_ptr[e];
            face_id.resize(keep.size());
            face_film.resize(keep.size());
            std::vector<int32_t> cur(face_ptr.begin(), face_ptr.end() - 1);
            for (int64_t k : keep) {
                const int32_t at = cur[p->conv_elem[k]]++;
                face_id[at] = p->conv_face[k];
                face_film[at] = p->conv_film[k];
            }
        }
        double* coords = mem.take(dupload(p->coords, 3 * n, st));
        int64_t* conn64 = mem.take(dupload(p->conn, ne * npe, st));
        int32_t* conn = mem.take(dalloc<int32_t>(ne * npe));
        gpu_narrow(conn64, ne * npe, conn, st);
        double* kcond = mem.take(dupload(p->conductivity, ne, st));
        double* rhoc = mem.take(dupload(p->rho_c, ne, st));
        uint8_t* fixed = mem.take(dupload(p->fixed, n, st));
        double* imp = mem.take(dupload(p->imposed, n, st));
        if (p->imposed)
            gpu_zero_free(n, fixed, imp, st);
        else
            CK(cudaMemsetAsync(imp, 0, n * sizeof(double), st));
        int64_t* inc_ptr = mem.take(dalloc<int64_t>(n + 1));
        int32_t* inc = mem.take(dalloc<int32_t>(ne * npe));
        double* f = p->f ? mem.take(dupload(p->f, n, st)) : nullptr;
        double* initial = mem.take(dupload(p->initial, n, st));
        int32_t* fptr = mem.take(dupload(face_ptr.data(), face_ptr.size(), st));
        int32_t* fid = mem.take(dupload(face_id.data(), face_id.size(), st));
        double* ffilm = mem.take(dupload(face_film.data(), face_film.size(), st));
        double* left = mem.take(dalloc<double>((size_t)np * ne));
        double* right = mem.take(dalloc<double>((size_t)np * ne));
        CK(cudaEventRecord(ev[1], st));
        {
            HeatElemIn in{ne, coords, conn, kcond, rhoc, fptr, fid, ffilm, p->time_step, p->theta, p->theta - 1.0};
            counted();
            if (npe == 4)
                k_heat_elem<4><<<(unsigned)((ne + HeatTet<4>::G - 1) / HeatTet<4>::G), kT, 0, st>>>(in, left, right);
            else
                k_heat_elem<10><<<(unsigned)((ne + HeatTet<10>::G - 1) / HeatTet<10>::G), kT, 0, st>>>(in, left, right);
            CK(cudaGetLastError());
        }
        CK(cudaEventRecord(ev[2], st));
        gpu_incidence(conn, ne * npe, n, st, inc_ptr, inc);
        if (host_ordering) {
            analysis.join();
            if (!analysed) return th_fail(err.status, err.message);
        } else {
            std::vector<int32_t> h_kept_of(n, -1), h_kept;
            for (int64_t v = 0; v < n; ++v)
                if (!p->fixed[v]) {
                    h_kept_of[v] = (int32_t)h_kept.size();
                    h_kept.push_back((int32_t)v);
                }
            int32_t* d_kept_of = mem.take(dupload(h_kept_of.data(), h_kept_of.size(), st));
            std::vector<int32_t> order, level;
            gpu_ordering(npe, ne, conn, d_kept_of, (int32_t)h_kept.size(), ordering, st, order, level);
            analysis.join();
            if (!analysed) return th_fail(err.status, err.message);
            apply_ordering(h_kept, order, level, fixed3.data(), sym);
        }
        if (sym.levels >= kMaxLevels) return th_fail(MAILLE_INVALID_INPUT, "too many IC(0) levels");
        const int32_t nb = sym.nb;
        int32_t* perm = mem.take(dupload(sym.perm.data(), sym.perm.size(), st));
        int32_t* inv = mem.take(dupload(sym.inv.data(), sym.inv.size(), st));
        std::vector<int32_t> fixed_nodes;
        for (int64_t v = 0; v < n; ++v)
            if (p->fixed[v]) fixed_nodes.push_back((int32_t)v);
        int32_t* fnodes = mem.take(dupload(fixed_nodes.data(), fixed_nodes.size(), st));
        PatternDev pt;
        gpu_pattern(npe, ne, conn, inv, nb, st, pt, sym.row_ptr, sym.diag);
        for (void* q : {(void*)pt.row_ptr, (void*)pt.col, (void*)pt.diag, (void*)pt.tpos, (void*)pt.lslot,
                        (void*)pt.lrow, (void*)pt.lptr, (void*)pt.contrib})
            mem.take(q);
        sym.blocks = pt.blocks;
        sym.nl = pt.nl;
        {
            // lanes per row: MAILLE_THERMAL_LPR_A (the SpMV layouts; 0 picks from the mean row
            // length), MAILLE_THERMAL_LPR_LU (the triangles; 2 measured best on Tet10 40^3 against
            // 1 and 4: the sweeps are latency-bound, 16 rows a slice balance slices against steps)
            auto env = [](const char* k, int d) {
                const char* e = std::getenv(k);
                return e ? std::atoi(e) : d;
            };
            const int lpr_a = env("MAILLE_THERMAL_LPR_A", 0), lpr_lu = env("MAILLE_THERMAL_LPR_LU", 2);
            std::thread tk([&] { build_sell(sym, SELL_FULL, lpr_a, sk.h); });
            std::thread tl([&] { build_sell(sym, SELL_LOWER, lpr_lu, sl.h); });
            build_sell(sym, SELL_UPPER, lpr_lu, su.h);
            tk.join();
            tl.join();
        }
        sk.upload(pt, nb, st);
        sl.upload(pt, nb, st);
        su.upload(pt, nb, st);
        // assembly of the left and right matrices on the free-node pattern
        double* A = mem.take(dalloc<double>((size_t)pt.blocks));
        double* R = mem.take(dalloc<double>((size_t)pt.blocks));
        double* F = mem.take(dalloc<double>((size_t)pt.blocks));
        CK(cudaEventRecord(ev[3], st));
        counted();
        k_heat_assemble<<<grid_of(pt.nl), kT, 0, st>>>(pt.nl, ne, np, pt.lslot, pt.lptr, pt.contrib, pt.tpos, left,
                                                       right, A, R);
        CK(cudaGetLastError());
        CK(cudaEventRecord(ev[6], st));
        // IC(0) with the shift ladder (Pcg::new, iterative.rs:201-207)
        int32_t* dfail = mem.take(dalloc<int32_t>(1));
        double shift_used = -1.0;
        for (double shift : kShifts) {
            CK(cudaMemsetAsync(dfail, 0, sizeof(int32_t), st));
            for (int32_t l = 0; l < sym.levels; ++l) {
                const int32_t r0 = sym.level_ptr[l], r1 = sym.level_ptr[l + 1];
                if (r1 <= r0) continue;
                counted();
                k_heat_factor<<<(unsigned)(((int64_t)(r1 - r0) * 32 + kT - 1) / kT), kT, 0, st>>>(
                    pt.row_ptr, pt.col, pt.diag, pt.tpos, r0, r1, A, F, shift, dfail);
            }
            CK(cudaGetLastError());
            int32_t h_fail = 0;
            CK(cudaMemcpyAsync(&h_fail, dfail, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (!h_fail) {
                shift_used = shift;
                break;
            }
        }
        if (shift_used < 0.0) return th_fail(MAILLE_SINGULAR, "Singular: IC(0) failed for every diagonal shift");
        // iteration operands
        auto slots = [&](const Slices& s) { return (int64_t)s.h.steps() * kStepSlots; };
        double* Av = mem.take(dalloc<double>((size_t)slots(sk)));
        double* Rv = mem.take(dalloc<double>((size_t)slots(sk)));
        double* Lv = mem.take(dalloc<double>((size_t)slots(sl)));
        double* Uv = mem.take(dalloc<double>((size_t)slots(su)));
        double* D = mem.take(dalloc<double>((size_t)nb + 1));
        counted();
        k_gather_slots<<<grid_of(slots(sk)), kT, 0, st>>>(slots(sk), sk.src, A, Av);
        counted();
        k_gather_slots<<<grid_of(slots(sk)), kT, 0, st>>>(slots(sk), sk.src, R, Rv);
        counted();
        k_gather_slots<<<grid_of(slots(sl)), kT, 0, st>>>(slots(sl), sl.src, F, Lv);
        counted();
        k_gather_slots<<<grid_of(slots(su)), kT, 0, st>>>(slots(su), su.src, F, Uv);
        counted();
        k_gather_diag<<<grid_of(nb), kT, 0, st>>>(nb, pt.diag, F, D);
        static const double kOne = 1.0;  // the dummy row's pivot (its entries are never read)
        CK(cudaMemcpyAsync(D + nb, &kOne, sizeof(double), cudaMemcpyHostToDevice, st));
        CK(cudaGetLastError());
        // vectors and the constant part of the right-hand side
        const int64_t nv = (int64_t)nb + 1;
        double *x = mem.take(dalloc<double>(nv)), *r = mem.take(dalloc<double>(nv)), *pp = mem.take(dalloc<double>(nv)),
               *ap = mem.take(dalloc<double>(nv)), *b = mem.take(dalloc<double>(nv)), *g = mem.take(dalloc<double>(nv));
        for (double* q : {x, r, pp, ap, b}) CK(cudaMemsetAsync(q, 0, nv * sizeof(double), st));
        // sweep records (value, tag): tags start at 0, below every epoch; the dummy node's tag is
        // the largest, so padding slots never wait
        const bool mixed = p->precision == MAILLE_MIXED;
        double2* yrec = nullptr;
        double2* zrec = nullptr;
        float2* yrec32 = nullptr;
        float2* zrec32 = nullptr;
        if (!mixed) {
            yrec = mem.take(dalloc<double2>(nv));
            zrec = mem.take(dalloc<double2>(nv));
            static thread_local double2 h_dummy;
            const long long all_ones = -1LL;
            h_dummy.x = 0.0;
            std::memcpy(&h_dummy.y, &all_ones, sizeof(double));
            for (double2* q : {yrec, zrec}) {
                CK(cudaMemsetAsync(q, 0, nv * sizeof(double2), st));
                CK(cudaMemcpyAsync(q + nb, &h_dummy, sizeof(double2), cudaMemcpyHostToDevice, st));
            }
        } else {
            yrec32 = mem.take(dalloc<float2>(nv));
            zrec32 = mem.take(dalloc<float2>(nv));
            static thread_local float2 h_dummy32;
            const unsigned int ones = 0xFFFFFFFFu;
            h_dummy32.x = 0.0f;
            std::memcpy(&h_dummy32.y, &ones, sizeof(float));
            for (float2* q : {yrec32, zrec32}) {
                CK(cudaMemsetAsync(q, 0, nv * sizeof(float2), st));
                CK(cudaMemcpyAsync(q + nb, &h_dummy32, sizeof(float2), cudaMemcpyHostToDevice, st));
            }
        }
        // mixed form: FP32 copies of the operands and the FP32 work vectors (x64 = x, r64 the
        // true residual)
        float *Av32 = nullptr, *Lv32 = nullptr, *Uv32 = nullptr, *D32 = nullptr, *x32 = nullptr, *r32 = nullptr,
              *p32 = nullptr, *ap32 = nullptr;
        double* r64 = nullptr;
        if (mixed) {
            Av32 = mem.take(dalloc<float>((size_t)slots(sk)));
            Lv32 = mem.take(dalloc<float>((size_t)slots(sl)));
            Uv32 = mem.take(dalloc<float>((size_t)slots(su)));
            D32 = mem.take(dalloc<float>((size_t)nb + 1));
            for (int k = 0; k < 4; ++k) counted();
            k_to_float<<<grid_of(slots(sk)), kT, 0, st>>>(slots(sk), Av, Av32);
            k_to_float<<<grid_of(slots(sl)), kT, 0, st>>>(slots(sl), Lv, Lv32);
            k_to_float<<<grid_of(slots(su)), kT, 0, st>>>(slots(su), Uv, Uv32);
            k_to_float<<<grid_of(nv), kT, 0, st>>>(nv, D, D32);
            CK(cudaGetLastError());
            for (float** q : {&x32, &r32, &p32, &ap32}) {
                *q = mem.take(dalloc<float>(nv));
                CK(cudaMemsetAsync(*q, 0, nv * sizeof(float), st));
            }
            r64 = mem.take(dalloc<double>(nv));
            CK(cudaMemsetAsync(r64, 0, nv * sizeof(double), st));
        }
        // U's slices in backward sweep order (levels descending)
        std::vector<int32_t> bwd;
        bwd.reserve(su.h.nslices());
        for (int32_t l = sym.levels - 1; l >= 0; --l)
            for (int32_t q = su.h.level_slices[l]; q < su.h.level_slices[l + 1]; ++q) bwd.push_back(q);
        int32_t* bwd_slice = mem.take(dupload(bwd.data(), bwd.size(), st));
        int32_t* timeout = mem.take(dalloc<int32_t>(1));
        CK(cudaMemsetAsync(timeout, 0, sizeof(int32_t), st));
        counted();
        k_heat_const<<<grid_of(nv), kT, 0, st>>>(nb, npe, ne, perm, inc_ptr, inc, conn, fixed, imp, f, left, right, g);
        CK(cudaGetLastError());
        // the history
        const bool want_flux = res && res->heat_fluxes;
        double* temps = mem.take(dalloc<double>((size_t)(steps + 1) * n));
        double* react = mem.take(dalloc<double>((size_t)(steps + 1) * n));
        double* flux = want_flux ? mem.take(dalloc<double>((size_t)(steps + 1) * ne * ng * 6)) : nullptr;
        int32_t* d_status = mem.take(dalloc<int32_t>(steps));
        int32_t* d_iters = mem.take(dalloc<int32_t>(steps));
        double* d_rel = mem.take(dalloc<double>(steps));
        CK(cudaMemsetAsync(react, 0, (size_t)(steps + 1) * n * sizeof(double), st));
        auto fluxes = [&](int32_t s) {
            if (!want_flux) return;
            counted();
            if (npe == 4)
                k_heat_flux<4><<<grid_of(ne * ng), kT, 0, st>>>(ne, coords, conn, kcond, temps + (size_t)s * n,
                                                               flux + (size_t)s * ne * ng * 6);
            else
                k_heat_flux<10><<<grid_of(ne * ng), kT, 0, st>>>(ne, coords, conn, kcond, temps + (size_t)s * n,
                                                                flux + (size_t)s * ne * ng * 6);
        };
        // the persistent kernel: every block co-resident
        // two blocks of 256 threads per SM (128 registers a thread): 3 or 4 blocks (80 or 64
        // registers) spill and make every grid barrier dearer, measured slower in every phase
        int per_sm = 0, sms = 0, dev = p->device;
        void* pcg_fn = mixed ? (void*)k_heat_pcg<float, true> : (void*)k_heat_pcg<double, false>;
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_fn, kT, 0));
        const int grid = sms * std::min(per_sm, 2);
        if (grid <= 0) return th_fail(MAILLE_CUDA_ERROR, "the PCG kernel does not fit on the device");
        double* partials = mem.take(dalloc<double>((size_t)4 * grid));
        // MAILLE_PHASE_TIMING: device time of the PCG phases (block 0), printed at the end
        unsigned long long* timing = nullptr;
        if (const char* e = std::getenv("MAILLE_PHASE_TIMING"); e && std::atoi(e) != 0) {
            timing = mem.take(dalloc<unsigned long long>(4));
            CK(cudaMemsetAsync(timing, 0, 4 * sizeof(unsigned long long), st));
        }
        const int32_t* d_cancel = cancel_flag_device(p->device);
        CK(cudaEventRecord(ev[4], st));
        counted();
        k_heat_initial<<<grid_of(n), kT, 0, st>>>(n, inv, fixed, imp, initial, temps, x);
        fluxes(0);
        for (int32_t s = 1; s <= steps; ++s) {
            counted();
            k_heat_rhs<<<grid_of((int64_t)sk.h.nslices() * 32), kT, 0, st>>>(sk.dev(), Rv, x, g, b);
            counted();
            k_heat_gate<<<1, 1, 0, st>>>(d_cancel, s > 1 ? d_status + (s - 2) : nullptr, d_status + (s - 1));
            counted();
            if (!mixed) {
                HeatPcg<double> a{nb, sk.dev(), sl.dev(), su.dev(), bwd_slice, Av, Lv, Uv, D, b, x, r, pp, ap,
                                  yrec, zrec, partials, timeout, (unsigned long long)s << 32, tol, max_iter,
                                  d_status + (s - 1), d_iters + (s - 1), d_rel + (s - 1), timing,
                                  nullptr, nullptr, nullptr, 0.0};
                void* args[] = {&a};
                CK(cudaLaunchCooperativeKernel(pcg_fn, dim3(grid), dim3(kT), args, 0, st));
            } else {
                // 32-bit tags: increment s starts after the sweeps every earlier increment can take
                const unsigned long long epoch0 = (unsigned long long)(s - 1) * ((unsigned long long)max_iter + 2);
                HeatPcg<float> a{nb, sk.dev(), sl.dev(), su.dev(), bwd_slice, Av32, Lv32, Uv32, D32, b, x32, r32,
                                 p32, ap32, yrec32, zrec32, partials, timeout, epoch0, tol, max_iter,
                                 d_status + (s - 1), d_iters + (s - 1), d_rel + (s - 1), timing,
                                 Av, x, r64, kHeatDelta};
                void* args[] = {&a};
                CK(cudaLaunchCooperativeKernel(pcg_fn, dim3(grid), dim3(kT), args, 0, st));
            }
            counted();
            k_heat_scatter<<<grid_of(n), kT, 0, st>>>(n, inv, fixed, imp, x, temps + (size_t)s * n);
            if (!fixed_nodes.empty()) {
                counted();
                k_heat_react<<<grid_of((int64_t)fixed_nodes.size()), kT, 0, st>>>(
                    (int64_t)fixed_nodes.size(), fnodes, npe, ne, inc_ptr, inc, conn, left, right, f,
                    temps + (size_t)s * n, temps + (size_t)(s - 1) * n, react + (size_t)s * n);
            }
            fluxes(s);
            CK(cudaGetLastError());
        }
        CK(cudaEventRecord(ev[5], st));
        // results
        std::vector<int32_t> h_status(steps), h_iters(steps);
        std::vector<double> h_rel(steps);
        CK(cudaMemcpyAsync(h_status.data(), d_status, steps * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(h_iters.data(), d_iters, steps * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(h_rel.data(), d_rel, steps * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (timing) {
            unsigned long long t[4] = {0, 0, 0, 0};
            CK(cudaMemcpy(t, timing, sizeof(t), cudaMemcpyDeviceToHost));
            std::fprintf(stderr, "maille thermal phase timing (ms, block 0): spmv %.3f update %.3f sweeps %.3f "
                         "p %.3f grid %d\n", t[0] * 1e-6, t[1] * 1e-6, t[2] * 1e-6, t[3] * 1e-6, grid);
        }
        const double t_dl0 = now_ms();
        if (res) {
            if (res->temperatures)
                CK(cudaMemcpy(res->temperatures, temps, (size_t)(steps + 1) * n * sizeof(double), cudaMemcpyDeviceToHost));
            if (res->reactions)
                CK(cudaMemcpy(res->reactions, react, (size_t)(steps + 1) * n * sizeof(double), cudaMemcpyDeviceToHost));
            if (want_flux)
                CK(cudaMemcpy(res->heat_fluxes, flux, (size_t)(steps + 1) * ne * ng * 6 * sizeof(double),
                              cudaMemcpyDeviceToHost));
            int64_t total = 0;
            double worst = 0.0;
            for (int32_t s = 0; s < steps; ++s) {
                total += h_iters[s];
                worst = std::max(worst, h_rel[s]);
                if (res->iterations) res->iterations[s] = h_iters[s];
            }
            res->iterations_total = total;
            res->max_rel_residual = worst;
            res->shift = shift_used;
            res->free_nodes = nb;
            res->nonzeros = pt.blocks;
            res->levels = sym.levels;
            float ms = 0.0f;
            res->ms_setup = t_setup1 - t_setup0;
            CK(cudaEventElapsedTime(&ms, ev[0], ev[1]));
            res->ms_upload = ms;
            float ms2 = 0.0f;
            CK(cudaEventElapsedTime(&ms, ev[1], ev[2]));
            CK(cudaEventElapsedTime(&ms2, ev[3], ev[6]));
            res->ms_assembly = ms + ms2;  // element matrices, then the left and right matrices
            CK(cudaEventElapsedTime(&ms, ev[6], ev[4]));
            res->ms_factor = ms;  // IC(0) with its shift retries, the operands' slot fills
            CK(cudaEventElapsedTime(&ms, ev[4], ev[5]));
            res->ms_steps = ms;
            res->ms_download = now_ms() - t_dl0;
        }
        for (int32_t s = 0; s < steps; ++s) {
            if (h_status[s] == 6)
                return th_fail(MAILLE_CANCELLED, "Cancelled before increment " + std::to_string(s + 1));
            if (h_status[s] == 1) return th_fail(MAILLE_SINGULAR, "Singular at increment " + std::to_string(s + 1));
            if (h_status[s] == 3)
                return th_fail(MAILLE_CUDA_ERROR, "a sweep record wait timed out at increment " + std::to_string(s + 1));
            if (h_status[s] == 2)
                return th_fail(MAILLE_NOT_CONVERGED, "IterativeNotConverged at increment " + std::to_string(s + 1) +
                                                         ": iterations " + std::to_string(h_iters[s]) +
                                                         ", relative residual " + std::to_string(h_rel[s]));
        }
    } catch (const CudaFailure& e) {
        return th_fail(MAILLE_CUDA_ERROR, e.what);
    }
    return MAILLE_OK;
}

// nodal_source (assembly.rs:476-484) of a uniform source q over element e on its rule
void source_loads(int npe, const double (*xyz)[3], double q, double* fs) {
    const Rules r = make_rules();
    const int Q = npe == 4 ? 0 : 1, ng = npe == 4 ? 1 : 4;
    for (int a = 0; a < npe; ++a) fs[a] = 0.0;
    for (int g = 0; g < ng; ++g) {
        const double* l = r.elem[Q][g];
        double iv[9];
        const double det = npe == 4 ? jacobian<4>(xyz, l, iv) : jacobian<10>(xyz, l, iv);
        const double w = l[4] * std::fabs(det);
        for (int a = 0; a < npe; ++a) fs[a] += w * (npe == 4 ? shape_value<4>(l, a) : shape_value<10>(l, a)) * q;
    }
}

}  // namespace
}  // namespace maille

using namespace maille;

extern "C" {

int32_t maille_gpu_thermal_transient(const MailleThermalProblem* problem, MailleThermalResult* result) {
    set_last_error("");
    if (!problem) return th_fail(MAILLE_INVALID_INPUT, "null problem");
    return thermal_transient(problem, result);
}

int32_t maille_gpu_thermal_cancel(int32_t device, int32_t flag) {
    // the last error stays: a caller reads the message of the step it just cancelled afterwards
    if (device < 0 || device >= kMaxCancelDevices) return th_fail(MAILLE_INVALID_INPUT, "device out of range");
    try {
        *(volatile int32_t*)(cancel_flags() + device) = flag ? 1 : 0;
    } catch (const CudaFailure& e) {
        return th_fail(MAILLE_CUDA_ERROR, e.what);
    }
    return MAILLE_OK;
}

int32_t maille_gpu_thermal_loads(int64_t n_nodes, const double* coords, int32_t npe, int64_t n_elems,
                                 const int64_t* conn, int64_t n_sources, const int64_t* s_elem,
                                 const double* s_value, int64_t n_convection, const int64_t* c_elem,
                                 const int32_t* c_face, const double* c_film, const double* c_sink,
                                 double* f) {
    set_last_error("");
    if (!coords || !conn || !f || (n_sources > 0 && (!s_elem || !s_value)) ||
        (n_convection > 0 && (!c_elem || !c_face || !c_film || !c_sink)))
        return th_fail(MAILLE_INVALID_INPUT, "null argument");
    if (npe != 4 && npe != 10) return th_fail(MAILLE_INVALID_INPUT, "nodes_per_elem must be 4 or 10");
    auto node_ok = [&](int64_t e) {
        for (int a = 0; a < npe; ++a)
            if (conn[e * npe + a] < 0 || conn[e * npe + a] >= n_nodes) return false;
        return true;
    };
    auto gather = [&](int64_t e, double (*xyz)[3]) {
        for (int a = 0; a < npe; ++a)
            for (int c = 0; c < 3; ++c) xyz[a][c] = coords[3 * conn[e * npe + a] + c];
    };
    // heat sources (model.rs:1110-1115)
    for (int64_t k = 0; k < n_sources; ++k) {
        const int64_t e = s_elem[k];
        if (e < 0 || e >= n_elems) continue;
        if (!node_ok(e)) return th_fail(MAILLE_INVALID_INPUT, "source element refers to an unknown node");
        double xyz[10][3], fs[10];
        gather(e, xyz);
        source_loads(npe, xyz, s_value[k], fs);
        for (int a = 0; a < npe; ++a) f[conn[e * npe + a]] += fs[a];
    }
    // convection loads (model.rs:1136-1140): grouped by element, the faces' order kept
    std::vector<int64_t> order;
    for (int64_t k = 0; k < n_convection; ++k)
        if (c_elem[k] >= 0 && c_elem[k] < n_elems && c_face[k] >= 0 && c_face[k] <= 3) order.push_back(k);
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return c_elem[a] < c_elem[b]; });
    for (int64_t k : order) {
        const int64_t e = c_elem[k];
        if (!node_ok(e)) return th_fail(MAILLE_INVALID_INPUT, "convection element refers to an unknown node");
        double xyz[10][3];
        gather(e, xyz);
        int pos[6];
        const int nn = face_nodes(npe, c_face[k], pos);
        const double area2 = twice_area(xyz[pos[0]], xyz[pos[1]], xyz[pos[2]]);
        double load[6] = {0, 0, 0, 0, 0, 0};
        for (int g = 0; g < nn; ++g) {
            double nv[6];
            const double w = face_point(nn, g, nv) * area2;
            for (int a = 0; a < nn; ++a) load[a] += c_film[k] * c_sink[k] * w * nv[a];
        }
        for (int a = 0; a < nn; ++a) f[conn[e * npe + pos[a]]] += load[a];
    }
    return MAILLE_OK;
}

}  // extern "C"
