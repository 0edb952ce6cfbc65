// kernels.cu -- sm_100a kernels of the linear-elastic solve path. See kernels.cuh for the layout.
//
// Tensor cores stay off on purpose: no step is a dense contraction. Every kernel here is
// HBM-bandwidth bound except the element integration (FP64 FMA).

#include <atomic>
#include <cmath>

#include "kernels.cuh"
#include "reduce.cuh"
#include "tet.cuh"

namespace maille {

// kernels launched by this library since load (graph launches add their kernel nodes)
std::atomic<long long> g_kernel_launches{0};
namespace {

// ---- element integration --------------------------------------------------------------------

// Gauss points in barycentric coordinates (l0, l1, l2, l3): c_gp[0][0] is TETRA_1 (the
// centroid), c_gp[1][g] are the 4 points of TETRA_4 (quadrature.rs:100-138).
__constant__ double c_gp[2][4][4];
// node pairs (a <= b) of the element matrix, in the order a, then b
__constant__ int c_pa4[10], c_pb4[10], c_pa10[55], c_pb10[55];

template <int NPE>
__device__ __forceinline__ const double* gauss_point(int g) {
    return NPE == 4 ? c_gp[0][0] : c_gp[1][g];
}
template <int NPE>
__device__ __forceinline__ int pair_a(int p) { return NPE == 4 ? c_pa4[p] : c_pa10[p]; }
template <int NPE>
__device__ __forceinline__ int pair_b(int p) { return NPE == 4 ? c_pb4[p] : c_pb10[p]; }

template <int NPE>
struct Tet {
    static constexpr int NG = NPE == 4 ? 1 : 4;
    static constexpr int NP = NPE * (NPE + 1) / 2;
    static constexpr int G = NPE == 4 ? 32 : 16;  // elements per block
};

// K_e = sum_g w |det J| B^T D B (solid_stiffness, element.rs:223-243), written per node pair
// (a <= b) with the isotropic closed form of the 3x3 block
//   K_ab = sum_g w |det J| (lambda g_a g_b^T + mu g_b g_a^T + mu (g_a . g_b) I),
// g_a = dN_a/dx. One block of kThreads threads integrates G elements: coordinates and
// connectivity are staged in shared memory, then Jacobians, gradients and the node-pair
// blocks are computed by successive thread sweeps.
template <int NPE>
__global__ void __launch_bounds__(kThreads) k_elem_stiffness(ElemIn in, double* __restrict__ ke) {
    using TT = Tet<NPE>;
    constexpr int G = TT::G, NG = TT::NG, NP = TT::NP;
    __shared__ double xyz[G][NPE][3];
    __shared__ double wdet[G][NG];
    __shared__ double inv[G][NG][9];
    __shared__ double grad[G][NG][NPE][3];
    __shared__ double lam[G], mu[G];
    const int64_t e0 = (int64_t)blockIdx.x * G;
    for (int t = threadIdx.x; t < G * NPE; t += blockDim.x) {
        const int e = t / NPE, a = t - e * NPE;
        if (e0 + e < in.ne) {
            const int32_t v = in.conn[(e0 + e) * NPE + a];
            xyz[e][a][0] = in.coords[3 * (int64_t)v];
            xyz[e][a][1] = in.coords[3 * (int64_t)v + 1];
            xyz[e][a][2] = in.coords[3 * (int64_t)v + 2];
        }
    }
    for (int t = threadIdx.x; t < G; t += blockDim.x)
        if (e0 + t < in.ne) {
            const double E = in.young[e0 + t], nu = in.poisson[e0 + t];
            lam[t] = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
            mu[t] = E / (2.0 * (1.0 + nu));
        }
    __syncthreads();
    const double w = NPE == 4 ? 1.0 / 6.0 : 1.0 / 24.0;
    for (int t = threadIdx.x; t < G * NG; t += blockDim.x) {
        const int e = t / NG, g = t - e * NG;
        if (e0 + e < in.ne) wdet[e][g] = w * fabs(jacobian<NPE>(xyz[e], gauss_point<NPE>(g), inv[e][g]));
    }
    __syncthreads();
    for (int t = threadIdx.x; t < G * NG * NPE; t += blockDim.x) {
        const int e = t / (NG * NPE), g = (t / NPE) % NG, a = t % NPE;
        if (e0 + e < in.ne) {
            double d[3];
            dshape<NPE>(gauss_point<NPE>(g), a, d);
            const double* iv = inv[e][g];
#pragma unroll
            for (int r = 0; r < 3; ++r) grad[e][g][a][r] = iv[3 * r] * d[0] + iv[3 * r + 1] * d[1] + iv[3 * r + 2] * d[2];
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < G * NP; t += blockDim.x) {
        const int e = t / NP, p = t - e * NP;
        if (e0 + e >= in.ne) continue;
        const int a = pair_a<NPE>(p), b = pair_b<NPE>(p);
        double k[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int g = 0; g < NG; ++g) {
            const double* ga = grad[e][g][a];
            const double* gb = grad[e][g][b];
            const double f = wdet[e][g];
            const double dotab = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    k[3 * i + j] += f * (lam[e] * ga[i] * gb[j] + mu[e] * gb[i] * ga[j] + (i == j ? mu[e] * dotab : 0.0));
        }
        double* out = ke + ((e0 + e) * NP + p) * 9;
#pragma unroll
        for (int q = 0; q < 9; ++q) out[q] = k[q];
    }
}

// ---- deterministic assembly -----------------------------------------------------------------

// One thread per lower slot (I, J), J <= I: sums its element-pair blocks in the order of the
// precomputed map (element order), applies the identity rows/columns of fixed DOFs, and writes
// the block and its transpose.
__global__ void k_assemble(Pattern pt, int64_t nl, const int64_t* __restrict__ lslot,
                           const int32_t* __restrict__ lrow, const int64_t* __restrict__ lptr,
                           const uint32_t* __restrict__ contrib, const double* __restrict__ ke,
                           double* __restrict__ K) {
    const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nl) return;
    const int64_t pos = lslot[l];
    const int32_t I = lrow[l], J = pt.col[pos];
    double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t k = lptr[l]; k < lptr[l + 1]; ++k) {
        const uint32_t c = contrib[k];
        const double* B = ke + (int64_t)(c & 0x7fffffffu) * 9;
        if (c & 0x80000000u) {
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int q = 0; q < 3; ++q) s[3 * r + q] += B[3 * q + r];
        } else {
#pragma unroll
            for (int q = 0; q < 9; ++q) s[q] += B[q];
        }
    }
    const uint8_t mi = pt.fixmask[I], mj = pt.fixmask[J];
    if (mi | mj) {
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int q = 0; q < 3; ++q)
                if (((mi >> r) & 1) || ((mj >> q) & 1)) s[3 * r + q] = (I == J && r == q) ? 1.0 : 0.0;
    }
    double* out = K + 9 * pos;
#pragma unroll
    for (int q = 0; q < 9; ++q) out[q] = s[q];
    if (I != J) {
        double* tr = K + 9 * pt.tpos[pos];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int q = 0; q < 3; ++q) tr[3 * q + r] = s[3 * r + q];
    }
}

// ---- IC(0) factorisation --------------------------------------------------------------------

// Block IC(0) of one level (rows r0..r1), one warp per block row I. Equal, up to rounding, to the
// reference's scalar row-oriented IC(0) (Csr::incomplete_cholesky, iterative.rs:146-170) on the
// same node ordering: for each lower block J (ascending)
//   L_IJ = (A_IJ - sum_{K<J, K in row I and row J} L_IK L_JK^T) L_JJ^-T,
// then L_II = chol(A_II - sum_K L_IK L_IK^T) with the diagonal entries scaled by (1 + shift) and
// every scalar pivot checked like the reference (NaN or <= 1e-12 a_ii fails the shift).
__global__ void __launch_bounds__(kThreads) k_factor(Pattern pt, int32_t r0, int32_t r1,
                                                      const double* __restrict__ K, double* F,
                                                      double shift, int32_t* fail) {
    const int lane = threadIdx.x & 31;
    const int32_t I = r0 + (int32_t)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (I >= r1) return;
    if (*(volatile int32_t*)fail) return;
    const int64_t rb = pt.row_ptr[I], rd = pt.diag[I];
    for (int64_t p = rb; p < rd; ++p) {
        const int32_t J = pt.col[p];
        const int64_t jb = pt.row_ptr[J], jd = pt.diag[J];
        double S[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int64_t q = rb + lane; q < p; q += 32) {
            const int32_t kc = pt.col[q];
            int64_t lo = jb, hi = jd;
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                if (pt.col[mid] < kc) lo = mid + 1; else hi = mid;
            }
            if (lo < jd && pt.col[lo] == kc) {
                const double* A = F + 9 * q;
                const double* B = F + 9 * lo;
#pragma unroll
                for (int r = 0; r < 3; ++r)
#pragma unroll
                    for (int c = 0; c < 3; ++c)
                        S[3 * r + c] += A[3 * r] * B[3 * c] + A[3 * r + 1] * B[3 * c + 1] + A[3 * r + 2] * B[3 * c + 2];
            }
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) S[k] = warp_sum(S[k]);
        if (lane == 0) {
            const double* A = K + 9 * p;
            const double* D = F + 9 * jd;  // L_JJ^-1, lower triangular
            double M[9], L[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) M[k] = A[k] - S[k];
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    L[3 * r + c] = M[3 * r] * D[3 * c] + M[3 * r + 1] * D[3 * c + 1] + M[3 * r + 2] * D[3 * c + 2];
            double* o = F + 9 * p;
            double* t = F + 9 * pt.tpos[p];
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    o[3 * r + c] = L[3 * r + c];
                    t[3 * c + r] = L[3 * r + c];
                }
        }
        __syncwarp();
    }
    double S[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t q = rb + lane; q < rd; q += 32) {
        const double* A = F + 9 * q;
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                S[3 * r + c] += A[3 * r] * A[3 * c] + A[3 * r + 1] * A[3 * c + 1] + A[3 * r + 2] * A[3 * c + 2];
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) S[k] = warp_sum(S[k]);
    if (lane == 0) {
        const double* A = K + 9 * rd;
        const double m00 = A[0] * (1.0 + shift) - S[0];
        const double m10 = A[3] - S[3], m20 = A[6] - S[6];
        const double m11 = A[4] * (1.0 + shift) - S[4];
        const double m21 = A[7] - S[7];
        const double m22 = A[8] * (1.0 + shift) - S[8];
        bool ok = true;
        const double p0 = m00;
        ok = ok && !(isnan(p0) || p0 <= 1e-12 * A[0]);
        const double l00 = sqrt(p0);
        const double l10 = m10 / l00, l20 = m20 / l00;
        const double p1 = m11 - l10 * l10;
        ok = ok && !(isnan(p1) || p1 <= 1e-12 * A[4]);
        const double l11 = sqrt(p1);
        const double l21 = (m21 - l20 * l10) / l11;
        const double p2 = m22 - l20 * l20 - l21 * l21;
        ok = ok && !(isnan(p2) || p2 <= 1e-12 * A[8]);
        const double l22 = sqrt(p2);
        if (!ok) {
            atomicExch(fail, 1);
        } else {
            const double d00 = 1.0 / l00, d11 = 1.0 / l11, d22 = 1.0 / l22;
            const double d10 = -l10 * d00 * d11;
            const double d21 = -l21 * d11 * d22;
            const double d20 = -(l20 * d00 + l21 * d10) * d22;
            double* o = F + 9 * rd;
            o[0] = d00; o[1] = 0.0; o[2] = 0.0;
            o[3] = d10; o[4] = d11; o[5] = 0.0;
            o[6] = d20; o[7] = d21; o[8] = d22;
        }
    }
}

// ---- right-hand side, solution, boundary products -------------------------------------------

// b_I = F_f - K_fc u_c in solver numbering (padded: 4 entries per node), 0 at fixed DOFs of kept nodes (FreeSystem::solve,
// model.rs:1503-1508).
__global__ void k_build_rhs(int32_t nb, const int32_t* __restrict__ perm,
                            const uint8_t* __restrict__ fixmask, const double* __restrict__ f,
                            const double* __restrict__ coupling, double* __restrict__ b) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * (int64_t)nb) return;
    const int32_t I = (int32_t)(t >> 2);
    const int c = (int)(t & 3);
    double v = 0.0;
    if (c < 3 && !((fixmask[I] >> c) & 1)) {
        const int64_t g = 3 * (int64_t)perm[I] + c;
        v = (f ? f[g] : 0.0) - (coupling ? coupling[g] : 0.0);
    }
    b[t] = v;  // padded layout: 4 entries per node, the 4th is 0
}

// u = imposed at fixed DOFs, x at free DOFs (model.rs:581, 1509-1514)
__global__ void k_gather_u(int64_t n_nodes, const int32_t* __restrict__ inv,
                           const uint8_t* __restrict__ fixed, const double* __restrict__ imposed,
                           const double* __restrict__ x, double* __restrict__ u) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= 3 * n_nodes) return;
    const int64_t v = g / 3;
    const int c = (int)(g - 3 * v);
    const int32_t I = inv[v];
    u[g] = (fixed && fixed[g]) ? imposed[g] : (I >= 0 ? x[4 * (int64_t)I + c] : 0.0);
}

__device__ __forceinline__ int pair_index(int npe, int a, int b) {
    return a * npe - a * (a - 1) / 2 + (b - a);
}

// ye[k] = K_e u_e for the listed elements, one thread per (element, local DOF row).
__global__ void k_elem_apply(int npe, int64_t nlist, const int32_t* __restrict__ list,
                             const int32_t* __restrict__ conn, const double* __restrict__ ke,
                             const double* __restrict__ u, double* __restrict__ ye) {
    const int m = 3 * npe;
    const int np = npe * (npe + 1) / 2;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nlist * m) return;
    const int64_t k = t / m;
    const int i = (int)(t - k * m);
    const int64_t e = list[k];
    const int a = i / 3, ii = i - 3 * (i / 3);
    double s = 0.0;
    for (int b = 0; b < npe; ++b) {
        const int64_t v = conn[e * npe + b];
        const double* B = a <= b ? ke + (e * np + pair_index(npe, a, b)) * 9
                                 : ke + (e * np + pair_index(npe, b, a)) * 9;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double kij = a <= b ? B[3 * ii + j] : B[3 * j + ii];
            s += kij * u[3 * v + j];
        }
    }
    ye[t] = s;
}

// y[3 v + c] = sum over the elements of node v of their ye rows (element order).
__global__ void k_node_gather(int npe, int64_t nnodes, const int32_t* __restrict__ nodes,
                              const int64_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc,
                              const int32_t* __restrict__ elem_slot, const double* __restrict__ ye,
                              double* __restrict__ y) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nnodes) return;
    const int32_t v = nodes[t];
    const int m = 3 * npe;
    double s0 = 0, s1 = 0, s2 = 0;
    for (int64_t q = inc_ptr[v]; q < inc_ptr[v + 1]; ++q) {
        const int32_t ea = inc[q];
        const int32_t e = ea / npe, a = ea - e * npe;
        const int32_t slot = elem_slot[e];
        if (slot < 0) continue;
        const double* r = ye + (int64_t)slot * m + 3 * a;
        s0 += r[0];
        s1 += r[1];
        s2 += r[2];
    }
    y[3 * (int64_t)v] = s0;
    y[3 * (int64_t)v + 1] = s1;
    y[3 * (int64_t)v + 2] = s2;
}

// reactions = K u - F at fixed DOFs (model.rs:586-593)
__global__ void k_reactions(const int32_t* __restrict__ nodes, int64_t nnodes,
                            const uint8_t* __restrict__ fixed, const double* __restrict__ y,
                            const double* __restrict__ f, double* __restrict__ react) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * nnodes) return;
    const int64_t g = 3 * (int64_t)nodes[t / 3] + (t % 3);
    react[g] = fixed[g] ? y[g] - (f ? f[g] : 0.0) : 0.0;
}

// sigma = D B u_e at every Gauss point and its von Mises value (solid_stresses,
// element.rs:270-302; Stress::von_mises, results.rs:24-32). One thread per (element, point).
template <int NPE>
__global__ void k_stresses(ElemIn in, const double* __restrict__ u, double* __restrict__ gauss,
                           double* __restrict__ vm) {
    constexpr int NG = Tet<NPE>::NG;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= in.ne * NG) return;
    const int64_t e = t / NG;
    const int g = (int)(t - e * NG);
    double xyz[NPE][3], ue[NPE][3];
    for (int a = 0; a < NPE; ++a) {
        const int64_t v = in.conn[e * NPE + a];
        for (int c = 0; c < 3; ++c) {
            xyz[a][c] = in.coords[3 * v + c];
            ue[a][c] = u[3 * v + c];
        }
    }
    const double* l = gauss_point<NPE>(g);
    double iv[9];
    jacobian<NPE>(xyz, l, iv);
    double eps[6] = {0, 0, 0, 0, 0, 0};  // xx, yy, zz, yz, xz, xy (engineering shears)
    double pos[3] = {0, 0, 0};
    for (int a = 0; a < NPE; ++a) {
        double d[3], gr[3];
        dshape<NPE>(l, a, d);
        for (int r = 0; r < 3; ++r) gr[r] = iv[3 * r] * d[0] + iv[3 * r + 1] * d[1] + iv[3 * r + 2] * d[2];
        eps[0] += gr[0] * ue[a][0];
        eps[1] += gr[1] * ue[a][1];
        eps[2] += gr[2] * ue[a][2];
        eps[3] += gr[2] * ue[a][1] + gr[1] * ue[a][2];
        eps[4] += gr[2] * ue[a][0] + gr[0] * ue[a][2];
        eps[5] += gr[1] * ue[a][0] + gr[0] * ue[a][1];
        const double n = shape_value<NPE>(l, a);
        for (int c = 0; c < 3; ++c) pos[c] += n * xyz[a][c];
    }
    const double E = in.young[e], nu = in.poisson[e];
    const double cc = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double gg = E / (2.0 * (1.0 + nu));
    const double dd = cc * (1.0 - nu), od = cc * nu;
    const double sxx = dd * eps[0] + od * eps[1] + od * eps[2];
    const double syy = od * eps[0] + dd * eps[1] + od * eps[2];
    const double szz = od * eps[0] + od * eps[1] + dd * eps[2];
    const double tyz = gg * eps[3], txz = gg * eps[4], txy = gg * eps[5];
    double* o = gauss + t * 9;
    o[0] = pos[0];
    o[1] = pos[1];
    o[2] = pos[2];
    o[3] = sxx;
    o[4] = syy;
    o[5] = szz;
    o[6] = txy;
    o[7] = tyz;
    o[8] = txz;
    if (vm) {
        const double shear = txy * txy + tyz * tyz + txz * txz;
        const double q = sxx * sxx + syy * syy + szz * szz - sxx * syy - syy * szz - szz * sxx + 3.0 * shear;
        vm[t] = sqrt(q > 0.0 ? q : 0.0);
    }
}

// Nodal smoothing of the Gauss-point stresses (nodal_stresses / smooth, results.rs:137-230): each
// element's Gauss values are extrapolated to its nodes (Tet4: the single point's value,
// TET4_EXTRAPOLATION results.rs:98; Tet10: TET10_EXTRAPOLATION results.rs:118-132, the weights of
// the 4 points for the 4 vertices and 6 mid-edge nodes) and averaged over the elements sharing
// the node; a node no element touches gets 0. One thread per node gathers its incident elements in
// element order (the incidence list is sorted by element), with separately rounded products and
// sums in the reference's order, so the result equals the sequential accumulation exactly. Also
// writes Stress::von_mises (results.rs:24-32) of the smoothed stress, in the reference's order.
// gauss: [ne * ng * 9] (x, y, z, sxx, syy, szz, txy, tyz, txz); stress: [n * 6] (sxx, syy, szz,
// txy, tyz, txz); vm: [n].
// TET10_EXTRAPOLATION (results.rs:114-132): with the barycentric coordinates a = (5 + 3 sqrt 5) / 20,
// b = (5 - sqrt 5) / 20 of TETRA_4's points, a vertex takes (3 sqrt 5 + 1) / 4 of its own point and
// -(sqrt 5 - 1) / 4 of the others, a mid-edge node (sqrt 5 + 1) / 4 of the points of its two
// vertices (Tet10 edge order 0-1, 1-2, 2-0, 0-3, 1-3, 2-3) and -(sqrt 5 - 1) / 4 of the others.
__device__ __forceinline__ double tet10_extrapolation(int a, int g) {
    constexpr double V = 1.9270509831248424, M = 0.8090169943749475, O = -0.30901699437494745;
    if (a < 4) return g == a ? V : O;
    constexpr int ei[6] = {0, 1, 2, 0, 1, 2}, ej[6] = {1, 2, 0, 3, 3, 3};
    return (g == ei[a - 4] || g == ej[a - 4]) ? M : O;
}

__global__ void k_nodal_stresses(int npe, int64_t n_nodes, const int64_t* __restrict__ inc_ptr,
                                 const int32_t* __restrict__ inc, const double* __restrict__ gauss,
                                 double* __restrict__ stress, double* __restrict__ vm) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_nodes) return;
    const int ng = npe == 4 ? 1 : 4;
    double s[6] = {0, 0, 0, 0, 0, 0};
    const int64_t q0 = inc_ptr[v], q1 = inc_ptr[v + 1];
    for (int64_t q = q0; q < q1; ++q) {
        const int32_t k = inc[q];
        const int64_t e = k / npe;
        const int a = (int)(k - e * npe);
        for (int g = 0; g < ng; ++g) {
            const double w = npe == 4 ? 1.0 : tet10_extrapolation(a, g);
            const double* p = gauss + (e * ng + g) * 9 + 3;
#pragma unroll
            for (int c = 0; c < 6; ++c) s[c] = __dadd_rn(s[c], __dmul_rn(w, p[c]));
        }
    }
    const double cnt = (double)(q1 - q0 > 0 ? q1 - q0 : 1);
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        s[c] = __ddiv_rn(s[c], cnt);
        stress[6 * v + c] = s[c];
    }
    const double a = s[0], b = s[1], c = s[2];
    const double shear = __dadd_rn(__dadd_rn(__dmul_rn(s[3], s[3]), __dmul_rn(s[4], s[4])), __dmul_rn(s[5], s[5]));
    double t = __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c));
    t = __dsub_rn(t, __dmul_rn(a, b));
    t = __dsub_rn(t, __dmul_rn(b, c));
    t = __dsub_rn(t, __dmul_rn(c, a));
    t = __dadd_rn(t, __dmul_rn(3.0, shear));
    vm[v] = __dsqrt_rn(t > 0.0 ? t : 0.0);
}

// dJ/dE_e = -lambda_e^T (dK_e/dE_e) u_e = -lambda_e^T K_e u_e / E_e (K_e is linear in E_e).
__global__ void k_adjoint_grad(int npe, int64_t ne, const int32_t* __restrict__ conn,
                               const double* __restrict__ ke, const double* __restrict__ young,
                               const double* __restrict__ lambda, const double* __restrict__ u,
                               double* __restrict__ grad) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const int np = npe * (npe + 1) / 2;
    double lam[10][3], uu[10][3];
    for (int a = 0; a < npe; ++a) {
        const int64_t v = conn[e * npe + a];
        for (int c = 0; c < 3; ++c) {
            lam[a][c] = lambda[3 * v + c];
            uu[a][c] = u[3 * v + c];
        }
    }
    double s = 0.0;
    for (int a = 0; a < npe; ++a)
        for (int b = a; b < npe; ++b) {
            const double* B = ke + (e * np + pair_index(npe, a, b)) * 9;
            double q = 0.0;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    q += lam[a][i] * B[3 * i + j] * uu[b][j];
                    if (a != b) q += lam[b][j] * B[3 * i + j] * uu[a][i];
                }
            s += q;
        }
    grad[e] = -s / young[e];
}

inline int blocks_for(int64_t n, int threads, int64_t cap) {
    int64_t b = (n + threads - 1) / threads;
    if (b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}

bool g_consts_ready[64] = {false};

void ensure_consts() {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && g_consts_ready[dev]) return;
    const double A = 0.5854101966249685, B = 0.1381966011250105;  // TET_A, TET_B
    // TETRA_4 point g = (xi, eta, zeta) has barycentric TET_A on vertex g and TET_B elsewhere.
    const double gp[2][4][4] = {
        {{0.25, 0.25, 0.25, 0.25}, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}},
        {{1.0 - B - B - B, B, B, B}, {1.0 - A - B - B, A, B, B}, {1.0 - B - A - B, B, A, B},
         {1.0 - B - B - A, B, B, A}}};
    cudaMemcpyToSymbol(c_gp, gp, sizeof(gp));
    int pa4[10], pb4[10], pa10[55], pb10[55];
    for (int npe : {4, 10}) {
        int q = 0;
        for (int a = 0; a < npe; ++a)
            for (int b = a; b < npe; ++b) {
                (npe == 4 ? pa4 : pa10)[q] = a;
                (npe == 4 ? pb4 : pb10)[q] = b;
                ++q;
            }
    }
    cudaMemcpyToSymbol(c_pa4, pa4, sizeof(pa4));
    cudaMemcpyToSymbol(c_pb4, pb4, sizeof(pb4));
    cudaMemcpyToSymbol(c_pa10, pa10, sizeof(pa10));
    cudaMemcpyToSymbol(c_pb10, pb10, sizeof(pb10));
    if (dev >= 0 && dev < 64) g_consts_ready[dev] = true;
}

}  // namespace

void launch_elem_stiffness(int npe, const ElemIn& in, double* ke_up, cudaStream_t st) {
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    ensure_consts();
    if (npe == 4)
        k_elem_stiffness<4><<<(unsigned)((in.ne + Tet<4>::G - 1) / Tet<4>::G), kThreads, 0, st>>>(in, ke_up);
    else
        k_elem_stiffness<10><<<(unsigned)((in.ne + Tet<10>::G - 1) / Tet<10>::G), kThreads, 0, st>>>(in, ke_up);
}

void launch_assemble(const Pattern& pt, int64_t nl, const int64_t* lslot, const int32_t* lrow,
                     const int64_t* lptr, const uint32_t* contrib, const double* ke_up, double* K,
                     cudaStream_t st) {
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    k_assemble<<<blocks_for(nl, kThreads, INT32_MAX), kThreads, 0, st>>>(pt, nl, lslot, lrow, lptr,
                                                                       contrib, ke_up, K);
}

void launch_factor_level(const Pattern& pt, int32_t r0, int32_t r1, const double* K, double* F,
                         double shift, int32_t* fail, cudaStream_t st) {
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    const int64_t rows = r1 - r0;
    k_factor<<<blocks_for(rows, kWarps, INT32_MAX), kThreads, 0, st>>>(pt, r0, r1, K, F, shift, fail);
}

void launch_build_rhs(int32_t nb, const int32_t* perm, const uint8_t* fixmask, const double* f,
                      const double* coupling, double* b, cudaStream_t st) {
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    k_build_rhs<<<blocks_for(4 * (int64_t)nb, kThreads, INT32_MAX), kThreads, 0, st>>>(nb, perm, fixmask, f, coupling, b);
}

void launch_gather_u(int64_t n_nodes, const int32_t* inv, const uint8_t* fixed,
                     const double* imposed, const double* x, double* u, cudaStream_t st) {
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    k_gather_u<<<blocks_for(3 * n_nodes, kThreads, INT32_MAX), kThreads, 0, st>>>(n_nodes, inv, fixed, imposed, x, u);
}

void launch_elem_apply(int npe, int64_t nlist, const int32_t* list, const int32_t* conn,
                       const double* ke_up, const double* u, double* ye, cudaStream_t st) {
    if (nlist <= 0) return;
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    k_elem_apply<<<blocks_for(nlist * 3 * npe, kThreads, INT32_MAX), kThreads, 0, st>>>(npe, nlist, list, conn, ke_up, u, ye);
}

void launch_node_gather(int npe, int64_t nnodes, const int32_t* nodes, const int64_t* inc_ptr,
                        const int32_t* inc, const int32_t* elem_slot, const double* ye, double* y,
                        cudaStream_t st) {
    if (nnodes <= 0) return;
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    k_node_gather<<<blocks_for(nnodes, kThreads, INT32_MAX), kThreads, 0, st>>>(npe, nnodes, nodes, inc_ptr, inc, elem_slot, ye, y);
}

void launch_reactions(int64_t n_nodes, const int32_t* nodes, int64_t nnodes, const uint8_t* fixed,
                      const double* y, const double* f, double* react, cudaStream_t st) {
    (void)n_nodes;
    if (nnodes <= 0) return;
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    k_reactions<<<blocks_for(3 * nnodes, kThreads, INT32_MAX), kThreads, 0, st>>>(nodes, nnodes, fixed, y, f, react);
}

void launch_stresses(int npe, const ElemIn& in, const double* u, double* gauss, double* vm,
                     cudaStream_t st) {
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    ensure_consts();
    const int ng = npe == 4 ? 1 : 4;
    if (npe == 4)
        k_stresses<4><<<blocks_for(in.ne * ng, 128, INT32_MAX), 128, 0, st>>>(in, u, gauss, vm);
    else
        k_stresses<10><<<blocks_for(in.ne * ng, 128, INT32_MAX), 128, 0, st>>>(in, u, gauss, vm);
}

void launch_nodal_stresses(int npe, int64_t n_nodes, const int64_t* inc_ptr, const int32_t* inc,
                           const double* gauss, double* stress, double* vm, cudaStream_t st) {
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    k_nodal_stresses<<<(unsigned)((n_nodes + 127) / 128), 128, 0, st>>>(npe, n_nodes, inc_ptr, inc, gauss,
                                                                        stress, vm);
}

void launch_adjoint_grad(int npe, int64_t ne, const int32_t* conn, const double* ke_up,
                         const double* young, const double* lambda, const double* u, double* grad,
                         cudaStream_t st) {
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    k_adjoint_grad<<<blocks_for(ne, 128, INT32_MAX), 128, 0, st>>>(npe, ne, conn, ke_up, young, lambda, u, grad);
}

}  // namespace maille
