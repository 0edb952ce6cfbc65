// large_strain.cu -- neo-Hookean Tet4 in large strain on the GPU: the quasi-static Newton loop of
// Model::solve_quasi_static (model.rs:720-1022) with IC(0)-PCG inner solves, per-increment
// checkpoints of the converged displacements, and the adjoint of increment reactions with
// respect to the per-element Lame parameters (C ABI maille_gpu_large_strain_*).
//
// Every Newton iteration runs on the device: element responses (internal force and tangent,
// large_strain_response, finite_strain.rs:119-214), the deterministic nodal gather of the
// internal force (internal_force, model.rs:1241-1249), the residual norms, then the linear
// step of the single-model handle (scatter-reduce assembly of the tangents, IC(0) with the shift
// ladder, PCG on K_ff du_f = -r_f - K_fc du_c, FreeSystem::new/solve, model.rs:1442-1516). The
// host reads three norms per iteration to decide convergence, as the reference does.
//
// The tangent uses a closed form of the neo-Hookean material term: with C^-1 the inverse right
// Cauchy-Green tensor, a_n = F C^-1 g_n for the shape gradient g_n of node n and
// m = mu - lambda ln J, the finite_strain.rs contraction sum_IJKL F_iI g_aJ C_IJKL F_kK g_bL equals
//   lambda (a_a)_i (a_b)_k + m [ delta_ik (g_a . C^-1 g_b) + (a_b)_i (a_a)_k ]
// because F C^-1 F^T = I; the geometric term adds delta_ik (g_a . S g_b).

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "handle.hpp"
#include "reduce.cuh"

namespace maille {

namespace {

constexpr int kLsThreads = 128;

struct Tet4Geo {
    double g[4][3];  // dN_a/dX
    double w;        // TETRA_1 weight x |det J|
};

// solid_gauss with TETRA_1 (element.rs:338-357) on a Tet4: constant shape gradients
__device__ __forceinline__ Tet4Geo tet4_geo(const double* __restrict__ coords, const int32_t* nd) {
    const double dl[4][3] = {{-1.0, -1.0, -1.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
    double x[4][3];
    for (int a = 0; a < 4; ++a)
        for (int r = 0; r < 3; ++r) x[a][r] = coords[3 * (int64_t)nd[a] + r];
    double j[3][3] = {};
    for (int k = 0; k < 4; ++k)
        for (int i = 0; i < 3; ++i)
            for (int r = 0; r < 3; ++r) j[i][r] += dl[k][i] * x[k][r];
    auto cof = [&](int r, int c) {
        const int r1 = (r + 1) % 3, r2 = (r + 2) % 3, c1 = (c + 1) % 3, c2 = (c + 2) % 3;
        return j[r1][c1] * j[r2][c2] - j[r1][c2] * j[r2][c1];
    };
    const double det = j[0][0] * cof(0, 0) + j[0][1] * cof(0, 1) + j[0][2] * cof(0, 2);
    Tet4Geo t;
    for (int k = 0; k < 4; ++k)
        for (int r = 0; r < 3; ++r)
            t.g[k][r] = (cof(0, r) * dl[k][0] + cof(1, r) * dl[k][1] + cof(2, r) * dl[k][2]) / det;
    t.w = fabs(det) / 6.0;
    return t;
}

struct NeoState {
    double f[3][3], ci[3][3], s[3][3], logj;
};

// F = I + sum_a u_a (x) g_a, C^-1, S = mu (I - C^-1) + lambda ln J C^-1 (finite_strain.rs:40-86)
__device__ __forceinline__ NeoState neo_state(const Tet4Geo& t, const double (&ue)[12], double lam, double mu) {
    NeoState n;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double v = i == j ? 1.0 : 0.0;
            for (int a = 0; a < 4; ++a) v += ue[3 * a + i] * t.g[a][j];
            n.f[i][j] = v;
        }
    double c[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) c[i][j] = n.f[0][i] * n.f[0][j] + n.f[1][i] * n.f[1][j] + n.f[2][i] * n.f[2][j];
    const double dc = c[0][0] * (c[1][1] * c[2][2] - c[1][2] * c[2][1]) - c[0][1] * (c[1][0] * c[2][2] - c[1][2] * c[2][0]) +
                      c[0][2] * (c[1][0] * c[2][1] - c[1][1] * c[2][0]);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const int r0 = (j + 1) % 3, r1 = (j + 2) % 3, c0 = (i + 1) % 3, c1 = (i + 2) % 3;
            n.ci[i][j] = (c[r0][c0] * c[r1][c1] - c[r0][c1] * c[r1][c0]) / dc;
        }
    const double (&f)[3][3] = n.f;
    const double jf = f[0][0] * (f[1][1] * f[2][2] - f[1][2] * f[2][1]) - f[0][1] * (f[1][0] * f[2][2] - f[1][2] * f[2][0]) +
                      f[0][2] * (f[1][0] * f[2][1] - f[1][1] * f[2][0]);
    n.logj = log(jf);  // NaN when J <= 0: the caller reports a non-finite residual
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) n.s[i][j] = mu * ((i == j ? 1.0 : 0.0) - n.ci[i][j]) + lam * n.logj * n.ci[i][j];
    return n;
}

__device__ __forceinline__ int pair_of(int a, int b) { return a * 4 - a * (a - 1) / 2 + (b - a); }

// Element internal forces fe [12 per element] and tangents as node-pair blocks a <= b
// (ke[(e * 10 + pair) * 9 + 3 i + k] = K_e[3a + i][3b + k]).
__global__ void __launch_bounds__(kLsThreads) k_ls_response(int64_t ne, const double* __restrict__ coords,
                                                            const int32_t* __restrict__ conn,
                                                            const double* __restrict__ lam_e,
                                                            const double* __restrict__ mu_e,
                                                            const double* __restrict__ u, double* __restrict__ fe,
                                                            double* __restrict__ ke) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    int32_t nd[4];
    for (int a = 0; a < 4; ++a) nd[a] = conn[e * 4 + a];
    const Tet4Geo t = tet4_geo(coords, nd);
    double ue[12];
    for (int a = 0; a < 4; ++a)
        for (int c = 0; c < 3; ++c) ue[3 * a + c] = u[3 * (int64_t)nd[a] + c];
    const double lam = lam_e[e], mu = mu_e[e];
    const NeoState n = neo_state(t, ue, lam, mu);
    // P = F S; f_a = w P g_a
    double p[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) p[i][j] = n.f[i][0] * n.s[0][j] + n.f[i][1] * n.s[1][j] + n.f[i][2] * n.s[2][j];
    for (int a = 0; a < 4; ++a)
        for (int i = 0; i < 3; ++i)
            fe[e * 12 + 3 * a + i] = t.w * (p[i][0] * t.g[a][0] + p[i][1] * t.g[a][1] + p[i][2] * t.g[a][2]);
    // a_n = F C^-1 g_n, sg_n = S g_n, cg_n = C^-1 g_n
    double av[4][3], sg[4][3], cg[4][3];
    for (int a = 0; a < 4; ++a)
        for (int i = 0; i < 3; ++i) {
            sg[a][i] = n.s[i][0] * t.g[a][0] + n.s[i][1] * t.g[a][1] + n.s[i][2] * t.g[a][2];
            cg[a][i] = n.ci[i][0] * t.g[a][0] + n.ci[i][1] * t.g[a][1] + n.ci[i][2] * t.g[a][2];
        }
    for (int a = 0; a < 4; ++a)
        for (int i = 0; i < 3; ++i) av[a][i] = n.f[i][0] * cg[a][0] + n.f[i][1] * cg[a][1] + n.f[i][2] * cg[a][2];
    const double m = mu - lam * n.logj;
    for (int a = 0; a < 4; ++a)
        for (int b = a; b < 4; ++b) {
            const double gsg = t.g[a][0] * sg[b][0] + t.g[a][1] * sg[b][1] + t.g[a][2] * sg[b][2];
            const double gcg = t.g[a][0] * cg[b][0] + t.g[a][1] * cg[b][1] + t.g[a][2] * cg[b][2];
            double* K = ke + (e * 10 + pair_of(a, b)) * 9;
            for (int i = 0; i < 3; ++i)
                for (int k = 0; k < 3; ++k)
                    K[3 * i + k] = t.w * ((i == k ? gsg + m * gcg : 0.0) + lam * av[a][i] * av[b][k] + m * av[b][i] * av[a][k]);
        }
}

// Nodal internal force: the incident elements' forces summed in element order (deterministic).
__global__ void k_ls_gather(int64_t n_nodes, const int64_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc,
                            const double* __restrict__ fe, double* __restrict__ fint) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * n_nodes) return;
    const int64_t v = t / 3;
    const int c = (int)(t - 3 * v);
    double s = 0.0;
    for (int64_t q = inc_ptr[v]; q < inc_ptr[v + 1]; ++q) s += fe[(int64_t)inc[q] * 3 + c];
    fint[t] = s;
}

// r = F_int - lambda F; minus_r = -r; ordered sums of |F_int|^2, |lambda F|^2 and |r_free|^2
__global__ void __launch_bounds__(256) k_ls_norms(int64_t n3, double lam, const double* __restrict__ fint,
                                                  const double* __restrict__ fext, const uint8_t* __restrict__ fixed,
                                                  double* __restrict__ resid, double* __restrict__ minus_r,
                                                  double* partials, unsigned int* ticket, double* out) {
    __shared__ double sh[8];
    double a = 0.0, b = 0.0, c = 0.0;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n3; g += (int64_t)gridDim.x * blockDim.x) {
        const double ext = fext ? lam * fext[g] : 0.0;
        const double r = fint[g] - ext;
        resid[g] = r;
        minus_r[g] = -r;
        a += fint[g] * fint[g];
        b += ext * ext;
        if (!fixed[g]) c += r * r;
    }
    const int G = gridDim.x;
    const double ta = block_sum(a, sh);
    const double tb = block_sum(b, sh);
    const double tc = block_sum(c, sh);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = ta;
        partials[G + blockIdx.x] = tb;
        partials[2 * G + blockIdx.x] = tc;
        __threadfence();
        last = atomicAdd(ticket, 1u) == (unsigned)G - 1;
    }
    __syncthreads();
    if (!last) return;
    const double sa = gather_sum(partials, G, sh);
    const double sb = gather_sum(partials + G, G, sh);
    const double sc = gather_sum(partials + 2 * G, G, sh);
    if (threadIdx.x == 0) {
        out[0] = sa;
        out[1] = sb;
        out[2] = sc;
        *ticket = 0;
    }
}

// du_c = lambda * imposed - u at fixed DOFs, 0 elsewhere (model.rs:1001-1007)
__global__ void k_ls_du_c(int64_t n3, double lam, const uint8_t* __restrict__ fixed, const double* __restrict__ imposed,
                          const double* __restrict__ u, double* __restrict__ duc) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n3) return;
    duc[g] = fixed[g] ? lam * imposed[g] - u[g] : 0.0;
}

__global__ void k_ls_add(int64_t n3, double* __restrict__ u, const double* __restrict__ du) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g < n3) u[g] += du[g];
}

// reactions = r at fixed DOFs (model.rs:985-990)
__global__ void k_ls_reactions(int64_t n3, const uint8_t* __restrict__ fixed, const double* __restrict__ r,
                               double* __restrict__ out) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g < n3) out[g] = fixed[g] ? r[g] : 0.0;
}

// w = g at fixed DOFs (the weights), 0 elsewhere
__global__ void k_ls_weights(int64_t n3, const uint8_t* __restrict__ fixed, const double* __restrict__ g,
                             double* __restrict__ w) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n3) w[t] = fixed[t] ? g[t] : 0.0;
}

// dJ/dmu_e += w_e . dfe/dmu, dJ/dlambda_e += w_e . dfe/dlambda at the displacements u:
// dfe/dmu_a = w F (I - C^-1) g_a, dfe/dlambda_a = w ln J F C^-1 g_a
__global__ void __launch_bounds__(kLsThreads) k_ls_grad(int64_t ne, const double* __restrict__ coords,
                                                        const int32_t* __restrict__ conn,
                                                        const double* __restrict__ lam_e, const double* __restrict__ mu_e,
                                                        const double* __restrict__ u, const double* __restrict__ wv,
                                                        double* __restrict__ gmu, double* __restrict__ glam) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    int32_t nd[4];
    for (int a = 0; a < 4; ++a) nd[a] = conn[e * 4 + a];
    const Tet4Geo t = tet4_geo(coords, nd);
    double ue[12];
    for (int a = 0; a < 4; ++a)
        for (int c = 0; c < 3; ++c) ue[3 * a + c] = u[3 * (int64_t)nd[a] + c];
    const NeoState n = neo_state(t, ue, lam_e[e], mu_e[e]);
    double dm = 0.0, dl = 0.0;
    for (int a = 0; a < 4; ++a) {
        double cg[3], hg[3];
        for (int i = 0; i < 3; ++i) {
            cg[i] = n.ci[i][0] * t.g[a][0] + n.ci[i][1] * t.g[a][1] + n.ci[i][2] * t.g[a][2];
            hg[i] = t.g[a][i] - cg[i];  // (I - C^-1) g_a
        }
        for (int i = 0; i < 3; ++i) {
            const double w = wv[3 * (int64_t)nd[a] + i];
            dm += w * t.w * (n.f[i][0] * hg[0] + n.f[i][1] * hg[1] + n.f[i][2] * hg[2]);
            dl += w * t.w * n.logj * (n.f[i][0] * cg[0] + n.f[i][1] * cg[1] + n.f[i][2] * cg[2]);
        }
    }
    gmu[e] += dm;
    if (glam) glam[e] += dl;
}

unsigned blocks_of(int64_t n, int threads) { return (unsigned)std::max<int64_t>(1, (n + threads - 1) / threads); }

constexpr double kNewtonTol = 1e-8;   // model.rs:1220
constexpr int kNewtonIters = 25;      // model.rs:1222
constexpr int kMaxCuts = 5;           // model.rs:1224
// Status of an inner PCG that hit its iteration cap inside the Newton loop: the reference's
// IterativeNotConverged (error.rs:226-229), which advance passes up without a cut (model.rs:839-842
// cuts on NotConverged, Singular and PlasticCollapse only). Reported as MAILLE_NOT_CONVERGED.
constexpr int32_t kIterativeNotConverged = 100;

}  // namespace
}  // namespace maille

struct MailleGpuLargeStrain {
    MailleGpuHandle* h = nullptr;
    int32_t increments = 10, newton_max = kNewtonIters;
    double newton_tol = kNewtonTol;
    int64_t n_nodes = 0, n_elems = 0;
    std::vector<double> h_young, h_poisson;
    // device
    double *lam = nullptr, *mu = nullptr, *fext = nullptr, *imp_final = nullptr, *u = nullptr, *u_trial = nullptr,
           *du = nullptr, *duc = nullptr, *fe = nullptr, *fint = nullptr, *resid = nullptr, *minus_r = nullptr,
           *zero = nullptr, *ckpt = nullptr, *react = nullptr, *wv = nullptr, *gmu = nullptr, *glam = nullptr,
           *partials = nullptr, *norms = nullptr, *h_norms = nullptr;
    unsigned int* ticket = nullptr;
    double* saved_imposed = nullptr;  // the handle's own imposed array (restored on destroy)
    bool has_fext = false, ran = false;
    double scale = 0.0;
    int64_t newton_total = 0, pcg_total = 0;
    std::vector<int32_t> newton_iters, cuts;
    int norm_grid = 0;  // 4 blocks per SM, set at creation
    ~MailleGpuLargeStrain() {
        if (h) {
            cudaSetDevice(h->device);
            h->imposed = saved_imposed;
            h->f_cur = h->f0;
        }
        for (double* p : {lam, mu, fext, imp_final, u, u_trial, du, duc, fe, fint, resid, minus_r, zero, ckpt, react,
                          wv, gmu, glam, partials, norms})
            dfree(p);
        dfree(ticket);
        pinned_slot_free(h_norms);
        if (h) maille_gpu_destroy(h);
    }
};

namespace {

using maille::CudaFailure;

int32_t ls_fail(int32_t status, const std::string& m) {
    maille::set_last_error(m);
    return status;
}

// element responses at `u` into h->ke (tangent) and fe, the nodal internal force and the norms
void ls_responses(MailleGpuLargeStrain* s, const double* u, double lam, double out[3]) {
    MailleGpuHandle* h = s->h;
    cudaStream_t st = h->st;
    const int64_t n3 = 3 * s->n_nodes;
    maille::k_ls_response<<<maille::blocks_of(s->n_elems, maille::kLsThreads), maille::kLsThreads, 0, st>>>(
        s->n_elems, h->coords, h->conn, s->lam, s->mu, u, s->fe, h->ke);
    maille::k_ls_gather<<<maille::blocks_of(n3, 256), 256, 0, st>>>(s->n_nodes, h->inc_ptr, h->inc, s->fe, s->fint);
    maille::k_ls_norms<<<s->norm_grid, 256, 0, st>>>(n3, lam, s->fint, s->has_fext ? s->fext : nullptr, h->fixed,
                                                     s->resid, s->minus_r, s->partials, s->ticket, s->norms);
    maille::g_kernel_launches.fetch_add(3, std::memory_order_relaxed);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(s->h_norms, s->norms, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int k = 0; k < 3; ++k) out[k] = s->h_norms[k];
}

// K_ff x_f = rhs_f - K_fc xc (xc at fixed DOFs) with the tangent in h->ke: assembly, IC(0), PCG,
// then x (caller numbering, xc at fixed DOFs) into `out`.
int32_t ls_linear_solve(MailleGpuLargeStrain* s, const double* rhs, const double* xc, double* out, std::string& msg) {
    MailleGpuHandle* h = s->h;
    maille::Error err{MAILLE_OK, ""};
    if (maille::handle_assemble_factor(h, err) != MAILLE_OK) {
        msg = err.message;
        return err.status;
    }
    h->f_cur = rhs;
    h->imposed = const_cast<double*>(xc);
    h->any_imposed = true;
    maille::handle_build_rhs(h);
    int32_t iters = 0, outer = 0;
    double rel = 0.0;
    const int32_t status = maille::handle_run_pcg(h, &iters, &outer, &rel);
    s->pcg_total += iters;
    if (status != MAILLE_OK) {
        msg = maille::handle_status_message(status, iters, rel);
        return status == MAILLE_NOT_CONVERGED ? maille::kIterativeNotConverged : status;
    }
    maille::launch_gather_u(s->n_nodes, h->inv, h->fixed, xc, h->x64, out, h->st);
    CK(cudaGetLastError());
    return MAILLE_OK;
}

// equilibrium (model.rs:923-1022): Newton from u_trial to F_int = lam F, u_c = lam imposed.
int32_t equilibrium(MailleGpuLargeStrain* s, double lam, double& sc, int32_t& iterations, std::string& msg) {
    MailleGpuHandle* h = s->h;
    cudaStream_t st = h->st;
    const int64_t n3 = 3 * s->n_nodes;
    int32_t count = 0;
    for (;;) {
        if (h->cancel.load()) {  // the observer's Flow::Stop between Newton iterations (model.rs:1203-1218)
            msg = "Cancelled";
            return MAILLE_CANCELLED;
        }
        double nr[3];
        ls_responses(s, s->u_trial, lam, nr);
        sc = std::max(std::max(sc, std::sqrt(nr[0])), std::sqrt(nr[1]));
        const double free = std::sqrt(nr[2]);
        const double relative = sc > 0.0 ? free / sc : free;
        if (!std::isfinite(relative)) {
            msg = "Newton-Raphson: non-finite residual";
            return MAILLE_NOT_CONVERGED;
        }
        ++count;
        ++s->newton_total;
        if (count > 1 && relative <= s->newton_tol) {
            iterations = count;
            return MAILLE_OK;
        }
        if (count > s->newton_max) {
            msg = "Newton-Raphson did not converge";
            return MAILLE_NOT_CONVERGED;
        }
        maille::k_ls_du_c<<<maille::blocks_of(n3, 256), 256, 0, st>>>(n3, lam, h->fixed, s->imp_final, s->u_trial, s->duc);
        maille::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
        const int32_t status = ls_linear_solve(s, s->minus_r, s->duc, s->du, msg);
        if (status != MAILLE_OK) return status;
        maille::k_ls_add<<<maille::blocks_of(n3, 256), 256, 0, st>>>(n3, s->u_trial, s->du);
        maille::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    }
}

// advance (model.rs:820-870): halves the interval up to kMaxCuts times when Newton does not
// converge or meets a tangent that is not positive definite (IC(0) failing every shift, or
// p.Ap <= 0 in the PCG); an inner PCG at its cap is passed up without a cut.
int32_t advance(MailleGpuLargeStrain* s, double t0, double t1, int cuts, int32_t& iterations, int32_t& cut_count,
                std::string& msg) {
    const int64_t n3 = 3 * s->n_nodes;
    cudaStream_t st = s->h->st;
    CK(cudaMemcpyAsync(s->u_trial, s->u, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    double sc = s->scale;
    const int32_t status = equilibrium(s, t1, sc, iterations, msg);  // amplitude lambda(t) = t
    if (status == MAILLE_OK) {
        CK(cudaMemcpyAsync(s->u, s->u_trial, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
        s->scale = sc;
        return MAILLE_OK;
    }
    if ((status == MAILLE_NOT_CONVERGED || status == MAILLE_SINGULAR) && cuts < maille::kMaxCuts) {
        const double middle = 0.5 * (t0 + t1);
        ++cut_count;
        const int32_t a = advance(s, t0, middle, cuts + 1, iterations, cut_count, msg);
        if (a != MAILLE_OK) return a;
        return advance(s, middle, t1, cuts + 1, iterations, cut_count, msg);
    }
    return status;
}

int32_t ls_run(MailleGpuLargeStrain* s, MailleLargeStrainResult* res) {
    NvtxRange nvtx("maille large-strain run");
    MailleGpuHandle* h = s->h;
    cudaStream_t st = h->st;
    const int64_t n3 = 3 * s->n_nodes;
    const double t0 = maille::now_ms();
    CK(cudaMemsetAsync(s->u, 0, n3 * sizeof(double), st));
    s->scale = 0.0;
    s->newton_total = 0;
    s->pcg_total = 0;
    s->newton_iters.assign(s->increments, 0);
    s->cuts.assign(s->increments, 0);
    s->ran = false;
    const double dt = 1.0 / s->increments;
    for (int inc = 1; inc <= s->increments; ++inc) {
        const double time = inc * dt;
        int32_t iterations = 0, cut_count = 0;
        std::string msg;
        const int32_t status = advance(s, time - dt, time, 0, iterations, cut_count, msg);
        s->cuts[inc - 1] = cut_count;
        if (status != MAILLE_OK) {
            if (res) {  // the failing increment's halvings and the counts so far
                if (res->newton_iterations)
                    std::memcpy(res->newton_iterations, s->newton_iters.data(), s->increments * sizeof(int32_t));
                if (res->cuts) std::memcpy(res->cuts, s->cuts.data(), s->increments * sizeof(int32_t));
                res->newton_total = s->newton_total;
                res->pcg_total = s->pcg_total;
                res->ms_total = maille::now_ms() - t0;
            }
            return ls_fail(status == maille::kIterativeNotConverged ? MAILLE_NOT_CONVERGED : status,
                           "increment " + std::to_string(inc) + ": " + msg);
        }
        s->newton_iters[inc - 1] = iterations;
        // checkpoint and reactions of the converged increment (resid holds F_int - lam F at u)
        CK(cudaMemcpyAsync(s->ckpt + (size_t)(inc - 1) * n3, s->u, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
        maille::k_ls_reactions<<<maille::blocks_of(n3, 256), 256, 0, st>>>(n3, h->fixed, s->resid,
                                                                            s->react + (size_t)(inc - 1) * n3);
        maille::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    }
    CK(cudaGetLastError());
    if (res) {
        if (res->u) CK(cudaMemcpyAsync(res->u, s->ckpt, s->increments * n3 * sizeof(double), cudaMemcpyDeviceToHost, st));
        if (res->reactions)
            CK(cudaMemcpyAsync(res->reactions, s->react, s->increments * n3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    s->ran = true;
    if (res) {
        if (res->newton_iterations) std::memcpy(res->newton_iterations, s->newton_iters.data(), s->increments * sizeof(int32_t));
        if (res->cuts) std::memcpy(res->cuts, s->cuts.data(), s->increments * sizeof(int32_t));
        res->newton_total = s->newton_total;
        res->pcg_total = s->pcg_total;
        res->ms_total = maille::now_ms() - t0;
    }
    return MAILLE_OK;
}

int32_t ls_backward(MailleGpuLargeStrain* s, const double* dJdR, double* dJdmu, double* dJdlambda) {
    NvtxRange nvtx("maille large-strain backward");
    if (!s->ran) return ls_fail(MAILLE_INVALID_INPUT, "backward needs a completed run");
    MailleGpuHandle* h = s->h;
    cudaStream_t st = h->st;
    const int64_t n3 = 3 * s->n_nodes;
    const size_t total = (size_t)s->increments * n3;
    for (size_t k = 0; k < total; ++k)
        if (!std::isfinite(dJdR[k])) return ls_fail(MAILLE_INVALID_INPUT, "non-finite dJ/dR");
    CK(cudaMemsetAsync(s->gmu, 0, s->n_elems * sizeof(double), st));
    CK(cudaMemsetAsync(s->glam, 0, s->n_elems * sizeof(double), st));
    for (int k = s->increments - 1; k >= 0; --k) {
        const double* g = dJdR + (size_t)k * n3;
        bool any = false;
        for (int64_t q = 0; q < n3 && !any; ++q) any = h->h_fixed[q] && g[q] != 0.0;
        if (!any) continue;
        // the weights at fixed DOFs, the tangent at the checkpoint
        CK(cudaMemcpyAsync(s->duc, g, n3 * sizeof(double), cudaMemcpyHostToDevice, st));
        maille::k_ls_weights<<<maille::blocks_of(n3, 256), 256, 0, st>>>(n3, h->fixed, s->duc, s->wv);
        maille::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
        double nr[3];
        const double* uk = s->ckpt + (size_t)k * n3;
        ls_responses(s, uk, 0.0, nr);
        // K_ff m_f = -K_fc g_c; w = (g_c, m_f)
        std::string msg;
        const int32_t status = ls_linear_solve(s, s->zero, s->wv, s->du, msg);
        if (status != MAILLE_OK) return ls_fail(status, "adjoint solve of increment " + std::to_string(k + 1) + ": " + msg);
        maille::k_ls_grad<<<maille::blocks_of(s->n_elems, maille::kLsThreads), maille::kLsThreads, 0, st>>>(
            s->n_elems, h->coords, h->conn, s->lam, s->mu, uk, s->du, s->gmu, s->glam);
        maille::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
        CK(cudaGetLastError());
    }
    CK(cudaMemcpyAsync(dJdmu, s->gmu, s->n_elems * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (dJdlambda) CK(cudaMemcpyAsync(dJdlambda, s->glam, s->n_elems * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return MAILLE_OK;
}

int32_t ls_set_materials(MailleGpuLargeStrain* s, const double* young, const double* poisson) {
    for (int64_t e = 0; e < s->n_elems; ++e) {
        const double E = young ? young[e] : s->h_young[e], nu = poisson ? poisson[e] : s->h_poisson[e];
        if (!std::isfinite(E) || !std::isfinite(nu) || E <= 0.0 || nu <= -1.0 || nu >= 0.5)
            return ls_fail(MAILLE_INVALID_INPUT, "invalid material of element " + std::to_string(e));
    }
    if (young) std::memcpy(s->h_young.data(), young, s->n_elems * sizeof(double));
    if (poisson) std::memcpy(s->h_poisson.data(), poisson, s->n_elems * sizeof(double));
    // large_strain_law (assembly.rs:55-61): lame(E, nu), finite_strain.rs:30-35
    std::vector<double> lam(s->n_elems), mu(s->n_elems);
    for (int64_t e = 0; e < s->n_elems; ++e) {
        const double E = s->h_young[e], nu = s->h_poisson[e];
        lam[e] = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
        mu[e] = E / (2.0 * (1.0 + nu));
    }
    cudaStream_t st = s->h->st;
    CK(cudaMemcpyAsync(s->lam, lam.data(), s->n_elems * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s->mu, mu.data(), s->n_elems * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    s->ran = false;
    return MAILLE_OK;
}

int32_t ls_create(const MailleLargeStrainProblem* p, MailleGpuLargeStrain** out) {
    if (!out) return ls_fail(MAILLE_INVALID_INPUT, "null handle pointer");
    *out = nullptr;
    if (!p) return ls_fail(MAILLE_INVALID_INPUT, "null problem");
    if (p->increments <= 0) return ls_fail(MAILLE_INVALID_INPUT, "increments must be positive");
    if (p->f)
        for (int64_t k = 0; k < 3 * p->n_nodes; ++k)
            if (!std::isfinite(p->f[k])) return ls_fail(MAILLE_INVALID_INPUT, "non-finite load");
    MailleElasticProblem ep{};
    ep.n_nodes = p->n_nodes;
    ep.coords = p->coords;
    ep.nodes_per_elem = 4;
    ep.n_elems = p->n_elems;
    ep.conn = p->conn;
    ep.young = p->young;
    ep.poisson = p->poisson;
    ep.fixed = p->fixed;
    ep.imposed = p->imposed;
    ep.f = nullptr;
    ep.rel_tol = p->rel_tol;
    ep.max_iter = p->max_iter;
    ep.precision = p->precision;
    ep.ordering = MAILLE_ORDER_MULTICOLOR;
    ep.device = p->device;
    auto s = std::make_unique<MailleGpuLargeStrain>();
    int32_t status = maille::handle_create(&ep, &s->h, nullptr);
    if (status != MAILLE_OK) return status;
    s->saved_imposed = s->h->imposed;
    s->increments = p->increments;
    s->newton_tol = p->newton_tol > 0 ? p->newton_tol : maille::kNewtonTol;
    s->newton_max = p->newton_max_iter > 0 ? p->newton_max_iter : maille::kNewtonIters;
    s->n_nodes = p->n_nodes;
    s->n_elems = p->n_elems;
    s->h_young.assign(p->young, p->young + p->n_elems);
    s->h_poisson.assign(p->poisson, p->poisson + p->n_elems);
    try {
        const int64_t n3 = 3 * p->n_nodes;
        cudaStream_t st = s->h->st;
        s->lam = maille::dalloc<double>(p->n_elems);
        s->mu = maille::dalloc<double>(p->n_elems);
        for (double** q : {&s->u, &s->u_trial, &s->du, &s->duc, &s->fint, &s->resid, &s->minus_r, &s->zero, &s->wv,
                           &s->imp_final}) {
            *q = maille::dalloc<double>(n3);
            CK(cudaMemsetAsync(*q, 0, n3 * sizeof(double), st));
        }
        // final imposed values at fixed DOFs (0 elsewhere)
        std::vector<double> imp(n3, 0.0);
        if (p->imposed && p->fixed)
            for (int64_t k = 0; k < n3; ++k)
                if (p->fixed[k]) imp[k] = p->imposed[k];
        CK(cudaMemcpyAsync(s->imp_final, imp.data(), n3 * sizeof(double), cudaMemcpyHostToDevice, st));
        if (p->f) {
            s->fext = maille::dupload(p->f, n3, st);
            s->has_fext = true;
        }
        s->fe = maille::dalloc<double>((size_t)p->n_elems * 12);
        s->ckpt = maille::dalloc<double>((size_t)p->increments * n3);
        s->react = maille::dalloc<double>((size_t)p->increments * n3);
        s->gmu = maille::dalloc<double>(p->n_elems);
        s->glam = maille::dalloc<double>(p->n_elems);
        s->norm_grid = 4 * maille::device_sms();
        s->partials = maille::dalloc<double>(3 * (size_t)s->norm_grid);
        s->norms = maille::dalloc<double>(4);
        s->ticket = maille::dalloc<unsigned int>(2);
        CK(cudaMemsetAsync(s->ticket, 0, 2 * sizeof(unsigned int), st));
        s->h_norms = static_cast<double*>(pinned_slot_alloc(4 * sizeof(double)));
        status = ls_set_materials(s.get(), nullptr, nullptr);
        if (status != MAILLE_OK) return status;
    } catch (const CudaFailure& e) {
        return ls_fail(MAILLE_CUDA_ERROR, e.what);
    }
    *out = s.release();
    return MAILLE_OK;
}

}  // namespace

extern "C" {

int32_t maille_gpu_large_strain_create(const MailleLargeStrainProblem* problem, MailleGpuLargeStrain** out) {
    maille::set_last_error("");
    return ls_create(problem, out);
}

int32_t maille_gpu_large_strain_run(MailleGpuLargeStrain* s, MailleLargeStrainResult* result) {
    maille::set_last_error("");
    if (!s) return ls_fail(MAILLE_INVALID_INPUT, "null handle");
    try {
        CK(cudaSetDevice(s->h->device));
        return ls_run(s, result);
    } catch (const CudaFailure& e) {
        return ls_fail(MAILLE_CUDA_ERROR, e.what);
    }
}

int32_t maille_gpu_large_strain_backward(MailleGpuLargeStrain* s, const double* dJdR, double* dJdmu,
                                         double* dJdlambda) {
    maille::set_last_error("");
    if (!s || !dJdR || !dJdmu) return ls_fail(MAILLE_INVALID_INPUT, "null argument");
    try {
        CK(cudaSetDevice(s->h->device));
        return ls_backward(s, dJdR, dJdmu, dJdlambda);
    } catch (const CudaFailure& e) {
        return ls_fail(MAILLE_CUDA_ERROR, e.what);
    }
}

int32_t maille_gpu_large_strain_set_materials(MailleGpuLargeStrain* s, const double* young, const double* poisson) {
    maille::set_last_error("");
    if (!s) return ls_fail(MAILLE_INVALID_INPUT, "null handle");
    try {
        CK(cudaSetDevice(s->h->device));
        return ls_set_materials(s, young, poisson);
    } catch (const CudaFailure& e) {
        return ls_fail(MAILLE_CUDA_ERROR, e.what);
    }
}

void maille_gpu_large_strain_cancel(MailleGpuLargeStrain* s, int32_t flag) {
    if (s && s->h) s->h->cancel.store(flag ? 1 : 0);
}

void maille_gpu_large_strain_destroy(MailleGpuLargeStrain* s) { delete s; }

}  // extern "C"
