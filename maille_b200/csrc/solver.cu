// solver.cu -- handle lifecycle, PCG driver (plain FP64 and mixed FP32/FP64 refinement) and the
// C ABI of include/maille_gpu.h.
//
// create = FreeSystem::new + Pcg::new (model.rs:1442-1499, iterative.rs:201-207) on the GPU:
//   symbolic analysis (host, setup.cpp) -> upload -> element integration -> scatter-reduce
//   assembly -> level-scheduled block IC(0) with the reference's diagonal-shift ladder.
// solve  = FreeSystem::solve + Pcg::solve (model.rs:1502-1516, iterative.rs:210-248), then the
//   reactions (product, model.rs:586-593) and Gauss-point stresses (model.rs:596-598).
// The PCG runs in the persistent cooperative kernel of persist.cu: one launch for the initial
// preconditioning, then launches of `persist_chunk` iterations until the device flags the end
// (the host reads the device scalars after each launch: stopping, cancel flag).

#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "common.hpp"
#include "cuda_host.hpp"
#include "handle.hpp"
#include "kernels.cuh"
#include "ordering.cuh"
#include "sparse.cuh"

using namespace maille;

namespace {

thread_local std::string g_last_error;

}  // namespace

MailleGpuHandle::~MailleGpuHandle() {
    cudaSetDevice(device);
    if (st) cudaStreamSynchronize(st);
    if (timing) {
        unsigned long long t[8] = {0};
        cudaMemcpy(t, timing, sizeof(t), cudaMemcpyDeviceToHost);
        std::fprintf(stderr,
                     "maille phase timing (ms, block 0): spmv %.3f axpy %.3f update %.3f fwd %.3f "
                     "bwd %.3f pupdate %.3f launches %llu grid %d\n",
                     t[0] * 1e-6, t[1] * 1e-6, t[2] * 1e-6, t[3] * 1e-6, t[4] * 1e-6, t[5] * 1e-6,
                     t[6], persist_grid);
    }
    void* bufs[] = {coords, young, poisson, imposed, f, f0, conn, fixed, perm, inv, col, lrow, fixmask,
                    row_ptr, diag, tpos, lslot, lptr, contrib, inc_ptr, inc, belem, bnodes,
                    elem_slot, ke, K, F, Ks64, Ls64, Us64, D64, Ks32, Ls32, Us32, D32, b64, x64,
                    r64, z64, p64, ap64, x32, r32, z32, p32, ap32, u_full, y_full, ye, gauss, vm,
                    react, lambda_full, grad, node_stress, node_vm, scal, partials, timing, claim, dsum, dticket, dfail};
    // one device synchronisation for all of them (a free per buffer waited for the device each time)
    const bool stage_timing = std::getenv("MAILLE_SETUP_TIMING") != nullptr;
    const double t0 = now_ms();
    std::vector<void*> all(std::begin(bufs), std::end(bufs));
    sk.gather(all);
    pl.gather(all);
    pu.gather(all);
    device_free_all(all);
    const double t1 = now_ms();
    pinned_slot_free(h_scal);
    pinned_slot_free(h_sum);
    const double t2 = now_ms();
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    if (st) cudaStreamDestroy(st);
    if (stage_timing)
        std::fprintf(stderr, "maille destroy: device frees %.1f ms, host frees %.1f ms, events and stream %.1f ms\n",
                     t1 - t0, t2 - t1, now_ms() - t2);
}

namespace {

float elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

int grid_for_slices(int64_t slices) {
    int64_t g = (slices + kWarps - 1) / kWarps;
    const int64_t cap = 8 * (int64_t)device_sms();
    if (g > cap) g = cap;
    return (int)(g < 1 ? 1 : g);
}

bool is_mixed(const MailleGpuHandle* h) { return h->precision == MAILLE_MIXED; }

template <typename T>
PcgArgs<T> pcg_args(MailleGpuHandle* h, const T* Kv, const T* Lv, const T* Uv, const T* D, T* x,
                    T* r, T* z, T* p, T* ap) {
    PcgArgs<T> a{};
    a.nb = h->sym.nb;
    a.levels = h->sym.levels;
    a.chunk = h->persist_chunk;
    a.K = h->sk.dev();
    a.L = h->pl.dev();
    a.U = h->pu.dev();
    a.Kv = Kv;
    a.Lv = Lv;
    a.Uv = Uv;
    a.D = D;
    a.x = x;
    a.r = r;
    a.z = z;
    a.p = p;
    a.ap = ap;
    a.K64 = h->Ks64;
    a.b64 = h->b64;
    a.x64 = h->x64;
    a.r64 = h->r64;
    a.s = h->scal;
    a.partials = h->partials;
    a.timing = h->timing;
    a.claim = h->claim;
    return a;
}

// The PCG with the persistent cooperative kernel: one launch for the initial preconditioning,
// then launches of `persist_chunk` iterations until the device flags the end.
int32_t run_pcg_persistent(MailleGpuHandle* h, int32_t* iterations, int32_t* updates, double* rel_res) {
    cudaStream_t st = h->st;
    const bool mixed = is_mixed(h);
    auto launch = [&](bool init) {
        if (mixed) {
            auto a = pcg_args<float>(h, h->Ks32, h->Ls32, h->Us32, h->D32, h->x32, h->r32, h->z32, h->p32, h->ap32);
            CK((launch_pcg_persistent<float, true>(a, h->persist_grid, init, st)));
        } else {
            auto a = pcg_args<double>(h, h->Ks64, h->Ls64, h->Us64, h->D64, h->x64, h->r64, h->z64, h->p64, h->ap64);
            CK((launch_pcg_persistent<double, false>(a, h->persist_grid, init, st)));
        }
    };
    CK(cudaMemsetAsync(h->claim, 0, 4 * sizeof(int32_t), st));
    launch(true);
    int32_t status = MAILLE_OK;
    for (;;) {
        launch(false);
        CK(cudaMemcpyAsync(h->h_scal, h->scal, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        const PcgScalars& s = *h->h_scal;
        if (s.done) {
            status = s.status == 1 ? MAILLE_SINGULAR
                   : s.status == 2 ? MAILLE_NOT_CONVERGED
                   : s.status == 3 ? MAILLE_CUDA_ERROR
                                   : MAILLE_OK;
            break;
        }
        if (h->cancel.load()) {
            status = MAILLE_CANCELLED;
            break;
        }
    }
    const PcgScalars& s = *h->h_scal;
    *iterations = s.iter;
    *updates = mixed ? s.updates : 1;
    *rel_res = s.bb > 0 ? std::sqrt((mixed ? s.rr_true : s.rr) / s.bb) : 0.0;
    return status;
}

// PCG on K x = b64 (b64 in padded solver numbering) into x64. Returns the MailleStatus.
int32_t run_pcg(MailleGpuHandle* h, int32_t* iterations, int32_t* updates, double* rel_res) {
    const int64_t n4 = 4 * (int64_t)h->sym.nb;
    cudaStream_t st = h->st;
    const bool mixed = is_mixed(h);
    CK(cudaMemsetAsync(h->x64, 0, n4 * sizeof(double), st));
    CK(cudaMemcpyAsync(h->r64, h->b64, n4 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    launch_norm2<double>(n4, h->b64, h->partials, h->dticket, &h->scal->bb, st);
    launch_pcg_init(h->scal, h->tol, h->max_iter, mixed ? h->delta : 0.0, st);
    if (mixed) {
        for (float* q : {h->x32, h->p32, h->ap32}) CK(cudaMemsetAsync(q, 0, n4 * sizeof(float), st));
        launch_cast(n4, h->b64, h->r32, st);
    } else {
        for (double* q : {h->p64, h->ap64}) CK(cudaMemsetAsync(q, 0, n4 * sizeof(double), st));
    }
    if (h->persist_grid <= 0) throw CudaFailure{"the persistent PCG kernel cannot be made co-resident on this device"};
    return run_pcg_persistent(h, iterations, updates, rel_res);
}

void set_error(const std::string& m) { g_last_error = m; }

int32_t fail(const Error& e) {
    set_error(e.message);
    return e.status;
}

bool check_problem(const MailleElasticProblem* p, Error& err) {
    if (!p) {
        err = {MAILLE_INVALID_INPUT, "null problem"};
        return false;
    }
    if (!p->coords || !p->conn || !p->young || !p->poisson) {
        err = {MAILLE_INVALID_INPUT, "coords, conn, young and poisson are required"};
        return false;
    }
    if (p->precision != MAILLE_FP64 && p->precision != MAILLE_MIXED) {
        err = {MAILLE_INVALID_INPUT, "unknown precision"};
        return false;
    }
    if (p->ordering < MAILLE_ORDER_AUTO || p->ordering > MAILLE_ORDER_MULTICOLOR_ITERATED) {
        err = {MAILLE_INVALID_INPUT, "unknown ordering"};
        return false;
    }
    for (int64_t k = 0; k < 3 * p->n_nodes; ++k)
        if (!std::isfinite(p->coords[k])) {
            err = {MAILLE_INVALID_INPUT, "non-finite coordinate at node " + std::to_string(k / 3)};
            return false;
        }
    for (int64_t e = 0; e < p->n_elems; ++e)
        if (!std::isfinite(p->young[e]) || !std::isfinite(p->poisson[e]) || p->young[e] <= 0.0 ||
            p->poisson[e] <= -1.0 || p->poisson[e] >= 0.5) {
            err = {MAILLE_INVALID_INPUT, "invalid material of element " + std::to_string(e)};
            return false;
        }
    if (p->f)
        for (int64_t k = 0; k < 3 * p->n_nodes; ++k)
            if (!std::isfinite(p->f[k])) {
                err = {MAILLE_INVALID_INPUT, "non-finite load at DOF " + std::to_string(k)};
                return false;
            }
    if (p->imposed && p->fixed)
        for (int64_t k = 0; k < 3 * p->n_nodes; ++k)
            if (p->fixed[k] && !std::isfinite(p->imposed[k])) {
                err = {MAILLE_INVALID_INPUT, "non-finite imposed value at DOF " + std::to_string(k)};
                return false;
            }
    return true;
}

// b64 (padded solver numbering) from the current load vector and K_fc u_c.
void build_rhs(MailleGpuHandle* h) {
    const double* coupling = nullptr;
    if (h->any_imposed) {
        // u_c: imposed values at fixed DOFs, 0 elsewhere; coupling = K u_c on boundary nodes
        CK(cudaMemsetAsync(h->y_full, 0, 3 * h->n_nodes * sizeof(double), h->st));
        launch_elem_apply(h->npe, (int64_t)h->sym.belem.size(), h->belem, h->conn, h->ke,
                          h->imposed, h->ye, h->st);
        launch_node_gather(h->npe, (int64_t)h->sym.bnodes.size(), h->bnodes, h->inc_ptr, h->inc,
                           h->elem_slot, h->ye, h->y_full, h->st);
        coupling = h->y_full;
    }
    launch_build_rhs(h->sym.nb, h->perm, h->fixmask, h->f_cur, coupling, h->b64, h->st);
}

int32_t factorize(MailleGpuHandle* h, Error& err) {
    const Pattern pt = h->pattern();
    for (double shift : kShifts) {
        CK(cudaMemsetAsync(h->dfail, 0, sizeof(int32_t), h->st));
        for (int l = 0; l < h->sym.levels; ++l)
            launch_factor_level(pt, h->sym.level_ptr[l], h->sym.level_ptr[l + 1], h->K, h->F, shift,
                                h->dfail, h->st);
        CK(cudaGetLastError());
        int32_t failed = 0;
        CK(cudaMemcpyAsync(&failed, h->dfail, sizeof(int32_t), cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
        if (!failed) {
            h->shift = shift;
            return MAILLE_OK;
        }
    }
    err = {MAILLE_SINGULAR, "IC(0) failed with every diagonal shift (Singular)"};
    return MAILLE_SINGULAR;
}

// Element integration + scatter-reduce assembly + IC(0), then the sliced copies the
// iterations read (FP64 for the plain form; FP32 K, L, L^T, D and the FP64 K for the mixed one).
int32_t assemble_factor(MailleGpuHandle* h, Error& err);

int32_t numeric_phase(MailleGpuHandle* h, Error& err) {
    ElemIn in{h->n_elems, h->coords, h->conn, h->young, h->poisson};
    launch_elem_stiffness(h->npe, in, h->ke, h->st);
    return assemble_factor(h, err);
}

int32_t assemble_factor(MailleGpuHandle* h, Error& err) {
    const Symbolic& s = h->sym;
    cudaStream_t st = h->st;
    launch_assemble(h->pattern(), s.nl, h->lslot, h->lrow, h->lptr, h->contrib,
                    h->ke, h->K, st);
    launch_sell_fill<double>(h->sk.h.steps(), h->sk.src, h->K, h->Ks64, st);
    CK(cudaGetLastError());
    CK(cudaEventRecord(h->ev[2], st));
    if (factorize(h, err) != MAILLE_OK) return err.status;
    if (is_mixed(h)) {
        launch_sell_fill<float>(h->sk.h.steps(), h->sk.src, h->K, h->Ks32, st);
        launch_sell_fill<float>(h->pl.h.steps(), h->pl.src, h->F, h->Ls32, st);
        launch_sell_fill<float>(h->pu.h.steps(), h->pu.src, h->F, h->Us32, st);
        launch_diag_fill<float>(s.nb, h->diag, h->F, h->D32, st);
    } else {
        launch_sell_fill<double>(h->pl.h.steps(), h->pl.src, h->F, h->Ls64, st);
        launch_sell_fill<double>(h->pu.h.steps(), h->pu.src, h->F, h->Us64, st);
        launch_diag_fill<double>(s.nb, h->diag, h->F, h->D64, st);
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(h->ev[3], st));
    return MAILLE_OK;
}

int env_int(const char* name, int dflt) {
    const char* e = std::getenv(name);
    return e ? std::atoi(e) : dflt;
}

int32_t create_impl(const MailleElasticProblem* p, MailleGpuHandle** out, MailleElasticResult* res) {
    NvtxRange nvtx("maille create: analysis, upload, assembly, IC(0)");
    Error err{MAILLE_OK, ""};
    if (!out) return fail({MAILLE_INVALID_INPUT, "null handle pointer"});
    *out = nullptr;
    if (!check_problem(p, err)) return fail(err);
    auto h = std::make_unique<MailleGpuHandle>();
    h->device = p->device;
    h->npe = p->nodes_per_elem;
    h->n_nodes = p->n_nodes;
    h->n_elems = p->n_elems;
    h->precision = p->precision;
    h->tol = p->rel_tol > 0 ? p->rel_tol : kDefaultTol;
    h->max_iter = p->max_iter > 0 ? p->max_iter : kDefaultMaxIter;
    if (const char* e = std::getenv("MAILLE_RELIABLE_DELTA")) h->delta = std::atof(e);
    const int64_t n3 = 3 * p->n_nodes;
    h->h_fixed.assign(n3, 0);
    if (p->fixed)
        for (int64_t k = 0; k < n3; ++k) h->h_fixed[k] = p->fixed[k] ? 1 : 0;
    // the element kernels index with the connectivity: check it before any device work (a
    // min / max pass; the offending entry is looked for only when there is one)
    if (p->nodes_per_elem != 4 && p->nodes_per_elem != 10)
        return fail({MAILLE_INVALID_INPUT, "nodes_per_elem must be 4 or 10"});
    {
        const int64_t nc = p->n_elems * p->nodes_per_elem;
        int64_t lo = INT64_MAX, hi = INT64_MIN;
        for (int64_t k = 0; k < nc; ++k) {
            lo = std::min(lo, p->conn[k]);
            hi = std::max(hi, p->conn[k]);
        }
        if (nc > 0 && (lo < 0 || hi >= p->n_nodes))
            for (int64_t k = 0; k < nc; ++k)
                if (p->conn[k] < 0 || p->conn[k] >= p->n_nodes)
                    return fail({MAILLE_INVALID_INPUT, "element " + std::to_string(k / p->nodes_per_elem) +
                                                           " refers to unknown node " + std::to_string(p->conn[k])});
    }
    if (std::all_of(h->h_fixed.begin(), h->h_fixed.end(), [](uint8_t f) { return f != 0; }))
        return fail({MAILLE_INVALID_INPUT, "every DOF is fixed"});
    if (p->n_nodes >= (int64_t(1) << 30) || p->n_elems * node_pairs(p->nodes_per_elem) >= (int64_t(1) << 31))
        return fail({MAILLE_INVALID_INPUT, "mesh too large for 32-bit node and element-pair indices"});
    // The ordering and the node incidence run on the device (ordering.cu) once the inputs are
    // there; the host keeps the part that does not depend on them (kept nodes, boundary lists, the
    // host copies of the loads and the imposed-value flag) on a thread of its own meanwhile.
    // MAILLE_HOST_ORDERING=1 orders on that host thread instead (the same permutation: the same
    // algorithms on the same graph). The pattern and scatter map follow on the device
    // (analysis.cu).
    const bool host_ordering = env_int("MAILLE_HOST_ORDERING", 0) != 0;
    // AUTO: MULTICOLOR_ITERATED (Tet10 40^3 mixed: 15 levels against 18, 1.6 % more iterations,
    // the step 4 % shorter than MULTICOLOR)
    const int ordering = p->ordering == MAILLE_ORDER_AUTO ? MAILLE_ORDER_MULTICOLOR_ITERATED : p->ordering;
    std::vector<int32_t> kept, kept_of;
    const double t_setup0 = now_ms();
    double t_setup1 = t_setup0;
    bool analysed = false;
    std::thread analysis([&] {
        if (host_ordering)
            analysed = analyse(p->n_nodes, p->nodes_per_elem, p->n_elems, p->conn, h->h_fixed.data(), ordering,
                               h->sym, err, /*pattern=*/false);
        else
            analysed = analyse_topology(p->n_nodes, p->nodes_per_elem, p->n_elems, p->conn, h->h_fixed.data(),
                                        h->sym, kept, kept_of, err, /*boundary_lists=*/true,
                                        /*incidence=*/false);
        if (p->imposed)
            for (int64_t k = 0; k < n3; ++k)
                if (h->h_fixed[k] && p->imposed[k] != 0.0) {
                    h->any_imposed = true;
                    break;
                }
        h->h_f.assign(n3, 0.0);
        if (p->f) std::memcpy(h->h_f.data(), p->f, n3 * sizeof(double));
        h->h_f0 = h->h_f;
        t_setup1 = now_ms();
    });
    struct Joiner {
        std::thread& t;
        ~Joiner() {
            if (t.joinable()) t.join();
        }
    } joiner{analysis};
    // MAILLE_SETUP_TIMING: wall time of the device-side set-up steps (stream synchronised)
    const bool stage_timing = std::getenv("MAILLE_SETUP_TIMING") != nullptr;
    double t_mark = now_ms();
    auto tmark = [&](const char* name) {
        if (!stage_timing) return;
        if (h->st) cudaStreamSynchronize(h->st);
        const double t = now_ms();
        std::fprintf(stderr, "maille create %-14s %8.1f ms\n", name, t - t_mark);
        t_mark = t;
    };
    try {
        int ndev = 0;
        CK(cudaGetDeviceCount(&ndev));
        if (p->device < 0 || p->device >= ndev)
            return fail({MAILLE_CUDA_ERROR, "no CUDA device " + std::to_string(p->device)});
        CK(cudaSetDevice(p->device));
        CK(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
        for (auto& e : h->ev) CK(cudaEventCreate(&e));
        cudaStream_t st = h->st;
        const Symbolic& s = h->sym;
        CK(cudaEventRecord(h->ev[0], st));
        tmark("context");
        const int np = node_pairs(h->npe);
        // inputs, straight from the caller's buffers: the connectivity is narrowed to 32 bits and
        // the imposed values kept at fixed DOFs only on the device
        const int64_t nconn = p->n_elems * p->nodes_per_elem;
        struct DevTemp {
            void* p = nullptr;
            ~DevTemp() { dfree(p); }
        } conn64;
        conn64.p = dupload(p->conn, nconn, st);
        h->coords = dupload(p->coords, n3, st);
        h->conn = dalloc<int32_t>(nconn);
        gpu_narrow(static_cast<const int64_t*>(conn64.p), nconn, h->conn, st);
        h->young = dupload(p->young, p->n_elems, st);
        h->poisson = dupload(p->poisson, p->n_elems, st);
        h->fixed = dupload(h->h_fixed.data(), n3, st);
        h->imposed = dupload(p->imposed, n3, st);
        if (p->imposed)
            gpu_zero_free(n3, h->fixed, h->imposed, st);
        else
            CK(cudaMemsetAsync(h->imposed, 0, n3 * sizeof(double), st));
        h->f0 = dupload(p->f, n3, st);
        if (!p->f) CK(cudaMemsetAsync(h->f0, 0, n3 * sizeof(double), st));
        h->f = dalloc<double>(n3);
        h->f_cur = h->f0;
        h->inc_ptr = dalloc<int64_t>(p->n_nodes + 1);
        h->inc = dalloc<int32_t>(nconn);
        h->ke = dalloc<double>((size_t)p->n_elems * np * 9);
        CK(cudaEventRecord(h->ev[8], st));  // inputs copied
        {
            ElemIn in{h->n_elems, h->coords, h->conn, h->young, h->poisson};
            launch_elem_stiffness(h->npe, in, h->ke, st);
        }
        CK(cudaEventRecord(h->ev[9], st));  // element matrices integrated
        const double t_wait0 = now_ms();
        gpu_incidence(h->conn, nconn, p->n_nodes, st, h->inc_ptr, h->inc);
        if (host_ordering) {
            analysis.join();
            if (!analysed) return fail(err);
        } else {
            // kept nodes: at least one free DOF (the same rule as analyse_topology)
            std::vector<int32_t> h_kept_of(p->n_nodes, -1), h_kept;
            for (int64_t v = 0; v < p->n_nodes; ++v)
                if (!(h->h_fixed[3 * v] && h->h_fixed[3 * v + 1] && h->h_fixed[3 * v + 2])) {
                    h_kept_of[v] = (int32_t)h_kept.size();
                    h_kept.push_back((int32_t)v);
                }
            int32_t* d_kept_of = dupload(h_kept_of.data(), h_kept_of.size(), st);
            std::vector<int32_t> order, level;
            try {
                gpu_ordering(h->npe, h->n_elems, h->conn, d_kept_of, (int32_t)h_kept.size(), ordering, st, order,
                             level);
            } catch (...) {
                dfree(d_kept_of);
                throw;
            }
            dfree(d_kept_of);
            analysis.join();
            if (!analysed) return fail(err);
            apply_ordering(h_kept, order, level, h->h_fixed.data(), h->sym);
        }
        const double t_wait1 = now_ms();
        CK(cudaEventRecord(h->ev[10], st));  // symbolic: the ordering is known
        if (h->sym.levels >= kMaxLevels) return fail({MAILLE_INVALID_INPUT, "too many IC(0) levels"});
        // symbolic
        h->perm = dupload(s.perm.data(), s.perm.size(), st);
        h->inv = dupload(s.inv.data(), s.inv.size(), st);
        h->fixmask = dupload(s.fixmask.data(), s.fixmask.size(), st);
        tmark("inputs");
        {
            PatternDev pt;
            gpu_pattern(h->npe, h->n_elems, h->conn, h->inv, s.nb, st, pt, h->sym.row_ptr, h->sym.diag);
            h->row_ptr = pt.row_ptr;
            h->col = pt.col;
            h->diag = pt.diag;
            h->tpos = pt.tpos;
            h->lslot = pt.lslot;
            h->lrow = pt.lrow;
            h->lptr = pt.lptr;
            h->contrib = pt.contrib;
            h->sym.blocks = pt.blocks;
            h->sym.nl = pt.nl;
            tmark("pattern");
            // layout plans from the row lengths (host, side by side), slot fills on the device
            const int lk = env_int("MAILLE_LPR_K", 0);
            std::thread tk([&] { build_sell(h->sym, SELL_FULL, lk, h->sk.h); });
            std::thread tl([&] { build_psell(h->sym, SELL_LOWER, h->pl.h); });
            build_psell(h->sym, SELL_UPPER, h->pu.h);
            tk.join();
            tl.join();
            h->pl.kind = SELL_LOWER;
            h->pu.kind = SELL_UPPER;
            tmark("layout plans");
            h->sk.upload(pt, s.nb, st);
            h->pl.upload(pt, s.nb, st);
            h->pu.upload(pt, s.nb, st);
        }
        CK(cudaEventRecord(h->ev[11], st));  // pattern and layouts on the device
        h->belem = dupload(s.belem.data(), s.belem.size(), st);
        h->bnodes = dupload(s.bnodes.data(), s.bnodes.size(), st);
        std::vector<int32_t> slot(p->n_elems, -1);
        for (size_t k = 0; k < s.belem.size(); ++k) slot[s.belem[k]] = (int32_t)k;
        h->elem_slot = dupload(slot.data(), slot.size(), st);
        // numeric buffers
        const int64_t n4 = 4 * ((int64_t)s.nb + 1);  // + the dummy node that padding points at
        h->K = dalloc<double>((size_t)s.blocks * 9);
        h->F = dalloc<double>((size_t)s.blocks * 9);
        h->Ks64 = dalloc<double>((size_t)h->sk.h.steps() * 9 * kStepSlots);
        for (double** q : {&h->b64, &h->x64, &h->r64, &h->p64, &h->ap64}) {
            *q = dalloc<double>(n4);
            CK(cudaMemsetAsync(*q, 0, n4 * sizeof(double), st));
        }
        if (is_mixed(h.get())) {
            h->Ks32 = dalloc<float>((size_t)h->sk.h.steps() * 9 * kStepSlots);
            h->Ls32 = dalloc<float>((size_t)h->pl.h.steps() * 9 * kStepSlots);
            h->Us32 = dalloc<float>((size_t)h->pu.h.steps() * 9 * kStepSlots);
            h->D32 = dalloc<float>((size_t)s.nb * 9);
            for (float** q : {&h->x32, &h->r32, &h->z32, &h->p32, &h->ap32}) {
                *q = dalloc<float>(n4);
                CK(cudaMemsetAsync(*q, 0, n4 * sizeof(float), st));
            }
            // the dummy node's sweep record is always ready (tag = the largest epoch)
            static const unsigned int kAlwaysReady = 0xFFFFFFFFu;
            CK(cudaMemcpyAsync(h->z32 + 4 * (int64_t)s.nb + 3, &kAlwaysReady, sizeof(unsigned int),
                               cudaMemcpyHostToDevice, st));
        } else {
            h->Ls64 = dalloc<double>((size_t)h->pl.h.steps() * 9 * kStepSlots);
            h->Us64 = dalloc<double>((size_t)h->pu.h.steps() * 9 * kStepSlots);
            h->D64 = dalloc<double>((size_t)s.nb * 9);
            // sweep records (z0, z1, z2, tag); the dummy node's tag is the largest epoch
            h->z64 = dalloc<double>(n4);
            CK(cudaMemsetAsync(h->z64, 0, n4 * sizeof(double), st));
            static const unsigned long long kAlwaysReady64 = ~0ull;
            CK(cudaMemcpyAsync(h->z64 + 4 * (int64_t)s.nb + 3, &kAlwaysReady64, sizeof(kAlwaysReady64),
                               cudaMemcpyHostToDevice, st));
        }
        h->u_full = dalloc<double>(n3);
        h->y_full = dalloc<double>(n3);
        h->react = dalloc<double>(n3);
        h->ye = dalloc<double>(std::max<size_t>(1, s.belem.size()) * 3 * h->npe);
        h->scal = dalloc<PcgScalars>(1);
        CK(cudaMemsetAsync(h->scal, 0, sizeof(PcgScalars), st));
        h->h_scal = static_cast<PcgScalars*>(pinned_slot_alloc(sizeof(PcgScalars)));
        h->h_sum = static_cast<double*>(pinned_slot_alloc(4 * sizeof(double)));
        h->dsum = dalloc<double>(4);
        h->dticket = dalloc<unsigned int>(1);
        CK(cudaMemsetAsync(h->dticket, 0, sizeof(unsigned int), st));
        h->dfail = dalloc<int32_t>(1);
        h->spmv_grid = grid_for_slices(h->sk.h.nslices());
        h->claim = dalloc<int32_t>(4);
        CK(cudaMemsetAsync(h->claim, 0, 4 * sizeof(int32_t), st));
        h->persist_grid = is_mixed(h.get()) ? pcg_persistent_grid<float, true>(h->sk.h.lpr)
                                            : pcg_persistent_grid<double, false>(h->sk.h.lpr);
        // 4 reduction slots for every block of the persistent grid and of the norm kernels
        // (grids capped at 8 and 4 blocks per SM)
        h->persist_grid = std::min(h->persist_grid, 8 * device_sms());
        // small systems: a grid sized to the work (one block of 8 warps per 8 slices of K, at
        // least half the SMs), so that each of the iteration's grid barriers spans fewer blocks
        // (the large-strain block, 587 slices: 74 blocks, 8 % faster than 296)
        h->persist_grid = std::min<int64_t>(
            h->persist_grid, std::max<int64_t>(device_sms() / 2, (h->sk.h.nslices() + 7) / 8));
        // MAILLE_PERSIST_GRID: fewer co-resident blocks than the occupancy allows (a tuning and
        // measurement knob: the phases' time against the warps in flight and the barrier cost)
        if (const int blocks = env_int("MAILLE_PERSIST_GRID", 0); blocks > 0)
            h->persist_grid = std::min(h->persist_grid, blocks);
        h->partials = dalloc<double>((size_t)4 * 8 * device_sms());
        if (env_int("MAILLE_PHASE_TIMING", 0)) {
            h->timing = dalloc<unsigned long long>(8);
            CK(cudaMemsetAsync(h->timing, 0, 8 * sizeof(unsigned long long), st));
        }
        h->persist_chunk = std::max(1, env_int("MAILLE_PERSIST_CHUNK", h->persist_chunk));
        tmark("layouts+buffers");
        CK(cudaEventRecord(h->ev[1], st));
        if (assemble_factor(h.get(), err) != MAILLE_OK) return fail(err);
        tmark("numeric");
        CK(cudaStreamSynchronize(st));
        if (res) {
            res->ms_setup = t_setup1 - t_setup0;
            res->ms_upload = elapsed(h->ev[0], h->ev[8]);
            res->ms_element = elapsed(h->ev[8], h->ev[9]);
            res->ms_ordering = t_wait1 - t_wait0;
            res->ms_symbolic = elapsed(h->ev[10], h->ev[11]);
            res->ms_buffers = elapsed(h->ev[11], h->ev[1]);
            res->ms_assembly = elapsed(h->ev[1], h->ev[2]);
            res->ms_factor = elapsed(h->ev[2], h->ev[3]);
        }
    } catch (const CudaFailure& e) {
        return fail({MAILLE_CUDA_ERROR, e.what});
    }
    *out = h.release();
    return MAILLE_OK;
}

const char* status_message(int32_t status, int32_t iters, double rel) {
    static thread_local std::string m;
    if (status == MAILLE_SINGULAR) m = "Singular: IC(0)-PCG met p.Ap <= 0 or NaN";
    else if (status == MAILLE_NOT_CONVERGED)
        m = "IterativeNotConverged: iterations " + std::to_string(iters) + ", relative residual " +
            std::to_string(rel);
    else if (status == MAILLE_CANCELLED) m = "Cancelled";
    else m = "";
    return m.c_str();
}

int32_t solve_impl(MailleGpuHandle* h, const double* f, MailleElasticResult* res) {
    NvtxRange nvtx("maille solve: PCG, reactions, stresses");
    if (!h) return fail({MAILLE_INVALID_INPUT, "null handle"});
    try {
        CK(cudaSetDevice(h->device));
        cudaStream_t st = h->st;
        const Symbolic& s = h->sym;
        const int64_t n3 = 3 * h->n_nodes;
        if (f) {
            for (int64_t k = 0; k < n3; ++k)
                if (!std::isfinite(f[k])) return fail({MAILLE_INVALID_INPUT, "non-finite load"});
            std::memcpy(h->h_f.data(), f, n3 * sizeof(double));
            CK(cudaMemcpyAsync(h->f, f, n3 * sizeof(double), cudaMemcpyHostToDevice, st));
            h->f_cur = h->f;
        } else {
            h->h_f = h->h_f0;
            h->f_cur = h->f0;
        }
        CK(cudaEventRecord(h->ev[4], st));
        build_rhs(h);
        int32_t iters = 0, outer = 1;
        double rel = 0.0;
        const int32_t status = run_pcg(h, &iters, &outer, &rel);
        CK(cudaEventRecord(h->ev[5], st));
        if (res) {
            res->iterations = iters;
            res->outer_iterations = outer;
            res->final_rel_residual = rel;
            res->shift = h->shift;
            res->free_dofs = s.free_dofs;
            res->block_rows = s.nb;
            res->blocks = s.blocks;
            res->levels = s.levels;
        }
        if (status != MAILLE_OK) {
            CK(cudaStreamSynchronize(st));
            set_error(status_message(status, iters, rel));
            return status;
        }
        // u in caller numbering, reactions, stresses
        launch_gather_u(h->n_nodes, h->inv, h->fixed, h->imposed, h->x64, h->u_full, st);
        CK(cudaMemsetAsync(h->react, 0, n3 * sizeof(double), st));
        if (!s.belem.empty()) {
            CK(cudaMemsetAsync(h->y_full, 0, n3 * sizeof(double), st));
            launch_elem_apply(h->npe, (int64_t)s.belem.size(), h->belem, h->conn, h->ke, h->u_full,
                              h->ye, st);
            launch_node_gather(h->npe, (int64_t)s.bnodes.size(), h->bnodes, h->inc_ptr, h->inc,
                               h->elem_slot, h->ye, h->y_full, st);
            launch_reactions(h->n_nodes, h->bnodes, (int64_t)s.bnodes.size(), h->fixed, h->y_full,
                             h->f_cur, h->react, st);
        }
        const int ng = gauss_points(h->npe);
        if (!h->gauss) {
            h->gauss = dalloc<double>((size_t)h->n_elems * ng * 9);
            h->vm = dalloc<double>((size_t)h->n_elems * ng);
        }
        ElemIn in{h->n_elems, h->coords, h->conn, h->young, h->poisson};
        launch_stresses(h->npe, in, h->u_full, h->gauss, h->vm, st);
        CK(cudaGetLastError());
        CK(cudaEventRecord(h->ev[6], st));
        if (res) {
            if (res->u) CK(cudaMemcpyAsync(res->u, h->u_full, n3 * sizeof(double), cudaMemcpyDeviceToHost, st));
            if (res->reactions)
                CK(cudaMemcpyAsync(res->reactions, h->react, n3 * sizeof(double), cudaMemcpyDeviceToHost, st));
            if (res->gauss_stress)
                CK(cudaMemcpyAsync(res->gauss_stress, h->gauss, (size_t)h->n_elems * ng * 9 * sizeof(double),
                                   cudaMemcpyDeviceToHost, st));
            if (res->von_mises)
                CK(cudaMemcpyAsync(res->von_mises, h->vm, (size_t)h->n_elems * ng * sizeof(double),
                                   cudaMemcpyDeviceToHost, st));
        }
        CK(cudaEventRecord(h->ev[7], st));
        CK(cudaStreamSynchronize(st));
        if (res) {
            res->ms_solve = elapsed(h->ev[4], h->ev[5]);
            res->ms_post = elapsed(h->ev[5], h->ev[6]);
            res->ms_download = elapsed(h->ev[6], h->ev[7]);
            // a fixed DOF that no element touches: K u = 0 there (product skips it)
            if (res->reactions && s.belem.size() < (size_t)h->n_elems) {
                for (int64_t v = 0; v < h->n_nodes; ++v)
                    if (s.inc_ptr[v] == s.inc_ptr[v + 1])
                        for (int c = 0; c < 3; ++c)
                            if (h->h_fixed[3 * v + c]) res->reactions[3 * v + c] = -h->h_f[3 * v + c];
            }
        }
        h->solved = true;
    } catch (const CudaFailure& e) {
        return fail({MAILLE_CUDA_ERROR, e.what});
    }
    return MAILLE_OK;
}

// FreeSystem::solve with device-resident loads and displacements: no reactions, stresses or host
// copies (the chained-solve form of solve_impl).
int32_t solve_device_impl(MailleGpuHandle* h, const double* f_dev, double* u_dev) {
    NvtxRange nvtx("maille solve (device buffers)");
    if (!h || !u_dev) return fail({MAILLE_INVALID_INPUT, "null handle or displacement buffer"});
    try {
        CK(cudaSetDevice(h->device));
        cudaStream_t st = h->st;
        const int64_t n3 = 3 * h->n_nodes;
        if (f_dev) {
            CK(cudaMemcpyAsync(h->f, f_dev, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
            h->f_cur = h->f;
        } else {
            h->h_f = h->h_f0;
            h->f_cur = h->f0;
        }
        build_rhs(h);
        int32_t iters = 0, outer = 1;
        double rel = 0.0;
        const int32_t status = run_pcg(h, &iters, &outer, &rel);
        if (status != MAILLE_OK) {
            CK(cudaStreamSynchronize(st));
            set_error(status_message(status, iters, rel));
            return status;
        }
        launch_gather_u(h->n_nodes, h->inv, h->fixed, h->imposed, h->x64, h->u_full, st);
        CK(cudaMemcpyAsync(u_dev, h->u_full, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CK(cudaStreamSynchronize(st));
        h->solved = true;
    } catch (const CudaFailure& e) {
        return fail({MAILLE_CUDA_ERROR, e.what});
    }
    return MAILLE_OK;
}

int32_t backward_impl(MailleGpuHandle* h, const double* dJdu, double* dJdE, double* lambda) {
    if (!h || !dJdu || !dJdE) return fail({MAILLE_INVALID_INPUT, "null argument"});
    if (!h->solved) return fail({MAILLE_INVALID_INPUT, "backward needs a solve first"});
    try {
        CK(cudaSetDevice(h->device));
        cudaStream_t st = h->st;
        const int64_t n3 = 3 * h->n_nodes;
        for (int64_t k = 0; k < n3; ++k)
            if (!std::isfinite(dJdu[k])) return fail({MAILLE_INVALID_INPUT, "non-finite dJ/du"});
        // adjoint right-hand side g at free DOFs; lambda = 0 at fixed DOFs (no coupling term)
        CK(cudaMemcpyAsync(h->y_full, dJdu, n3 * sizeof(double), cudaMemcpyHostToDevice, st));
        launch_build_rhs(h->sym.nb, h->perm, h->fixmask, h->y_full, nullptr, h->b64, st);
        if (!h->lambda_full) {
            h->lambda_full = dalloc<double>(n3);
            h->grad = dalloc<double>(h->n_elems);
        }
        // K is symmetric: the same PCG and factor solve K lambda = g (u stays in u_full)
        int32_t iters = 0, outer = 0;
        double rel = 0.0;
        const int32_t status = run_pcg(h, &iters, &outer, &rel);
        if (status != MAILLE_OK) {
            CK(cudaStreamSynchronize(st));
            set_error(std::string("adjoint solve: ") + status_message(status, iters, rel));
            return status;
        }
        CK(cudaMemsetAsync(h->y_full, 0, n3 * sizeof(double), st));
        launch_gather_u(h->n_nodes, h->inv, h->fixed, h->y_full, h->x64, h->lambda_full, st);
        launch_adjoint_grad(h->npe, h->n_elems, h->conn, h->ke, h->young, h->lambda_full, h->u_full,
                            h->grad, st);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(dJdE, h->grad, h->n_elems * sizeof(double), cudaMemcpyDeviceToHost, st));
        if (lambda)
            CK(cudaMemcpyAsync(lambda, h->lambda_full, n3 * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    } catch (const CudaFailure& e) {
        return fail({MAILLE_CUDA_ERROR, e.what});
    }
    return MAILLE_OK;
}

}  // namespace

namespace maille {
void set_last_error(const std::string& message) { g_last_error = message; }
int32_t handle_create(const MailleElasticProblem* p, MailleGpuHandle** out, MailleElasticResult* res) {
    return create_impl(p, out, res);
}
int32_t handle_assemble_factor(MailleGpuHandle* h, Error& err) { return assemble_factor(h, err); }
void handle_build_rhs(MailleGpuHandle* h) { build_rhs(h); }
int32_t handle_run_pcg(MailleGpuHandle* h, int32_t* iterations, int32_t* updates, double* rel_res) {
    return run_pcg(h, iterations, updates, rel_res);
}
const char* handle_status_message(int32_t status, int32_t iters, double rel) {
    return status_message(status, iters, rel);
}
}  // namespace maille

// ---- C ABI -------------------------------------------------------------------------------------

extern "C" {

const char* maille_gpu_last_error(void) { return g_last_error.c_str(); }

const char* maille_gpu_version(void) { return "maille-b200 0.1.0 (sm_100a)"; }

int32_t maille_gpu_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int32_t maille_gpu_create(const MailleElasticProblem* problem, MailleGpuHandle** out) {
    g_last_error.clear();
    return create_impl(problem, out, nullptr);
}

int32_t maille_gpu_solve(MailleGpuHandle* h, const double* f, MailleElasticResult* result) {
    g_last_error.clear();
    return solve_impl(h, f, result);
}

int32_t maille_gpu_solve_device(MailleGpuHandle* h, const double* f_dev, double* u_dev) {
    g_last_error.clear();
    return solve_device_impl(h, f_dev, u_dev);
}

int32_t maille_gpu_backward(MailleGpuHandle* h, const double* dJdu, double* dJdE, double* lambda) {
    g_last_error.clear();
    return backward_impl(h, dJdu, dJdE, lambda);
}

void maille_gpu_cancel(MailleGpuHandle* h, int32_t flag) {
    if (h) h->cancel.store(flag ? 1 : 0);
}

void* maille_gpu_stream(MailleGpuHandle* h) { return h ? (void*)h->st : nullptr; }

void maille_gpu_destroy(MailleGpuHandle* h) { delete h; }

int32_t maille_gpu_elastic_solve(const MailleElasticProblem* problem, MailleElasticResult* result) {
    g_last_error.clear();
    MailleGpuHandle* h = nullptr;
    const bool timing = std::getenv("MAILLE_SETUP_TIMING") != nullptr;
    const double t0 = now_ms();
    int32_t s = create_impl(problem, &h, result);
    if (s != MAILLE_OK) return s;
    const double t1 = now_ms();
    s = solve_impl(h, nullptr, result);
    const double t2 = now_ms();
    delete h;
    if (timing)
        std::fprintf(stderr, "maille one-shot: create %.1f ms, solve %.1f ms, destroy %.1f ms\n", t1 - t0,
                     t2 - t1, now_ms() - t2);
    return s;
}

int32_t maille_gpu_refactor(MailleGpuHandle* h, const double* young, const double* poisson) {
    g_last_error.clear();
    if (!h) return fail({MAILLE_INVALID_INPUT, "null handle"});
    for (int64_t e = 0; e < h->n_elems; ++e) {
        const double E = young ? young[e] : 1.0, nu = poisson ? poisson[e] : 0.0;
        if (!std::isfinite(E) || !std::isfinite(nu) || E <= 0.0 || nu <= -1.0 || nu >= 0.5)
            return fail({MAILLE_INVALID_INPUT, "invalid material of element " + std::to_string(e)});
    }
    try {
        CK(cudaSetDevice(h->device));
        if (young)
            CK(cudaMemcpyAsync(h->young, young, h->n_elems * sizeof(double), cudaMemcpyHostToDevice, h->st));
        if (poisson)
            CK(cudaMemcpyAsync(h->poisson, poisson, h->n_elems * sizeof(double), cudaMemcpyHostToDevice, h->st));
        Error err{MAILLE_OK, ""};
        if (numeric_phase(h, err) != MAILLE_OK) return fail(err);
        h->solved = false;
    } catch (const CudaFailure& e) {
        return fail({MAILLE_CUDA_ERROR, e.what});
    }
    return MAILLE_OK;
}

int32_t maille_gpu_spmv_device(MailleGpuHandle* h, int32_t precision, int32_t count) {
    g_last_error.clear();
    if (!h || count < 0) return fail({MAILLE_INVALID_INPUT, "null handle or negative count"});
    if (precision == MAILLE_MIXED && !h->Ks32)
        return fail({MAILLE_INVALID_INPUT, "the handle holds no FP32 matrix"});
    try {
        CK(cudaSetDevice(h->device));
        for (int32_t k = 0; k < count; ++k) {
            if (precision == MAILLE_MIXED)
                launch_spmv<float>(h->sk.dev(), h->Ks32, h->p32, h->ap32, h->spmv_grid, h->st);
            else
                launch_spmv<double>(h->sk.dev(), h->Ks64, h->p64, h->ap64, h->spmv_grid, h->st);
        }
        CK(cudaGetLastError());
    } catch (const CudaFailure& e) {
        return fail({MAILLE_CUDA_ERROR, e.what});
    }
    return MAILLE_OK;
}

int32_t maille_gpu_multiply(MailleGpuHandle* h, const double* x, double* y) {
    g_last_error.clear();
    if (!h || !x || !y) return fail({MAILLE_INVALID_INPUT, "null argument"});
    try {
        CK(cudaSetDevice(h->device));
        const int64_t n3 = 3 * h->n_nodes;
        CK(cudaMemcpyAsync(h->y_full, x, n3 * sizeof(double), cudaMemcpyHostToDevice, h->st));
        launch_build_rhs(h->sym.nb, h->perm, h->fixmask, h->y_full, nullptr, h->p64, h->st);
        launch_spmv<double>(h->sk.dev(), h->Ks64, h->p64, h->ap64, h->spmv_grid, h->st);
        CK(cudaMemsetAsync(h->react, 0, n3 * sizeof(double), h->st));
        launch_gather_u(h->n_nodes, h->inv, h->fixed, h->react, h->ap64, h->y_full, h->st);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(y, h->y_full, n3 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
        h->solved = false;
    } catch (const CudaFailure& e) {
        return fail({MAILLE_CUDA_ERROR, e.what});
    }
    return MAILLE_OK;
}

int32_t maille_gpu_nodal_stresses(MailleGpuHandle* h, double* stress, double* von_mises) {
    g_last_error.clear();
    if (!h || !stress || !von_mises) return fail({MAILLE_INVALID_INPUT, "null argument"});
    if (!h->solved || !h->gauss)
        return fail({MAILLE_INVALID_INPUT, "nodal stresses need the Gauss stresses of a solve"});
    try {
        CK(cudaSetDevice(h->device));
        if (!h->node_stress) {
            h->node_stress = dalloc<double>((size_t)h->n_nodes * 6);
            h->node_vm = dalloc<double>((size_t)h->n_nodes);
        }
        launch_nodal_stresses(h->npe, h->n_nodes, h->inc_ptr, h->inc, h->gauss, h->node_stress,
                              h->node_vm, h->st);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(stress, h->node_stress, (size_t)h->n_nodes * 6 * sizeof(double),
                           cudaMemcpyDeviceToHost, h->st));
        CK(cudaMemcpyAsync(von_mises, h->node_vm, (size_t)h->n_nodes * sizeof(double),
                           cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
    } catch (const CudaFailure& e) {
        return fail({MAILLE_CUDA_ERROR, e.what});
    }
    return MAILLE_OK;
}

int32_t maille_gpu_wait_selftest(int32_t device, int32_t stale, int32_t* timed_out) {
    g_last_error.clear();
    if (!timed_out) return fail({MAILLE_INVALID_INPUT, "null argument"});
    try {
        CK(cudaSetDevice(device));
        const unsigned int epoch = 7;
        const unsigned int tags[4] = {epoch, epoch, stale ? epoch - 1 : epoch, epoch + 1};
        wait_selftest(tags, epoch, 4096, timed_out);
    } catch (const CudaFailure& e) {
        return fail({MAILLE_CUDA_ERROR, e.what});
    }
    return MAILLE_OK;
}

int32_t maille_gpu_trim_memory(int32_t device) {
    g_last_error.clear();
    if (trim_device_memory(device) != 0) return fail({MAILLE_CUDA_ERROR, "cannot trim the memory pool of device " + std::to_string(device)});
    return MAILLE_OK;
}

int64_t maille_gpu_kernel_launches(void) { return (int64_t)g_kernel_launches.load(); }

int32_t maille_gpu_face_pressure_loads(int64_t n_nodes, const double* coords, int32_t npe,
                                       int64_t n_elems, const int64_t* conn, int64_t n_press,
                                       const int64_t* p_elem, const int32_t* p_face,
                                       const double* p_value, double* f) {
    g_last_error.clear();
    Error err{MAILLE_OK, ""};
    if (!coords || !conn || !f || (n_press > 0 && (!p_elem || !p_face || !p_value)))
        return fail({MAILLE_INVALID_INPUT, "null argument"});
    if (!face_pressure_loads(n_nodes, coords, npe, n_elems, conn, n_press, p_elem, p_face, p_value,
                             f, err))
        return fail(err);
    return MAILLE_OK;
}

}  // extern "C"
