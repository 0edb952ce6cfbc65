// handle.hpp -- the single-model solve handle (maille_gpu_create ... maille_gpu_destroy) and the
// pipeline steps other drivers in this library reuse (the large-strain Newton driver).
#pragma once

#include <atomic>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "analysis.cuh"
#include "common.hpp"
#include "cuda_host.hpp"
#include "kernels.cuh"
#include "sparse.cuh"

// the handle types live at global scope (the C ABI names them); their members are library types
using namespace maille;

// A sliced layout: host plan (level slices) plus its device index arrays; the slot columns and
// CSR sources are filled on the device from the plan and the device pattern.
struct SellBuf {
    SellHost h;
    int32_t* rowid = nullptr;
    int64_t* off = nullptr;
    int32_t* col = nullptr;
    int32_t* src = nullptr;
    int32_t pad = 0;  // the dummy node nb that padding slots point at
    SellDev dev() const { return SellDev{h.lpr, h.nslices(), rowid, off, col, pad}; }
    void upload(const PatternDev& pt, int32_t nb, cudaStream_t st) {
        pad = nb;
        rowid = dupload(h.rowid.data(), h.rowid.size(), st);
        off = dupload(h.off.data(), h.off.size(), st);
        col = dalloc<int32_t>((size_t)h.steps() * 128);
        src = dalloc<int32_t>((size_t)h.steps() * 128);
        fill_sell(SELL_FULL, h.lpr, h.nslices(), h.steps(), rowid, off, pt.row_ptr, pt.col, pt.diag,
                  nb, col, src, st);
    }
    // hands the device buffers to `out` (freed together by the caller) and forgets them
    void gather(std::vector<void*>& out) {
        for (void* p : {(void*)rowid, (void*)off, (void*)col, (void*)src}) out.push_back(p);
        rowid = nullptr;
        off = nullptr;
        col = nullptr;
        src = nullptr;
    }
    void release() {
        for (void* p : {(void*)rowid, (void*)off, (void*)col, (void*)src}) dfree(p);
        rowid = nullptr;
        off = nullptr;
        col = nullptr;
        src = nullptr;
    }
};

// A packed layout of a factor triangle: host description plus its device arrays.
struct PsellBuf {
    PsellHost h;
    SellKind kind = SELL_LOWER;
    int64_t* off = nullptr;
    int32_t* col = nullptr;
    int32_t* src = nullptr;
    uint32_t* head = nullptr;
    int32_t* row0 = nullptr;
    int32_t* rows = nullptr;
    PsellDev dev() const {
        return PsellDev{h.nslices(), off, col, reinterpret_cast<const uint4*>(head), row0, rows, pad};
    }
    int32_t pad = 0;  // the dummy node nb that padding slots point at
    void upload(const PatternDev& pt, int32_t nb, cudaStream_t st) {
        pad = nb;
        off = dupload(h.off.data(), h.off.size(), st);
        head = dupload(h.head.data(), h.head.size(), st);
        row0 = dupload(h.row0.data(), h.row0.size(), st);
        rows = dupload(h.rows.data(), h.rows.size(), st);
        int64_t* rstart = dupload(h.rstart.data(), h.rstart.size(), st);
        col = dalloc<int32_t>((size_t)h.steps() * 128);
        src = dalloc<int32_t>((size_t)h.steps() * 128);
        fill_psell(kind, (int64_t)h.rows.size(), h.steps(), rows, rstart, pt.row_ptr, pt.col, pt.diag,
                   nb, col, src, st);
        CK(cudaStreamSynchronize(st));
        dfree(rstart);
    }
    void gather(std::vector<void*>& out) {
        for (void* p : {(void*)off, (void*)col, (void*)src, (void*)head, (void*)row0, (void*)rows}) out.push_back(p);
        off = nullptr;
        col = nullptr;
        src = nullptr;
        head = nullptr;
        row0 = nullptr;
        rows = nullptr;
    }
    void release() {
        for (void* p : {(void*)off, (void*)col, (void*)src, (void*)head, (void*)row0, (void*)rows}) dfree(p);
        off = nullptr;
        col = nullptr;
        src = nullptr;
        head = nullptr;
        row0 = nullptr;
        rows = nullptr;
    }
};

struct MailleGpuHandle {
    int device = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev[12] = {};  // 0-7: phases of create and solve; 8-11: the set-up split of create
    Symbolic sym;
    int npe = 0;
    int64_t n_nodes = 0, n_elems = 0;
    int precision = MAILLE_FP64;
    double tol = kDefaultTol;
    int32_t max_iter = kDefaultMaxIter;
    double delta = 0.3;  // reliable update when the FP32 residual fell by this factor
    std::vector<uint8_t> h_fixed;
    std::vector<double> h_f, h_f0;
    bool any_imposed = false;
    // device: inputs (caller numbering)
    double *coords = nullptr, *young = nullptr, *poisson = nullptr, *imposed = nullptr, *f = nullptr,
           *f0 = nullptr;  // f: loads of the current solve, f0: the problem's loads
    const double* f_cur = nullptr;
    int32_t* conn = nullptr;
    uint8_t* fixed = nullptr;
    // device: symbolic
    int32_t *perm = nullptr, *inv = nullptr, *col = nullptr, *lrow = nullptr;
    uint8_t* fixmask = nullptr;
    int64_t *row_ptr = nullptr, *diag = nullptr, *tpos = nullptr, *lslot = nullptr, *lptr = nullptr;
    uint32_t* contrib = nullptr;
    int64_t* inc_ptr = nullptr;
    int32_t *inc = nullptr, *belem = nullptr, *bnodes = nullptr, *elem_slot = nullptr;
    // device: numeric (CSR K and factor F; sliced copies for the iterations)
    double* ke = nullptr;
    double *K = nullptr, *F = nullptr;
    SellBuf sk;      // K, sliced, for the SpMV
    PsellBuf pl, pu;  // strictly lower / upper blocks of the factor, packed, for the sweeps
    double *Ks64 = nullptr, *Ls64 = nullptr, *Us64 = nullptr, *D64 = nullptr;
    float *Ks32 = nullptr, *Ls32 = nullptr, *Us32 = nullptr, *D32 = nullptr;
    // padded solver vectors (4 entries per block row); z64 / z32 hold the sweep records
    // (z0, z1, z2, tag) of the persistent kernel
    double *b64 = nullptr, *x64 = nullptr, *r64 = nullptr, *z64 = nullptr, *p64 = nullptr,
           *ap64 = nullptr;
    float *x32 = nullptr, *r32 = nullptr, *z32 = nullptr, *p32 = nullptr, *ap32 = nullptr;
    double *u_full = nullptr, *y_full = nullptr, *ye = nullptr, *gauss = nullptr, *vm = nullptr,
           *react = nullptr, *lambda_full = nullptr, *grad = nullptr;
    double *node_stress = nullptr, *node_vm = nullptr;  // smoothed nodal stresses [6 n], von Mises [n]
    PcgScalars* scal = nullptr;
    PcgScalars* h_scal = nullptr;  // pinned
    double* partials = nullptr;
    double* dsum = nullptr;        // [4] misc sums
    double* h_sum = nullptr;       // pinned [4]
    unsigned int* dticket = nullptr;
    int32_t* dfail = nullptr;
    int spmv_grid = 1;
    int persist_grid = 0;             // co-resident grid of the persistent PCG kernel
    int persist_chunk = 64;           // iterations per persistent launch
    unsigned long long* timing = nullptr;  // per-phase ns when MAILLE_PHASE_TIMING is set
    int32_t* claim = nullptr;              // [4]; claim[2]: the sweeps' timeout flag
    std::atomic<int> cancel{0};
    double shift = 0.0;
    bool solved = false;
    Pattern pattern() const {
        return Pattern{sym.nb, row_ptr, col, diag, tpos, fixmask};
    }
    ~MailleGpuHandle();
};

namespace maille {

// create: analysis, upload, element integration, assembly, IC(0) (FreeSystem::new + Pcg::new)
int32_t handle_create(const MailleElasticProblem* p, MailleGpuHandle** out, MailleElasticResult* res);
// assembly of the element matrices in h->ke, IC(0) with the shift ladder, sliced copies
int32_t handle_assemble_factor(MailleGpuHandle* h, Error& err);
// b64 = f_cur - K_fc imposed at free DOFs (solver numbering); K_fc from h->ke
void handle_build_rhs(MailleGpuHandle* h);
// PCG on K x64 = b64 (the handle's form); returns the MailleStatus
int32_t handle_run_pcg(MailleGpuHandle* h, int32_t* iterations, int32_t* updates, double* rel_res);
const char* handle_status_message(int32_t status, int32_t iters, double rel);

}  // namespace maille
