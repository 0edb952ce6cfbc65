// analysis.cuh -- the symbolic analysis steps that run on the device (analysis.cu): the full
// 3x3-block pattern in solver numbering, its transpose positions, the lower slots with their
// element-pair scatter map, and the slot columns of the SpMV and sweep layouts. The host keeps the
// ordering (RCM, greedy colouring, levels: setup.cpp); everything here is a deterministic
// function of the connectivity and that ordering, equal entry for entry to the host analysis.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "common.hpp"

namespace maille {

// Device arrays of the analysed pattern; the caller owns them (cudaFree) once built.
struct PatternDev {
    int64_t* row_ptr = nullptr;    // [nb + 1]
    int32_t* col = nullptr;        // [blocks], ascending per row
    int64_t* diag = nullptr;       // [nb]
    int64_t* tpos = nullptr;       // [blocks] position of the transposed block
    int64_t* lslot = nullptr;      // [nl] full-pattern position of each lower slot
    int32_t* lrow = nullptr;       // [nl] row of each lower slot
    int64_t* lptr = nullptr;       // [nl + 1]
    uint32_t* contrib = nullptr;   // [lptr[nl]] (e * npairs + pair) | (transposed << 31)
    int64_t blocks = 0, nl = 0, ncontrib = 0;
};

// Builds the pattern of the kept nodes from the connectivity (conn: [n_elems * npe] on the
// device, caller numbering) and inv (caller node -> solver row, -1 when dropped; on the device).
// Also returns host copies of row_ptr and diag (the layout plans need the row lengths).
// Throws CudaFailure on a CUDA error.
void gpu_pattern(int npe, int64_t n_elems, const int32_t* conn, const int32_t* inv, int32_t nb,
                 cudaStream_t st, PatternDev& out, std::vector<int64_t>& h_row_ptr,
                 std::vector<int64_t>& h_diag);

// Slot columns (col, padding = nb) and CSR sources (src, padding = -1) of a sliced K layout
// (kind SELL_FULL) from its plan (rowid, off already on the device) and the device pattern.
void fill_sell(SellKind kind, int32_t lpr, int32_t nslices, int64_t steps, const int32_t* rowid,
               const int64_t* off, const int64_t* row_ptr, const int32_t* col, const int64_t* diag,
               int32_t nb, int32_t* slot_col, int32_t* slot_src, cudaStream_t st);

// The same for a packed factor layout (rows, rstart of the plan on the device).
void fill_psell(SellKind kind, int64_t nrows, int64_t steps, const int32_t* rows, const int64_t* rstart,
                const int64_t* row_ptr, const int32_t* col, const int64_t* diag, int32_t nb,
                int32_t* slot_col, int32_t* slot_src, cudaStream_t st);

}  // namespace maille
