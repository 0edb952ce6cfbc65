// common.hpp -- shared host/device definitions of the B200 linear-elastic solve library.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/maille_gpu.h"

namespace maille {

// Tet element facts: nodes per element, Gauss points (TETRA_1 / TETRA_4, assembly.rs:212-229),
// node pairs (a <= b) of the symmetric element matrix.
inline int gauss_points(int npe) { return npe == 4 ? 1 : 4; }
inline int node_pairs(int npe) { return npe * (npe + 1) / 2; }

// Error carried up to the C ABI.
struct Error {
    int32_t status;
    std::string message;
};

// Symbolic analysis of one mesh: everything that depends on topology and the fixed-DOF mask but
// not on material values or loads. Built on the host (setup.cpp), uploaded once per handle.
//
// Block system: one 3x3 block row per "kept" node (a node with at least one free DOF). Fixed
// DOFs of a kept node become identity rows/columns, so the free-DOF matrix K_ff is embedded
// exactly; nodes with all three DOFs fixed are dropped. Rows are numbered in solver order
// (perm[new] = old node), grouped by level: rows of level l are [level_ptr[l], level_ptr[l+1])
// and depend only on rows of earlier levels in the lower triangle.
struct Symbolic {
    int64_t n_nodes = 0, n_elems = 0;
    int npe = 0;
    int32_t nb = 0;                    // block rows
    int64_t free_dofs = 0;
    std::vector<int32_t> perm;         // new -> old node
    std::vector<int32_t> inv;          // old node -> new row, -1 when dropped
    std::vector<uint8_t> fixmask;      // per new row: bit c set when DOF c is fixed
    std::vector<int32_t> level_ptr;    // [levels + 1]
    int32_t levels = 0;
    // full symmetric 3x3-block CSR pattern in new numbering, columns ascending
    std::vector<int64_t> row_ptr;      // [nb + 1]
    std::vector<int32_t> col;          // [B]
    std::vector<int64_t> diag;         // [nb] position of the diagonal block
    std::vector<int64_t> tpos;         // [B] position of the transposed block
    int64_t blocks = 0;
    // deterministic assembly: lower slots (col <= row), each summing a sorted list of element
    // node-pair blocks. contrib entry = (e * npairs + pair) | (transpose << 31)
    int64_t nl = 0;                    // lower slots
    std::vector<int64_t> lslot;        // [NL] position of the lower slot in the full pattern
    std::vector<int64_t> lptr;         // [NL + 1]
    std::vector<uint32_t> contrib;     // [pairs kept]
    // node -> (element, local node) incidence over all nodes, sorted by element
    std::vector<int64_t> inc_ptr;      // [n_nodes + 1]
    std::vector<int32_t> inc;          // [n_elems * npe] e * npe + a
    // elements that touch a fixed DOF (for the coupling K_fc u_c and the reactions)
    std::vector<int32_t> belem;
    std::vector<int32_t> bnodes;       // nodes with a fixed DOF that belong to a boundary element
    double ms = 0.0;
};

// Sliced 3x3-block layout of one matrix part (see sparse.cuh): K (full rows), L (strictly
// lower blocks) or U (strictly upper blocks, holding L^T). Slices never cross a level; inside a
// level rows are taken by decreasing length. src maps each slot to its block in the CSR
// pattern (-1 for padding), so the numeric values are filled by one gather per assembly.
// Padding slots point at column nb, a dummy node whose vector entries stay 0.
// Plan of the sliced layout of K (the slot columns and CSR sources are filled on the device from
// the plan and the pattern: fill_sell in analysis.cu).
struct SellHost {
    int32_t lpr = 1;
    std::vector<int32_t> rowid;         // [nslices * 32 / lpr], -1 when empty
    std::vector<int64_t> off{0};        // [nslices + 1] first step of each slice
    std::vector<int32_t> level_slices;  // [levels + 1]
    int64_t steps() const { return off.back(); }
    int32_t nslices() const { return (int32_t)off.size() - 1; }
};

enum SellKind { SELL_FULL = 0, SELL_LOWER = 1, SELL_UPPER = 2 };

// Packed sliced layout of the strictly lower (L) or upper (U) factor blocks, the operands of the
// dataflow sweeps. The rows of one level are packed in order into slices of one step of 128 slots
// (32 lanes x 4 consecutive slots, value plane k of step g at vals[(g * 9 + k) * 128 + slot] as in
// SellHost). A row takes max(1, length) consecutive slots and may span lanes; a slice closes when
// the next row does not fit or it holds 32 rows, and its unused slots are padding (the dummy node,
// zero values) that count as part of its last row. A row longer than 128 blocks gets a slice of its own over several
// steps. Bit b of head[4 s + w] is set when slot 32 w + b of slice s starts a row; the rows of
// slice s, in slot order, are rows[row0[s] .. row0[s + 1]). Slices are stored in sweep order:
// levels ascending for L (forward sweep), descending for U (backward sweep); level_slices[q] is
// the first slice of the q-th level swept.
// (Plan only: the slot columns and CSR sources are filled on the device, fill_psell.)
struct PsellHost {
    std::vector<int64_t> off{0};        // [nslices + 1] first step of each slice
    std::vector<uint32_t> head;         // [nslices * 4] row-start bits
    std::vector<int32_t> row0{0};       // [nslices + 1]
    std::vector<int32_t> rows;          // [nb] matrix row of each packed row
    std::vector<int64_t> rstart;        // [nb] first slot of each packed row
    std::vector<int32_t> level_slices;  // [levels + 1]
    int64_t steps() const { return off.back(); }
    int32_t nslices() const { return (int32_t)off.size() - 1; }
};

// Sliced layout of the batched solver (block-diagonal system of many instances, several
// right-hand sides). A slice holds `rows` rows of ONE instance (and, for L and U, of one level);
// each row's blocks are spread over `sub` lanes of 4 slots per step, so a step holds
// rows * sub * 4 slots: value plane k of step g at vals[(g * 9 + k) * slots + slot], columns at
// col[g * slots + slot]. K slices are ordered instance-major; L and U slices level-major, and
// inside a level instance by instance. Padding slots point at the dummy node nb.
struct BSellHost {
    int rows = 4, sub = 1;
    int slots() const { return rows * sub * 4; }
    std::vector<int32_t> rowid;         // [nslices * rows], -1 when empty
    std::vector<int64_t> off{0};        // [nslices + 1] first step of each slice
    std::vector<int32_t> col, src;      // [steps * slots]
    std::vector<int32_t> inst;          // [nslices] instance of the slice
    std::vector<int32_t> level_slices;  // [levels + 1] (L and U)
    int64_t steps() const { return off.back(); }
    int32_t nslices() const { return (int32_t)off.size() - 1; }
};

// Builds the batched layout of one part of the analysed pattern; group[row] is the row's
// instance (rows of one instance must form one connected block of the matrix).
void build_bsell(const Symbolic& s, SellKind kind, int rows, int sub, const std::vector<int32_t>& group,
                 BSellHost& out);

// Plans the sliced layout of one part of the analysed pattern (reads s.row_ptr, s.diag and the
// levels only). lpr <= 0 picks lanes per row from the mean row length.
void build_sell(const Symbolic& s, SellKind kind, int lpr, SellHost& out);

// Plans the packed layout of the strictly lower (SELL_LOWER) or upper (SELL_UPPER) blocks (reads
// s.row_ptr, s.diag and the levels only).
void build_psell(const Symbolic& s, SellKind kind, PsellHost& out);

// Builds the symbolic analysis. conn is [n_elems * npe] in the caller's node numbering. With
// pattern = false it stops after the ordering, the levels and the boundary lists (perm, inv,
// fixmask, level_ptr, incidence, belem, bnodes): the block pattern and the scatter map are then
// built on the device (analysis.cu). With boundary_lists = false, belem and bnodes (the elements
// and nodes of the elastic reactions) are left empty.
bool analyse(int64_t n_nodes, int npe, int64_t n_elems, const int64_t* conn,
             const uint8_t* fixed, int ordering, Symbolic& s, Error& err, bool pattern = true,
             bool boundary_lists = true);

// The part of analyse that does not depend on the ordering: the input checks, the node incidence
// (with incidence = false only its run starts inc_ptr: the device builds inc, ordering.cuh
// gpu_incidence), the kept nodes (a
// node with a free DOF: kept in caller order, kept_of[v] its kept index or -1), the free DOF count
// and, with boundary_lists, belem and bnodes.
bool analyse_topology(int64_t n_nodes, int npe, int64_t n_elems, const int64_t* conn, const uint8_t* fixed,
                      Symbolic& s, std::vector<int32_t>& kept, std::vector<int32_t>& kept_of, Error& err,
                      bool boundary_lists, bool incidence = true);

// The ordering fields of s (nb, perm, inv, fixmask, levels, level_ptr) from an ordering computed
// elsewhere: order[new row] = kept index with rows grouped by level, level[kept index].
void apply_ordering(const std::vector<int32_t>& kept, const std::vector<int32_t>& order,
                    const std::vector<int32_t>& level, const uint8_t* fixed, Symbolic& s);

// Face pressure loads f_a -= p * integral(N_a n dS) added into f (assembly.rs:650-674 with the
// tet branch of face_rule, assembly.rs:556-585). Host-side: part of the host program's assemble.
bool face_pressure_loads(int64_t n_nodes, const double* coords, int npe, int64_t n_elems,
                         const int64_t* conn, int64_t n_press, const int64_t* p_elem,
                         const int32_t* p_face, const double* p_value, double* f, Error& err);

}  // namespace maille
