/* maille_gpu.h -- C ABI of the B200 linear-elastic solve path (Tet4/Tet10 stiffness, deterministic
 * sparse assembly, IC(0)-preconditioned conjugate gradients, Gauss-point stresses), and of the
 * transient heat conduction step built on the same machinery (maille_gpu_thermal_transient).
 *
 * The entry points replace the iterative branch of maille-core's solve (reference paths, relative
 * to the reference project root):
 *   - Model::solve                      crates/maille-core/src/model.rs:548-610
 *   - FreeSystem::new / ::solve         crates/maille-core/src/model.rs:1442-1516
 *   - FreeMatrix / Factor dispatch      crates/maille-core/src/model.rs:1390-1423
 *   - Pcg::new / Pcg::solve             crates/maille-core/src/iterative.rs:199-248
 *   - element_stiffness / _stresses     crates/maille-core/src/assembly.rs:64-79, 304-312
 *   - product (reactions)               crates/maille-core/src/model.rs:1353-1369
 * A host program calls them where SolverKind::is_iterative (solve.rs:187-195) selects the PCG
 * path; the skyline direct solver stays in the host program.
 *
 * Conventions: all pointers are caller-owned host memory unless stated; the library copies in and
 * out and never keeps host pointers. Every call returns a MailleStatus; no call aborts or throws
 * across the ABI. Device code never traps: failures are written to an on-device status word that
 * the host reads. A handle is used by one host thread at a time (it may move between threads).
 */
#ifndef MAILLE_GPU_H
#define MAILLE_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Return codes, mirroring MailleError on this path (crates/maille-core/src/error.rs). */
typedef enum {
    MAILLE_OK = 0,
    MAILLE_SINGULAR = 1,      /* IC(0) failed every diagonal shift, or p.Ap <= 0 / NaN
                                 -> MailleError::Singular (error.rs:224) */
    MAILLE_NOT_CONVERGED = 2, /* iteration cap reached -> IterativeNotConverged{iterations,
                                 residual} (error.rs:226-229) */
    MAILLE_INVALID_INPUT = 3, /* bad sizes, node index out of range, non-finite input */
    MAILLE_CUDA_ERROR = 4,    /* message through maille_gpu_last_error() */
    MAILLE_CANCELLED = 5      /* the cancel flag was raised (MailleError::Cancelled, error.rs:156) */
} MailleStatus;

/* Storage precision of the matrix and preconditioner. */
typedef enum {
    MAILLE_FP64 = 0,  /* plain form: FP64 throughout */
    MAILLE_MIXED = 1  /* FP32 matrix and IC(0) factor in an FP32 inner PCG, inside FP64
                         iterative refinement (outer residual f - K u against FP64 K, FP64
                         solution accumulation, FP64 refinement dots, FP64 factor pivots) */
} MaillePrecision;

/* Ordering of the free nodes for the level-scheduled IC(0). */
typedef enum {
    MAILLE_ORDER_AUTO = 0,           /* the path's measured best: MULTICOLOR_ITERATED for the
                                        elastic solves, MULTICOLOR_BFS for the thermal step */
    MAILLE_ORDER_MULTICOLOR = 1,     /* greedy colouring of the node graph visited in RCM order:
                                        one level per colour, a few dozen levels */
    MAILLE_ORDER_RCM = 2,            /* reverse Cuthill-McKee on the node graph (the reference's
                                        algorithm, solve.rs:200-245, applied to nodes): the
                                        reference's convergence, hundreds of levels */
    MAILLE_ORDER_MULTICOLOR_BFS = 3, /* greedy colouring visited in reverse breadth-first order
                                        from a minimum-degree node (one breadth-first pass, no
                                        pseudo-peripheral search): usually one colour fewer and
                                        fewer FP64 iterations than MULTICOLOR */
    MAILLE_ORDER_MULTICOLOR_ITERATED = 4 /* MULTICOLOR's colouring, then two passes of iterated
                                        greedy (each recolours the nodes visited by colour class,
                                        the last class first): fewer colours, hence fewer levels
                                        (15 against 18 on the Tet10 cube), never more */
} MailleOrdering;

/* A linear static Tet4/Tet10 model (Model after `assemble`, model.rs:1070-1147). */
typedef struct {
    int64_t n_nodes;
    const double* coords;    /* [3 n_nodes] x, y, z per node */
    int32_t nodes_per_elem;  /* 4 (Tet4, TETRA_1 rule) or 10 (Tet10, TETRA_4 rule) */
    int64_t n_elems;
    const int64_t* conn;     /* [n_elems * nodes_per_elem], Maille node order (Tet10 mid-edge
                                nodes in TET10_EDGES order, shape.rs:135) */
    const double* young;     /* [n_elems] E per element (Tet4/Tet10 carry their Material) */
    const double* poisson;   /* [n_elems] nu per element */
    const uint8_t* fixed;    /* [3 n_nodes] 1 where a Bc fixes the DOF (3 node + c) */
    const double* imposed;   /* [3 n_nodes] imposed values at fixed DOFs (ignored elsewhere, any
                                value there), or NULL for zero */
    const double* f;         /* [3 n_nodes] assembled nodal loads F (loads + face pressures), or
                                NULL for zero */
    double rel_tol;          /* stop at ||r|| <= rel_tol ||b|| (the reference uses 1e-12);
                                <= 0 selects 1e-12 */
    int32_t max_iter;        /* <= 0 selects 10000 (iterative.rs:11) */
    int32_t precision;       /* MaillePrecision */
    int32_t ordering;        /* MailleOrdering */
    int32_t device;          /* CUDA device ordinal */
} MailleElasticProblem;

/* Results, caller-allocated; any output pointer may be NULL to skip it. */
typedef struct {
    double* u;             /* [3 n_nodes] displacements (Field::displacements) */
    double* reactions;     /* [3 n_nodes] K u - F at fixed DOFs, 0 elsewhere (Field::reactions) */
    double* gauss_stress;  /* [n_elems * ngp * 9] per Gauss point: x, y, z, sxx, syy, szz, txy,
                              tyz, txz (Stress, results.rs:6-20); ngp = 1 (Tet4) or 4 (Tet10) */
    double* von_mises;     /* [n_elems * ngp] Stress::von_mises (results.rs:24-32) */
    /* filled by the library */
    int32_t iterations;         /* PCG iterations (mixed: total inner iterations) */
    int32_t outer_iterations;   /* mixed: refinement steps; plain: 1 */
    double final_rel_residual;  /* ||f - K u|| / ||f|| in FP64 on the free DOFs */
    double shift;               /* diagonal shift IC(0) succeeded with (iterative.rs:14) */
    int64_t free_dofs;
    int64_t block_rows;         /* free nodes in the 3x3-block system */
    int64_t blocks;             /* 3x3 blocks of the full symmetric pattern */
    int32_t levels;             /* levels of the IC(0) sweeps */
    double ms_setup;            /* host analysis on a thread that runs while the device takes the
                                   inputs (create): node incidence and boundary lists, and with
                                   MAILLE_HOST_ORDERING=1 the ordering too */
    double ms_upload;           /* host -> device copies of the inputs (create) */
    double ms_assembly;         /* scatter-reduce assembly of the element matrices (create,
                                   refactor) */
    double ms_factor;           /* IC(0) factorisation incl. shift retries */
    double ms_solve;            /* PCG iterations (mixed: incl. refinement) */
    double ms_post;             /* reactions + stresses + von Mises */
    double ms_download;         /* device -> host copies */
    /* the rest of create, in order on the device stream (each 0 after solve-only calls): */
    double ms_element;          /* element integration (Ke of every element) */
    double ms_ordering;         /* wall time from the element integration to a known ordering:
                                   the device node incidence, the device ordering (node graph,
                                   RCM, greedy colouring) and the join of the host thread */
    double ms_symbolic;         /* device pattern and scatter map (radix sorts), the host plan of
                                   the sliced layouts and their slot fills */
    double ms_buffers;          /* numeric buffers and the remaining index uploads */
} MailleElasticResult;

typedef struct MailleGpuHandle MailleGpuHandle;

/* Last error message of the calling thread (empty string when none). */
const char* maille_gpu_last_error(void);

/* Library version string. */
const char* maille_gpu_version(void);

/* Number of CUDA devices visible (0 when none; never an error). */
int32_t maille_gpu_device_count(void);

/* One-shot solve: create + solve + destroy. Replaces, for a Tet4/Tet10 linear static model,
 * FreeSystem::new (model.rs:1442-1499) with Pcg::new (iterative.rs:201-207), FreeSystem::solve
 * (model.rs:1502-1516) with Pcg::solve (iterative.rs:210-248), then product (model.rs:586-593,
 * 1353-1369) and element_stresses (model.rs:596-598). */
int32_t maille_gpu_elastic_solve(const MailleElasticProblem* problem, MailleElasticResult* result);

/* Handle API (reuse one analysis for several right-hand sides; the adjoint).
 * create: symbolic analysis + upload + element integration + assembly + IC(0) factorisation
 * (FreeSystem::new + Pcg::new). The handle owns all device memory. */
int32_t maille_gpu_create(const MailleElasticProblem* problem, MailleGpuHandle** out);

/* Solve K_ff u_f = F_f - K_fc u_c for a new load vector f ([3 n_nodes], NULL = the problem's),
 * then reactions and stresses into `result` (FreeSystem::solve + product + element_stresses). */
int32_t maille_gpu_solve(MailleGpuHandle* h, const double* f, MailleElasticResult* result);

/* The same solve with device-resident buffers, for callers that chain solves on the GPU (load
 * cases, an optimisation loop): f_dev [3 n_nodes] device pointer on the handle's device (NULL =
 * the problem's loads), the displacements (imposed values at fixed DOFs) written to u_dev
 * [3 n_nodes] device pointer; no reactions, stresses or host copies (FreeSystem::solve,
 * model.rs:1502-1516, without product and element_stresses). The loads are not checked on the
 * host: non-finite values end in MAILLE_SINGULAR. Returns when u_dev is written; a backward may
 * follow. */
int32_t maille_gpu_solve_device(MailleGpuHandle* h, const double* f_dev, double* u_dev);

/* Adjoint of the last solve: with g = dJ/du ([3 n_nodes], host), solves K_ff lambda_f = g_f with
 * the same PCG and factor (lambda = 0 on fixed DOFs), then
 *   dJ/dE_e = -lambda_e^T (dK_e/dE_e) u_e = -lambda_e^T K_e u_e / E_e
 * for every element into dJdE ([n_elems]). lambda ([3 n_nodes]) is returned when not NULL.
 * No counterpart in the reference (it has no gradients). */
int32_t maille_gpu_backward(MailleGpuHandle* h, const double* dJdu, double* dJdE, double* lambda);

/* Numeric refactorisation on the handle's topology: new per-element materials ([n_elems] each,
 * NULL keeps the current ones), then element integration, assembly and IC(0) again, as the
 * reference rebuilds FreeSystem when the matrix changes (model.rs:1011). The ordering, pattern
 * and scatter map are reused; the next solve uses the new matrix. */
int32_t maille_gpu_refactor(MailleGpuHandle* h, const double* young, const double* poisson);

/* y = K x with the assembled free-DOF matrix (Csr::multiply, iterative.rs:131-142): x and y are
 * [3 n_nodes] in the caller's numbering; x is read at free DOFs, y is 0 at fixed DOFs. */
int32_t maille_gpu_multiply(MailleGpuHandle* h, const double* x, double* y);

/* Nodal stresses of the last solve (nodal_stresses / smooth, results.rs:137-230, and the
 * `stress` / `von_mises` point arrays of maille-io/src/vtk/fields.rs:54-74): the Gauss-point
 * stresses extrapolated to each element's nodes (Tet4: the point value; Tet10: the
 * TET10_EXTRAPOLATION weights, results.rs:114-132) and averaged over the elements sharing a node,
 * in element order; a node no element touches gets 0. stress: [6 n_nodes] (sxx, syy, szz, txy,
 * tyz, txz per node), von_mises: [n_nodes] (Stress::von_mises of the smoothed stress). Needs a
 * solve on the handle (MAILLE_INVALID_INPUT otherwise). */
int32_t maille_gpu_nodal_stresses(MailleGpuHandle* h, double* stress, double* von_mises);

/* Self-test of the bounded waits of the IC(0) sweeps (failure detection without a GPU fault): one
 * warp awaits four sweep records, one of them stale when `stale` is non-zero (its tag is the epoch
 * before the awaited one and nothing writes it), with the sweeps' re-read loop limited to 4096
 * rounds. *timed_out is 1 when the wait ran out and 0 when all records were current; the call
 * itself returns MAILLE_OK unless CUDA failed. A sweep whose wait runs out the same way ends the
 * solve with MAILLE_CUDA_ERROR. No counterpart in the reference. */
int32_t maille_gpu_wait_selftest(int32_t device, int32_t stale, int32_t* timed_out);

/* Device memory: the library allocates from one memory pool per device that keeps freed memory
 * reserved, so creating and destroying handles repeatedly does not map and unmap GBs each time.
 * This returns the pool's unused memory of `device` to the device (call it when no handle is
 * alive and the memory is wanted elsewhere). No counterpart in the reference. */
int32_t maille_gpu_trim_memory(int32_t device);

/* Enqueues `count` launches of the PCG's 3x3-block SpMV kernel on the handle's device vectors
 * and stream (precision MAILLE_FP64 or MAILLE_MIXED for the FP32 matrix), without waiting: for
 * timing the kernel with events on maille_gpu_stream(). No counterpart in the reference. */
int32_t maille_gpu_spmv_device(MailleGpuHandle* h, int32_t precision, int32_t count);

/* Kernels this library has launched in the process (a CUDA graph launch adds its kernel nodes).
 * No counterpart in the reference. */
int64_t maille_gpu_kernel_launches(void);

/* Raise (1) or clear (0) the cancel flag; checked between PCG iteration chunks. Safe to call
 * from another thread while a solve runs (the Observer / Flow::Stop role, model.rs:1203-1218). */
void maille_gpu_cancel(MailleGpuHandle* h, int32_t flag);

/* CUDA stream (cudaStream_t) the handle launches on, for event timing by the caller. */
void* maille_gpu_stream(MailleGpuHandle* h);

void maille_gpu_destroy(MailleGpuHandle* h);

/* Host helper: adds the nodal forces of face pressures to f ([3 n_nodes]):
 * f_a -= p * integral over the face of N_a n dS, n the outward normal (face_pressure,
 * assembly.rs:650-674, with the tet branch of face_rule, assembly.rs:556-585; TRIANGLE_3 on Tet4
 * faces, TRIANGLE_6 on Tet10 faces). Faces are (element, face in 0..3: 0-1-2, 0-3-1, 1-3-2,
 * 2-3-0) pairs; an out-of-range element or face adds nothing, like face_rule's None. Runs on the
 * host: it is the part of the host program's `assemble` (model.rs:1124-1131) a caller without
 * its own face integration needs. */
int32_t maille_gpu_face_pressure_loads(int64_t n_nodes, const double* coords, int32_t npe,
                                       int64_t n_elems, const int64_t* conn, int64_t n_press,
                                       const int64_t* p_elem, const int32_t* p_face,
                                       const double* p_value, double* f);

/* ---- Batched solves ------------------------------------------------------------------------
 * No counterpart in the reference, whose Model::solve (model.rs:548-610) takes one mesh and one
 * load vector: a host program with many independent models (or one model and several load cases)
 * calls Model::solve once per model and load case. The batch entry points take many Tet4/Tet10
 * models of uneven size, each with the same number of load cases, and solve them all in one
 * persistent kernel over the packed block-diagonal matrix (per-instance offsets): block PCG over
 * the right-hand sides of each instance (the matrix and factor are read once for all load
 * cases), per-instance convergence masks, the solve captured as a CUDA graph. The lane layout,
 * block size and task packing are chosen by an autotuner at the first solve and cached per
 * matrix shape for the process (environment MAILLE_AUTOTUNE_CACHE = a file keeps them across
 * processes). Each instance follows its own Model::solve contract: IC(0)-PCG to
 * ||r|| <= rel_tol ||b|| per load case, u = imposed values at fixed DOFs. */

/* Largest number of load cases per instance. */
#define MAILLE_BATCH_MAX_RHS 8

typedef struct {
    int32_t n_instances;
    int32_t nodes_per_elem;      /* 4 or 10, every instance */
    int32_t n_rhs;               /* load cases per instance, 1..MAILLE_BATCH_MAX_RHS */
    const int64_t* node_offset;  /* [n_instances + 1] instance k owns nodes [node_offset[k],
                                    node_offset[k + 1]) of the packed node arrays */
    const int64_t* elem_offset;  /* [n_instances + 1] and elements [elem_offset[k], ...) */
    const double* coords;        /* [3 total_nodes] */
    const int64_t* conn;         /* [total_elems * nodes_per_elem] node ids LOCAL to the
                                    instance (0 .. its node count - 1) */
    const double* young;         /* [total_elems] */
    const double* poisson;       /* [total_elems] */
    const uint8_t* fixed;        /* [3 total_nodes] */
    const double* imposed;       /* [3 total_nodes] imposed values at fixed DOFs, or NULL */
    const double* f;             /* [n_rhs][3 total_nodes] load cases (load case j of instance k
                                    at f[j * 3 total_nodes + 3 node_offset[k] ...]), or NULL */
    double rel_tol;              /* <= 0 selects 1e-12 */
    int32_t max_iter;            /* per instance; <= 0 selects 10000 */
    int32_t precision;           /* MaillePrecision */
    int32_t device;
} MailleBatchProblem;

typedef struct {
    double* u;                   /* [n_rhs][3 total_nodes] displacements, or NULL */
    int32_t* iterations;         /* [n_instances * n_rhs] iterations each load case took, or NULL */
    double* rel_residual;        /* [n_instances * n_rhs] final ||r|| / ||b||, or NULL */
    int32_t* status;             /* [n_instances] MailleStatus of each instance, or NULL */
    /* filled by the library */
    int32_t max_iterations;      /* iterations of the slowest instance */
    int32_t levels;
    int64_t free_dofs;           /* over all instances (per load case) */
    int64_t block_rows;
    int64_t blocks;
    int32_t lanes_per_row;       /* autotuned: lanes sharing one row (load-case groups x sub-lanes) */
    int32_t rhs_per_lane;        /* autotuned: load cases one lane carries */
    int32_t threads;             /* autotuned: threads per block */
    int32_t task_slices;         /* autotuned: slices per vector task */
    int32_t autotuned;           /* 1 when this call ran the tuner, 0 when the cache served it */
    double ms_setup, ms_upload, ms_assembly, ms_factor, ms_tune, ms_solve, ms_download;
} MailleBatchResult;

typedef struct MailleGpuBatch MailleGpuBatch;

/* One-shot: create + solve + destroy. Returns MAILLE_OK when every instance converged, else the
 * first failing instance's status (per-instance statuses in result->status). */
int32_t maille_gpu_batched_solve(const MailleBatchProblem* problem, MailleBatchResult* result);

/* Packing + symbolic analysis + upload + element integration + assembly + IC(0) of all
 * instances. */
int32_t maille_gpu_batch_create(const MailleBatchProblem* problem, MailleGpuBatch** out);

/* Solves every instance for every load case (f as in the problem, NULL = the problem's). */
int32_t maille_gpu_batch_solve(MailleGpuBatch* b, const double* f, MailleBatchResult* result);

/* New per-element materials ([total_elems] each, NULL keeps the current ones): element
 * integration, assembly and IC(0) again on the same packing. */
int32_t maille_gpu_batch_refactor(MailleGpuBatch* b, const double* young, const double* poisson);

/* Raise (1) or clear (0) the batch's cancel flag; the running kernel polls it once per PCG
 * pass and the solve returns MAILLE_CANCELLED. Safe to call from another thread. */
void maille_gpu_batch_cancel(MailleGpuBatch* b, int32_t flag);

/* CUDA stream of the batch, for event timing by the caller. */
void* maille_gpu_batch_stream(MailleGpuBatch* b);

void maille_gpu_batch_destroy(MailleGpuBatch* b);

/* ---- Large strain: neo-Hookean Tet4, quasi-static Newton, adjoint ----------------------------
 * Replaces, for a Tet4 model with Kinematics::Large and Hyperelasticity::NeoHookean on every
 * element, Model::solve_quasi_static (model.rs:720-806) over Step::quasi_static(1, increments)
 * with the linear amplitude (0,0)-(1,1): each increment is Newton-Raphson to F_int(u) = lambda F
 * with imposed values lambda * imposed (equilibrium, model.rs:923-1022: relative residual
 * ||r_free|| / scale <= newton_tol after at least two residuals, at most newton_max_iter, the
 * increment halved up to 5 times when Newton does not converge or the tangent is not positive
 * definite, advance, model.rs:820-870; an inner PCG at its cap ends the run without a cut, as the
 * reference's IterativeNotConverged does), each linear step
 * K_ff du_f = -r_f - K_fc du_c solved by this library's assembly + IC(0)-PCG. The element
 * response is large_strain_response (finite_strain.rs:119-214) with the neo-Hookean law
 * (finite_strain.rs:40-86), lambda and mu = lame(E, nu) per element (finite_strain.rs:30-35).
 * Follower pressures, contacts and plasticity are not part of this path.
 *
 * backward (no counterpart in the reference): for J = sum_k dJdR[k] . R_k, R_k the reactions of
 * increment k (F_int - lambda F at fixed DOFs), the reverse pass recomputes the tangent at each
 * increment's checkpointed displacements, solves K_ff m_f = -K_fc g_c with the same PCG and
 * accumulates dJ/dmu_e and dJ/dlambda_e = w_e . dF_int,e/dp_e, w = (g_c, m_f). */
typedef struct {
    int64_t n_nodes;
    const double* coords;     /* [3 n_nodes] */
    int64_t n_elems;
    const int64_t* conn;      /* [n_elems * 4] Tet4 */
    const double* young;      /* [n_elems] E per element (lambda, mu = lame(E, nu)) */
    const double* poisson;    /* [n_elems] */
    const uint8_t* fixed;     /* [3 n_nodes] */
    const double* imposed;    /* [3 n_nodes] imposed values at the end of the step */
    const double* f;          /* [3 n_nodes] external loads at the end of the step, or NULL */
    int32_t increments;       /* equal increments of the step (> 0) */
    double newton_tol;        /* <= 0 selects 1e-8 (model.rs:1220) */
    int32_t newton_max_iter;  /* <= 0 selects 25 (model.rs:1222) */
    double rel_tol;           /* PCG tolerance, <= 0 selects 1e-12 */
    int32_t max_iter;         /* PCG iterations, <= 0 selects 10000 */
    int32_t precision;        /* MaillePrecision of the PCG */
    int32_t device;
} MailleLargeStrainProblem;

typedef struct {
    double* u;                  /* [increments][3 n_nodes] converged displacements, or NULL */
    double* reactions;          /* [increments][3 n_nodes] F_int - lambda F at fixed DOFs, or NULL */
    int32_t* newton_iterations; /* [increments] residuals of the last equilibrium, or NULL */
    int32_t* cuts;              /* [increments] interval halvings, or NULL; when the run fails,
                                   the failing increment's entry holds its halvings so far */
    int64_t newton_total;       /* filled: Newton iterations over the step */
    int64_t pcg_total;          /* filled: PCG iterations over the step */
    double ms_total;
} MailleLargeStrainResult;

typedef struct MailleGpuLargeStrain MailleGpuLargeStrain;

int32_t maille_gpu_large_strain_create(const MailleLargeStrainProblem* problem, MailleGpuLargeStrain** out);
/* Runs the whole step; the per-increment displacements stay on the device as checkpoints. */
int32_t maille_gpu_large_strain_run(MailleGpuLargeStrain* s, MailleLargeStrainResult* result);
/* dJdR [increments][3 n_nodes] (read at fixed DOFs) -> dJdmu [n_elems], dJdlambda [n_elems] or NULL */
int32_t maille_gpu_large_strain_backward(MailleGpuLargeStrain* s, const double* dJdR, double* dJdmu,
                                         double* dJdlambda);
/* New per-element E and nu (NULL keeps them); the next run starts from rest. */
int32_t maille_gpu_large_strain_set_materials(MailleGpuLargeStrain* s, const double* young,
                                              const double* poisson);
/* Raise (1) or clear (0) the run's cancel flag (the observer's Flow::Stop of
 * solve_quasi_static_with, model.rs:732, 1203-1218): checked before every Newton iteration and
 * between the inner PCG's launches; the run then returns MAILLE_CANCELLED (MailleError::Cancelled,
 * error.rs:156) without a cut. Safe to call from another thread while a run is in progress; a
 * raised flag stays raised until cleared. */
void maille_gpu_large_strain_cancel(MailleGpuLargeStrain* s, int32_t flag);
void maille_gpu_large_strain_destroy(MailleGpuLargeStrain* s);

/* ---- Transient heat conduction: the theta-method ---------------------------------------------
 * Replaces, for a Tet4/Tet10 model with Analysis::Thermal, Model::solve_step / solve_step_with
 * (model.rs:621-706) on the iterative FreeSystem: element conduction K_e (conduction,
 * element.rs:451-463, rule TETRA_1 / TETRA_4) plus the convection terms h int N N^T dS of the
 * model's Convection faces (FaceConvection::add_matrix, assembly.rs:495-503), consistent capacity
 * C_e (capacity, element.rs:465-477, rule TETRA_4 / TETRA_14, element_capacity,
 * assembly.rs:413-433), then per increment
 *   (C/dt + theta K) T_{n+1} = (C/dt - (1 - theta) K) T_n + F
 * with the left matrix assembled and IC(0)-factorised once (FreeSystem::new, model.rs:1442-1499;
 * Pcg::new) and each increment solved by IC(0)-PCG from a zero start to ||r|| <= rel_tol ||b||
 * (Pcg::solve, iterative.rs:210-248); reactions R = C (T_{n+1} - T_n)/dt + K (theta T_{n+1} +
 * (1 - theta) T_n) - F on imposed nodes and the heat fluxes q = -k grad T (heat_fluxes,
 * element.rs:480-506) of every increment. Imposed temperatures replace the initial field at
 * their nodes from t = 0. The whole step runs on the device: one host synchronisation at the
 * end, the history kept in device memory until then. */
typedef struct {
    int64_t n_nodes;
    const double* coords;         /* [3 n_nodes] */
    int32_t nodes_per_elem;       /* 4 or 10 */
    int64_t n_elems;
    const int64_t* conn;          /* [n_elems * nodes_per_elem], Maille node order */
    const double* conductivity;   /* [n_elems] k of each element's Material */
    const double* rho_c;          /* [n_elems] density x specific heat */
    const uint8_t* fixed;         /* [n_nodes] 1 where a Bc imposes T (Dof::T) */
    const double* imposed;        /* [n_nodes] imposed T at fixed nodes (ignored elsewhere) */
    const double* f;              /* [n_nodes] assembled heat loads F: nodal loads, heat sources
                                     and the convection loads h T_inf int N dS (assemble,
                                     model.rs:1070-1147; maille_gpu_thermal_loads adds the last
                                     two), or NULL for zero */
    int64_t n_convection;         /* convection faces whose h int N N^T dS joins K */
    const int64_t* conv_elem;     /* [n_convection] element */
    const int32_t* conv_face;     /* [n_convection] face 0..3 (0-1-2, 0-3-1, 1-3-2, 2-3-0); an
                                     out-of-range face adds nothing, like face_rule's None */
    const double* conv_film;      /* [n_convection] h */
    const double* initial;        /* [n_nodes] T at t = 0 */
    double time_step;             /* dt > 0 (Step::time_step, model.rs:171-173) */
    double theta;                 /* 0.5 <= theta <= 1 (Step::with_theta, model.rs:151-156) */
    int32_t increments;           /* > 0 */
    double rel_tol;               /* <= 0 selects 1e-12 */
    int32_t max_iter;             /* per increment; <= 0 selects 10000 */
    int32_t ordering;             /* MailleOrdering of the free nodes */
    int32_t device;
    int32_t precision;            /* MaillePrecision: MAILLE_FP64 (0), or MAILLE_MIXED: FP32 matrices
                                     and vectors in the PCG with FP64 reliable updates (x accumulated
                                     in FP64, true residual b - A x against the FP64 matrix, the
                                     stopping test on it) */
} MailleThermalProblem;

typedef struct {
    double* temperatures;   /* [(increments + 1) n_nodes] T of every increment, t = 0 first, or NULL */
    double* reactions;      /* [(increments + 1) n_nodes] R at imposed nodes, 0 elsewhere and at
                               t = 0, or NULL */
    double* heat_fluxes;    /* [(increments + 1) n_elems ngp 6] per Gauss point x, y, z, qx, qy,
                               qz (HeatFlux, results.rs); ngp = 1 (Tet4) or 4 (Tet10); or NULL */
    int32_t* iterations;    /* [increments] PCG iterations of each increment, or NULL */
    /* filled by the library */
    int64_t iterations_total;
    double max_rel_residual;  /* largest final ||r|| / ||b|| over the increments */
    double shift;             /* diagonal shift IC(0) succeeded with */
    int64_t free_nodes;
    int64_t nonzeros;         /* entries of the full symmetric pattern of the free nodes */
    int32_t levels;           /* levels of the IC(0) sweeps */
    double ms_setup;          /* host node incidence (and the ordering with MAILLE_HOST_ORDERING=1) */
    double ms_upload;         /* host -> device copies and device analysis */
    double ms_assembly;       /* element matrices + assembly of the left and right matrices */
    double ms_factor;         /* IC(0) incl. shift retries */
    double ms_steps;          /* every increment: right-hand side, PCG, reactions, fluxes */
    double ms_download;       /* device -> host copies of the history */
} MailleThermalResult;

/* The whole transient step (Model::solve_step). MAILLE_SINGULAR / MAILLE_NOT_CONVERGED name the
 * first increment whose solve failed; MAILLE_CANCELLED the first increment the cancel flag
 * stopped; the history before it is returned. */
int32_t maille_gpu_thermal_transient(const MailleThermalProblem* problem, MailleThermalResult* result);

/* Raise (1) or clear (0) the thermal cancel flag of `device` (the observer's Flow::Stop of
 * solve_step_with, model.rs:628, 1203-1218): every thermal step running or started on that device
 * checks it on the device before each increment's solve and, when raised, skips that increment
 * and the rest and returns MAILLE_CANCELLED (MailleError::Cancelled, error.rs:156), with the
 * history of the increments completed before it. The flag is per device, not per call: it stops
 * every thermal step on the device and stays raised until cleared. Safe to call from another
 * thread while a step runs. MAILLE_INVALID_INPUT for a device ordinal outside 0..63. */
int32_t maille_gpu_thermal_cancel(int32_t device, int32_t flag);

/* Host helper: adds to f ([n_nodes]) the heat-source loads int N q dV of uniform sources
 * (element, q) (element_heat_source / nodal_source, assembly.rs:466-484, element rule TETRA_1 /
 * TETRA_4) and the convection loads h T_inf int N dS of faces (element, face, h, T_inf)
 * (face_convection, assembly.rs:595-626; FaceConvection::add_load), in the order of the
 * reference's assemble (model.rs:1101-1140). Elements or faces out of range add nothing. */
int32_t maille_gpu_thermal_loads(int64_t n_nodes, const double* coords, int32_t npe, int64_t n_elems,
                                 const int64_t* conn, int64_t n_sources, const int64_t* s_elem,
                                 const double* s_value, int64_t n_convection, const int64_t* c_elem,
                                 const int32_t* c_face, const double* c_film, const double* c_sink,
                                 double* f);

/* Largest n_block_rows that maille_gpu_bsr3_spmv_dot_noalloc accepts (2^26 block rows, i.e.
 * about 2e8 DOFs, inside the 32-bit column indices of the matrix). */
#define MAILLE_NOALLOC_MAX_BLOCK_ROWS (INT64_C(1) << 26)

/* No counterpart in the reference. For callers that cannot allocate device memory where they
 * need the product (code running during CUDA stream capture, plugins whose host framework owns
 * every device allocation, real-time loops): y = A x and *xy = x . y for a 3x3-block CSR matrix
 * A held by the caller on `device` -- row_ptr [n_block_rows + 1] (int64), col [blocks] (int32
 * block columns), vals [9 * blocks] (row-major blocks), x and y [3 * n_block_rows], xy [1], all
 * device pointers the caller owns -- enqueued on `stream` (cudaStream_t, NULL = the legacy
 * default stream) without waiting. x, y and xy must not overlap (an in-place product is refused
 * with MAILLE_INVALID_INPUT). It calls no cudaMalloc, cudaFree or allocating routine: the
 * reduction's partial sums and ticket live in a fixed device array inside the library (8200
 * bytes: 1024 FP64 partial sums and a 4-byte ticket, at a 256-byte boundary), shared by all
 * calls, so calls that overlap on the GPU race and must be ordered by the caller.
 * The first call on a device looks up that array's address (cudaGetSymbolAddress) with the
 * device current: make it before any stream capture. Sizes beyond
 * MAILLE_NOALLOC_MAX_BLOCK_ROWS are rejected with MAILLE_INVALID_INPUT. The current device of
 * the calling thread is restored on return. */
int32_t maille_gpu_bsr3_spmv_dot_noalloc(int32_t device, int64_t n_block_rows,
                                         const int64_t* row_ptr, const int32_t* col,
                                         const double* vals, const double* x, double* y,
                                         double* xy, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* MAILLE_GPU_H */
