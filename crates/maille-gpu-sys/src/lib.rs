//! Raw bindings to `include/maille_gpu.h` (the C ABI of libmaille_gpu) and a thin safe layer
//! for the elastic handle, the one maille-core's solve would hold where
//! `SolverKind::is_iterative` (crates/maille-core/src/solve.rs:187-195) selects the PCG path.
//!
//! Every `#[repr(C)]` struct lists the header's fields in the header's order; every function of
//! the header is declared in the `extern "C"` block. All pointers in the problem and result
//! structs are caller-owned host memory unless the header says "device".

#![allow(non_camel_case_types)]

use std::ffi::{c_char, c_void, CStr};
use std::ptr;

pub const MAILLE_OK: i32 = 0;
pub const MAILLE_SINGULAR: i32 = 1;
pub const MAILLE_NOT_CONVERGED: i32 = 2;
pub const MAILLE_INVALID_INPUT: i32 = 3;
pub const MAILLE_CUDA_ERROR: i32 = 4;
pub const MAILLE_CANCELLED: i32 = 5;

pub const MAILLE_FP64: i32 = 0;
pub const MAILLE_MIXED: i32 = 1;

pub const MAILLE_ORDER_AUTO: i32 = 0;
pub const MAILLE_ORDER_MULTICOLOR: i32 = 1;
pub const MAILLE_ORDER_RCM: i32 = 2;
pub const MAILLE_ORDER_MULTICOLOR_BFS: i32 = 3;
pub const MAILLE_ORDER_MULTICOLOR_ITERATED: i32 = 4;

pub const MAILLE_BATCH_MAX_RHS: i32 = 8;
pub const MAILLE_NOALLOC_MAX_BLOCK_ROWS: i64 = 1 << 26;

#[repr(C)]
#[derive(Clone, Copy)]
pub struct MailleElasticProblem {
    pub n_nodes: i64,
    pub coords: *const f64,
    pub nodes_per_elem: i32,
    pub n_elems: i64,
    pub conn: *const i64,
    pub young: *const f64,
    pub poisson: *const f64,
    pub fixed: *const u8,
    pub imposed: *const f64,
    pub f: *const f64,
    pub rel_tol: f64,
    pub max_iter: i32,
    pub precision: i32,
    pub ordering: i32,
    pub device: i32,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct MailleElasticResult {
    pub u: *mut f64,
    pub reactions: *mut f64,
    pub gauss_stress: *mut f64,
    pub von_mises: *mut f64,
    pub iterations: i32,
    pub outer_iterations: i32,
    pub final_rel_residual: f64,
    pub shift: f64,
    pub free_dofs: i64,
    pub block_rows: i64,
    pub blocks: i64,
    pub levels: i32,
    pub ms_setup: f64,
    pub ms_upload: f64,
    pub ms_assembly: f64,
    pub ms_factor: f64,
    pub ms_solve: f64,
    pub ms_post: f64,
    pub ms_download: f64,
    pub ms_element: f64,
    pub ms_ordering: f64,
    pub ms_symbolic: f64,
    pub ms_buffers: f64,
}

// Raw pointers have no Default: every output pointer starts null (skipped by the library).
impl Default for MailleElasticResult {
    fn default() -> Self {
        MailleElasticResult {
            u: ptr::null_mut(),
            reactions: ptr::null_mut(),
            gauss_stress: ptr::null_mut(),
            von_mises: ptr::null_mut(),
            iterations: 0,
            outer_iterations: 0,
            final_rel_residual: 0.0,
            shift: 0.0,
            free_dofs: 0,
            block_rows: 0,
            blocks: 0,
            levels: 0,
            ms_setup: 0.0,
            ms_upload: 0.0,
            ms_assembly: 0.0,
            ms_factor: 0.0,
            ms_solve: 0.0,
            ms_post: 0.0,
            ms_download: 0.0,
            ms_element: 0.0,
            ms_ordering: 0.0,
            ms_symbolic: 0.0,
            ms_buffers: 0.0,
        }
    }
}

// All-zero is a valid value of every field (null pointers, zero counts).
impl Default for MailleThermalResult {
    fn default() -> Self {
        unsafe { std::mem::zeroed() }
    }
}

impl Default for MailleLargeStrainResult {
    fn default() -> Self {
        unsafe { std::mem::zeroed() }
    }
}

impl Default for MailleBatchResult {
    fn default() -> Self {
        unsafe { std::mem::zeroed() }
    }
}

#[repr(C)]
pub struct MailleGpuHandle {
    _private: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct MailleBatchProblem {
    pub n_instances: i32,
    pub nodes_per_elem: i32,
    pub n_rhs: i32,
    pub node_offset: *const i64,
    pub elem_offset: *const i64,
    pub coords: *const f64,
    pub conn: *const i64,
    pub young: *const f64,
    pub poisson: *const f64,
    pub fixed: *const u8,
    pub imposed: *const f64,
    pub f: *const f64,
    pub rel_tol: f64,
    pub max_iter: i32,
    pub precision: i32,
    pub device: i32,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct MailleBatchResult {
    pub u: *mut f64,
    pub iterations: *mut i32,
    pub rel_residual: *mut f64,
    pub status: *mut i32,
    pub max_iterations: i32,
    pub levels: i32,
    pub free_dofs: i64,
    pub block_rows: i64,
    pub blocks: i64,
    pub lanes_per_row: i32,
    pub rhs_per_lane: i32,
    pub threads: i32,
    pub task_slices: i32,
    pub autotuned: i32,
    pub ms_setup: f64,
    pub ms_upload: f64,
    pub ms_assembly: f64,
    pub ms_factor: f64,
    pub ms_tune: f64,
    pub ms_solve: f64,
    pub ms_download: f64,
}

#[repr(C)]
pub struct MailleGpuBatch {
    _private: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct MailleLargeStrainProblem {
    pub n_nodes: i64,
    pub coords: *const f64,
    pub n_elems: i64,
    pub conn: *const i64,
    pub young: *const f64,
    pub poisson: *const f64,
    pub fixed: *const u8,
    pub imposed: *const f64,
    pub f: *const f64,
    pub increments: i32,
    pub newton_tol: f64,
    pub newton_max_iter: i32,
    pub rel_tol: f64,
    pub max_iter: i32,
    pub precision: i32,
    pub device: i32,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct MailleLargeStrainResult {
    pub u: *mut f64,
    pub reactions: *mut f64,
    pub newton_iterations: *mut i32,
    pub cuts: *mut i32,
    pub newton_total: i64,
    pub pcg_total: i64,
    pub ms_total: f64,
}

#[repr(C)]
pub struct MailleGpuLargeStrain {
    _private: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct MailleThermalProblem {
    pub n_nodes: i64,
    pub coords: *const f64,
    pub nodes_per_elem: i32,
    pub n_elems: i64,
    pub conn: *const i64,
    pub conductivity: *const f64,
    pub rho_c: *const f64,
    pub fixed: *const u8,
    pub imposed: *const f64,
    pub f: *const f64,
    pub n_convection: i64,
    pub conv_elem: *const i64,
    pub conv_face: *const i32,
    pub conv_film: *const f64,
    pub initial: *const f64,
    pub time_step: f64,
    pub theta: f64,
    pub increments: i32,
    pub rel_tol: f64,
    pub max_iter: i32,
    pub ordering: i32,
    pub device: i32,
    pub precision: i32,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct MailleThermalResult {
    pub temperatures: *mut f64,
    pub reactions: *mut f64,
    pub heat_fluxes: *mut f64,
    pub iterations: *mut i32,
    pub iterations_total: i64,
    pub max_rel_residual: f64,
    pub shift: f64,
    pub free_nodes: i64,
    pub nonzeros: i64,
    pub levels: i32,
    pub ms_setup: f64,
    pub ms_upload: f64,
    pub ms_assembly: f64,
    pub ms_factor: f64,
    pub ms_steps: f64,
    pub ms_download: f64,
}

extern "C" {
    pub fn maille_gpu_last_error() -> *const c_char;
    pub fn maille_gpu_version() -> *const c_char;
    pub fn maille_gpu_device_count() -> i32;
    pub fn maille_gpu_elastic_solve(p: *const MailleElasticProblem, r: *mut MailleElasticResult) -> i32;
    pub fn maille_gpu_create(p: *const MailleElasticProblem, out: *mut *mut MailleGpuHandle) -> i32;
    pub fn maille_gpu_solve(h: *mut MailleGpuHandle, f: *const f64, r: *mut MailleElasticResult) -> i32;
    pub fn maille_gpu_solve_device(h: *mut MailleGpuHandle, f_dev: *const f64, u_dev: *mut f64) -> i32;
    pub fn maille_gpu_backward(h: *mut MailleGpuHandle, djdu: *const f64, djde: *mut f64, lambda: *mut f64) -> i32;
    pub fn maille_gpu_refactor(h: *mut MailleGpuHandle, young: *const f64, poisson: *const f64) -> i32;
    pub fn maille_gpu_multiply(h: *mut MailleGpuHandle, x: *const f64, y: *mut f64) -> i32;
    pub fn maille_gpu_nodal_stresses(h: *mut MailleGpuHandle, stress: *mut f64, von_mises: *mut f64) -> i32;
    pub fn maille_gpu_wait_selftest(device: i32, stale: i32, timed_out: *mut i32) -> i32;
    pub fn maille_gpu_trim_memory(device: i32) -> i32;
    pub fn maille_gpu_spmv_device(h: *mut MailleGpuHandle, precision: i32, count: i32) -> i32;
    pub fn maille_gpu_kernel_launches() -> i64;
    pub fn maille_gpu_cancel(h: *mut MailleGpuHandle, flag: i32);
    pub fn maille_gpu_stream(h: *mut MailleGpuHandle) -> *mut c_void;
    pub fn maille_gpu_destroy(h: *mut MailleGpuHandle);
    pub fn maille_gpu_face_pressure_loads(
        n_nodes: i64,
        coords: *const f64,
        npe: i32,
        n_elems: i64,
        conn: *const i64,
        n_press: i64,
        p_elem: *const i64,
        p_face: *const i32,
        p_value: *const f64,
        f: *mut f64,
    ) -> i32;
    pub fn maille_gpu_batched_solve(p: *const MailleBatchProblem, r: *mut MailleBatchResult) -> i32;
    pub fn maille_gpu_batch_create(p: *const MailleBatchProblem, out: *mut *mut MailleGpuBatch) -> i32;
    pub fn maille_gpu_batch_solve(b: *mut MailleGpuBatch, f: *const f64, r: *mut MailleBatchResult) -> i32;
    pub fn maille_gpu_batch_refactor(b: *mut MailleGpuBatch, young: *const f64, poisson: *const f64) -> i32;
    pub fn maille_gpu_batch_cancel(b: *mut MailleGpuBatch, flag: i32);
    pub fn maille_gpu_batch_stream(b: *mut MailleGpuBatch) -> *mut c_void;
    pub fn maille_gpu_batch_destroy(b: *mut MailleGpuBatch);
    pub fn maille_gpu_large_strain_create(
        p: *const MailleLargeStrainProblem,
        out: *mut *mut MailleGpuLargeStrain,
    ) -> i32;
    pub fn maille_gpu_large_strain_run(s: *mut MailleGpuLargeStrain, r: *mut MailleLargeStrainResult) -> i32;
    pub fn maille_gpu_large_strain_backward(
        s: *mut MailleGpuLargeStrain,
        djdr: *const f64,
        djdmu: *mut f64,
        djdlambda: *mut f64,
    ) -> i32;
    pub fn maille_gpu_large_strain_set_materials(
        s: *mut MailleGpuLargeStrain,
        young: *const f64,
        poisson: *const f64,
    ) -> i32;
    pub fn maille_gpu_large_strain_cancel(s: *mut MailleGpuLargeStrain, flag: i32);
    pub fn maille_gpu_large_strain_destroy(s: *mut MailleGpuLargeStrain);
    pub fn maille_gpu_thermal_transient(p: *const MailleThermalProblem, r: *mut MailleThermalResult) -> i32;
    pub fn maille_gpu_thermal_cancel(device: i32, flag: i32) -> i32;
    pub fn maille_gpu_thermal_loads(
        n_nodes: i64,
        coords: *const f64,
        npe: i32,
        n_elems: i64,
        conn: *const i64,
        n_sources: i64,
        s_elem: *const i64,
        s_value: *const f64,
        n_convection: i64,
        c_elem: *const i64,
        c_face: *const i32,
        c_film: *const f64,
        c_sink: *const f64,
        f: *mut f64,
    ) -> i32;
    pub fn maille_gpu_bsr3_spmv_dot_noalloc(
        device: i32,
        n_block_rows: i64,
        row_ptr: *const i64,
        col: *const i32,
        vals: *const f64,
        x: *const f64,
        y: *mut f64,
        xy: *mut f64,
        stream: *mut c_void,
    ) -> i32;
}

/// The calling thread's last error message.
pub fn last_error() -> String {
    unsafe {
        let p = maille_gpu_last_error();
        if p.is_null() {
            String::new()
        } else {
            CStr::from_ptr(p).to_string_lossy().into_owned()
        }
    }
}

/// A failed call, by MailleStatus. maille-core maps these to MailleError: Singular
/// (error.rs:224), IterativeNotConverged { iterations, residual } (error.rs:226-229), Cancelled
/// (error.rs:156); input and CUDA errors carry the library's message.
#[derive(Debug, Clone, PartialEq)]
pub enum GpuError {
    Singular,
    NotConverged { iterations: usize, residual: f64 },
    InvalidInput(String),
    Cuda(String),
    Cancelled,
}

/// MailleStatus -> Result; `r` supplies the iteration count and residual of a capped solve.
pub fn check(code: i32, r: Option<&MailleElasticResult>) -> Result<(), GpuError> {
    match code {
        MAILLE_OK => Ok(()),
        MAILLE_SINGULAR => Err(GpuError::Singular),
        MAILLE_NOT_CONVERGED => Err(GpuError::NotConverged {
            iterations: r.map_or(0, |r| r.iterations as usize),
            residual: r.map_or(0.0, |r| r.final_rel_residual),
        }),
        MAILLE_CANCELLED => Err(GpuError::Cancelled),
        MAILLE_INVALID_INPUT => Err(GpuError::InvalidInput(last_error())),
        _ => Err(GpuError::Cuda(last_error())),
    }
}

/// The outputs of one elastic solve, in the layout of maille-core's Field
/// (crates/maille-core/src/results.rs:51-76): u and reactions per DOF, per Gauss point
/// x, y, z, sxx, syy, szz, txy, tyz, txz and the von Mises value.
#[derive(Debug, Clone, Default)]
pub struct ElasticOutput {
    pub u: Vec<f64>,
    pub reactions: Vec<f64>,
    pub gauss_stress: Vec<f64>,
    pub von_mises: Vec<f64>,
    pub iterations: usize,
    pub shift: f64,
}

/// One analysed and factorised free system on the GPU (FreeSystem's role, model.rs:1442-1516):
/// create once, solve many load vectors, backward for gradients. Send but not Sync: one thread
/// at a time, which matches maille-gui's worker thread (crates/maille-gui/src/compute.rs:134).
pub struct GpuSystem {
    h: *mut MailleGpuHandle,
    n_dofs: usize,
    n_gauss: usize,
}

unsafe impl Send for GpuSystem {}

impl GpuSystem {
    /// Symbolic analysis, upload, element integration, assembly and IC(0) (the shift ladder of
    /// Pcg::new, iterative.rs:201-207). The problem's arrays are read during the call only.
    pub fn new(problem: &MailleElasticProblem) -> Result<GpuSystem, GpuError> {
        let mut h = ptr::null_mut();
        check(unsafe { maille_gpu_create(problem, &mut h) }, None)?;
        let ngp = if problem.nodes_per_elem == 4 { 1 } else { 4 };
        Ok(GpuSystem { h, n_dofs: 3 * problem.n_nodes as usize, n_gauss: ngp * problem.n_elems as usize })
    }

    /// K_ff u_f = F_f - K_fc u_c for `f` (None: the problem's loads), then reactions and stresses.
    pub fn solve(&mut self, f: Option<&[f64]>) -> Result<ElasticOutput, GpuError> {
        if let Some(f) = f {
            if f.len() != self.n_dofs {
                return Err(GpuError::InvalidInput(format!("{} loads for {} DOFs", f.len(), self.n_dofs)));
            }
        }
        let mut out = ElasticOutput {
            u: vec![0.0; self.n_dofs],
            reactions: vec![0.0; self.n_dofs],
            gauss_stress: vec![0.0; 9 * self.n_gauss],
            von_mises: vec![0.0; self.n_gauss],
            ..Default::default()
        };
        let mut r = MailleElasticResult {
            u: out.u.as_mut_ptr(),
            reactions: out.reactions.as_mut_ptr(),
            gauss_stress: out.gauss_stress.as_mut_ptr(),
            von_mises: out.von_mises.as_mut_ptr(),
            ..Default::default()
        };
        let fp = f.map_or(ptr::null(), |f| f.as_ptr());
        check(unsafe { maille_gpu_solve(self.h, fp, &mut r) }, Some(&r))?;
        out.iterations = r.iterations as usize;
        out.shift = r.shift;
        Ok(out)
    }

    /// dJ/dE per element for J with gradient dJdu at the last solve's displacements.
    pub fn backward(&mut self, djdu: &[f64], n_elems: usize) -> Result<Vec<f64>, GpuError> {
        let mut g = vec![0.0; n_elems];
        check(unsafe { maille_gpu_backward(self.h, djdu.as_ptr(), g.as_mut_ptr(), ptr::null_mut()) }, None)?;
        Ok(g)
    }

    /// The observer's Flow::Stop (model.rs:1203-1218): safe from another thread while a solve runs.
    pub fn canceller(&self) -> Canceller {
        Canceller(self.h)
    }
}

impl Drop for GpuSystem {
    fn drop(&mut self) {
        unsafe { maille_gpu_destroy(self.h) }
    }
}

/// Raises or clears a GpuSystem's cancel flag from any thread; valid while the GpuSystem lives.
#[derive(Clone, Copy)]
pub struct Canceller(*mut MailleGpuHandle);

unsafe impl Send for Canceller {}
unsafe impl Sync for Canceller {}

impl Canceller {
    pub fn set(&self, flag: bool) {
        unsafe { maille_gpu_cancel(self.0, flag as i32) }
    }
}
