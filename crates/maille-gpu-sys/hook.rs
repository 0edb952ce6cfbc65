// hook.rs -- the maille-core side of the GPU path, a module a maintainer adds to
// crates/maille-core/src (as `mod gpu;`, behind `#[cfg(feature = "gpu")]`) and calls from
// Model::solve (model.rs:548-610) right after `let a = self.assemble()?;`:
//
//     #[cfg(feature = "gpu")]
//     if let Some(field) = gpu::try_solve(self, &a)? { return Ok(field); }
//
// It uses maille-core's own types (Model, Assembly, Field, Stress, MailleError) with the field
// names of results.rs:6-20 (Stress) and 51-76 (Field).

use maille_gpu_sys as sys;

use crate::error::MailleError;
use crate::model::{Analysis, Assembly, Kinematics, Model};
use crate::results::{Field, Stress};

fn to_maille(e: sys::GpuError) -> MailleError {
    match e {
        sys::GpuError::Singular => MailleError::Singular,
        sys::GpuError::NotConverged { iterations, residual } => {
            MailleError::IterativeNotConverged { iterations, residual }
        }
        sys::GpuError::Cancelled => MailleError::Cancelled,
        // a new variant carrying the library's message, for bad input and CUDA failures
        sys::GpuError::InvalidInput(m) | sys::GpuError::Cuda(m) => MailleError::Gpu(m),
    }
}

/// The conditions under which the iterative branch of Model::solve moves to the GPU.
fn gpu_eligible(model: &Model, a: &Assembly) -> bool {
    let free = a.fixed.iter().filter(|&&c| !c).count();
    let family = model.mesh.elements.first().map(|e| e.nodes().len());
    model.analysis == Analysis::Static
        && model.kinematics == Kinematics::Small
        && model.temperatures.is_none()
        && model.contacts.is_empty()
        && matches!(family, Some(4) | Some(10))
        && model.mesh.elements.iter().all(|e| Some(e.nodes().len()) == family)
        && model.mesh.elements.iter().all(|e| e.material().plasticity.is_none())
        && model.solver.is_iterative(free)
}

/// Some(field) when the GPU solved the model, None when the model stays on the CPU path.
pub fn try_solve(model: &Model, a: &Assembly) -> Result<Option<Field>, MailleError> {
    if !gpu_eligible(model, a) {
        return Ok(None);
    }
    let mesh = &model.mesh;
    let coords: Vec<f64> = mesh.nodes.iter().flat_map(|n| [n.x, n.y, n.z]).collect();
    let npe = mesh.elements[0].nodes().len();
    let conn: Vec<i64> = mesh.elements.iter().flat_map(|e| e.nodes().iter().map(|&n| n as i64)).collect();
    let (young, poisson): (Vec<f64>, Vec<f64>) = mesh
        .elements
        .iter()
        .map(|e| (e.material().young, e.material().poisson))
        .unzip();
    let fixed: Vec<u8> = a.fixed.iter().map(|&c| c as u8).collect();
    let problem = sys::MailleElasticProblem {
        n_nodes: mesh.nodes.len() as i64,
        coords: coords.as_ptr(),
        nodes_per_elem: npe as i32,
        n_elems: mesh.elements.len() as i64,
        conn: conn.as_ptr(),
        young: young.as_ptr(),
        poisson: poisson.as_ptr(),
        fixed: fixed.as_ptr(),
        imposed: a.imposed.as_ptr(),
        f: a.f.as_ptr(),
        rel_tol: 1e-12,   // iterative.rs:9
        max_iter: 10_000, // iterative.rs:11
        precision: sys::MAILLE_FP64,
        ordering: sys::MAILLE_ORDER_AUTO,
        device: 0,
    };
    let mut system = sys::GpuSystem::new(&problem).map_err(to_maille)?;
    let out = system.solve(None).map_err(to_maille)?;
    // 9 values per Gauss point: x, y, z, sxx, syy, szz, txy, tyz, txz; 1 (Tet4) or 4 (Tet10)
    // Gauss points per element, elements in Mesh::elements order
    let ngp = if npe == 4 { 1 } else { 4 };
    let stresses: Vec<Vec<Stress>> = out
        .gauss_stress
        .chunks_exact(9 * ngp)
        .map(|element| {
            element
                .chunks_exact(9)
                .map(|g| Stress {
                    x: g[0],
                    y: g[1],
                    z: g[2],
                    sigma_xx: g[3],
                    sigma_yy: g[4],
                    sigma_zz: g[5],
                    tau_xy: g[6],
                    tau_yz: g[7],
                    tau_xz: g[8],
                })
                .collect()
        })
        .collect();
    Ok(Some(Field {
        displacements: out.u,
        reactions: out.reactions,
        stresses,
        equivalent_plastic_strains: Vec::new(),
        temperatures: Vec::new(),
        heat_fluxes: Vec::new(),
        contact_forces: Vec::new(),
        rigid_forces: Vec::new(),
        contact_pressures: Vec::new(),
    }))
}
