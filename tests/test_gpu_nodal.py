"""GPU nodal stress smoothing (nodal_stresses / smooth, results.rs:137-230) against the oracle.

The kernel accumulates each node's extrapolated Gauss values in element order with separately
rounded products and sums, like the reference's sequential loop, so on the same Gauss values it
must equal the oracle's smoothing bit for bit; against the oracle's own solve the nodal values
carry the solve's 1e-10 parity.
"""
import numpy as np
import pytest

import cases
import maille_b200 as mb
from maille_b200 import meshgen as mg
from maille_b200._lib import MAILLE_FP64

pytestmark = pytest.mark.gpu


def handle_of(p, tol=1e-12):
    m = mb.Model.from_arrays(p.coords, p.conn, p.young, p.poisson, p.fixed, p.imposed, p.loads,
                             (p.p_elem, p.p_face, p.p_value))
    m.with_solver(mb.SolverKind.ITERATIVE).with_tolerance(tol).with_precision(MAILLE_FP64)
    return mb.SolverHandle(m)


def records(stress6):
    """(n, 6) sxx syy szz txy tyz txz -> the oracle's 9-value stress records."""
    r = np.zeros((stress6.shape[0], 9))
    r[:, 3:] = stress6
    return r


@pytest.mark.parametrize("mesh", ["tet4", "tet10"])
def test_nodal_stresses_equal_the_oracle_smoothing_of_the_same_gauss_values(gpu, oracle_lib, mesh):
    p = mg.plain_tet4(8) if mesh == "tet4" else mg.mixed_tet10(5)
    h = handle_of(p)
    try:
        f = h.solve()
        stress, vm = h.nodal_stresses()
    finally:
        h.close()
    ref = oracle_lib.nodal_stresses(p, f.stresses)
    assert np.array_equal(stress, ref)
    ref_vm = np.array([oracle_lib.von_mises(r) for r in records(ref)])
    assert np.array_equal(vm, ref_vm)


def test_nodal_stresses_of_the_plain_config_match_the_oracle_solve(gpu, oracle_lib):
    # Tet4 20^3 plain configuration: nodal values within the solve's 1e-10 relative L2
    p = mg.plain_tet4(20)
    h = handle_of(p)
    try:
        h.solve()
        stress, vm = h.nodal_stresses()
    finally:
        h.close()
    r = oracle_lib.model_solve(p, solver=2, tol=1e-12)
    ref = oracle_lib.nodal_stresses(p, r["gauss"])
    ref_vm = np.array([oracle_lib.von_mises(x) for x in records(ref)])
    assert np.linalg.norm(stress - ref) / np.linalg.norm(ref) < 1e-10
    assert np.linalg.norm(vm - ref_vm) / np.linalg.norm(ref_vm) < 1e-10


@pytest.mark.parametrize("quadratic", [False, True])
def test_nodal_stresses_of_the_uniform_strain_patch_are_exact(gpu, quadratic):
    # tests/solid.rs:52-116 carried to the nodes: a uniform stress extrapolates and averages to itself
    p = cases.patch(quadratic)
    h = handle_of(p)
    try:
        h.solve()
        stress, _ = h.nodal_stresses()
    finally:
        h.close()
    sigma = cases.d_matrix() @ cases.EPS  # xx yy zz yz xz xy
    expect = np.array([sigma[0], sigma[1], sigma[2], sigma[5], sigma[3], sigma[4]])
    assert np.abs(stress - expect).max() <= 1e-9 * np.abs(sigma).max()


def test_nodal_stresses_need_a_solve(gpu):
    p = mg.plain_tet4(4)
    h = handle_of(p)
    try:
        with pytest.raises(mb.MailleError):
            h.nodal_stresses()
    finally:
        h.close()
