"""GPU adjoint (SolverHandle.backward -> maille_gpu_backward) against the oracle's CPU FP64
adjoint and against central finite differences through GPU re-solves.

The differences use the cancellation-free identity of tests/test_oracle_adjoint.py: for J = g.u
with K(+) u(+) = K(-) u(-) = f and K(+) lambda(+) = g,
    J(+) - J(-) = -lambda(+)^T (K(+) - K(-)) u(-),
with u(+-) and lambda(+) from GPU solves after maille_gpu_refactor with the perturbed material;
K(+) - K(-) touches one element, whose unit-E matrix comes from the oracle (the checker).
Tolerances: the gradient within 1e-9 relative L2 of the oracle's (FP64, both converged to
1e-13), 1e-7 for the mixed form; finite differences within 1e-6 (relative step 1e-6).
"""
import copy
import json
import os

import numpy as np
import pytest

import maille_b200 as mb
from maille_b200 import meshgen as mg
from maille_b200._lib import MAILLE_FP64, MAILLE_MIXED, MAILLE_ORDER_MULTICOLOR

pytestmark = pytest.mark.gpu

E0 = 210000.0


def handle_of(p, tol=1e-13, precision=MAILLE_FP64):
    m = mb.Model.from_arrays(p.coords, p.conn, p.young, p.poisson, p.fixed, p.imposed, p.loads,
                             (p.p_elem, p.p_face, p.p_value))
    m.with_solver(mb.SolverKind.ITERATIVE).with_tolerance(tol).with_precision(precision)
    m.ordering = MAILLE_ORDER_MULTICOLOR
    m.max_iterations = 20000
    return mb.SolverHandle(m)


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def unit_young(prob, e):
    q = copy.copy(prob)
    q.conn = prob.conn[e:e + 1]
    q.young = np.ones(1)
    q.poisson = np.full(1, float(np.broadcast_to(prob.poisson, (prob.n_elems,))[e]))
    return q


def compliance_fd(oracle_lib, h, p, rho, elements):
    """Central differences of J = f.u in rho_e through GPU refactor + solve (exact form)."""
    out = []
    for e in elements:
        step = 1e-6 * rho[e]
        sol = {}
        for s in (1, -1):
            rr = rho.copy()
            rr[e] += s * step
            h.refactor(young=E0 * rr ** 3)
            sol[s] = h.solve().displacements
        b = oracle_lib.element_bilinear(unit_young(p, e), sol[1], sol[-1])[0]
        out.append(-E0 * ((rho[e] + step) ** 3 - (rho[e] - step) ** 3) * b / (2 * step))
    h.refactor(young=E0 * rho ** 3)
    return np.array(out)


def test_compliance_gradient_matches_the_oracle(gpu, oracle_lib):
    p, rho = mg.simp_tet4(8)
    h = handle_of(p)
    try:
        fld = h.solve()
        f = h._f
        dJdE, lam = h.backward(f)
    finally:
        h.close()
    r = oracle_lib.model_solve(p, solver=2, tol=1e-13)
    assert rel(fld.displacements, r["u"]) < 1e-10
    g_ref, lam_ref, _ = oracle_lib.adjoint_gradient(p, r["u"], r["f"], tol=1e-13)
    assert rel(dJdE, g_ref) < 1e-9
    assert rel(lam, lam_ref) < 1e-10
    assert rel(lam, fld.displacements) < 1e-10  # compliance is self-adjoint
    assert np.all(dJdE < 0)


def test_displacement_objective_gradient_tet10(gpu, oracle_lib):
    """J = mean z-displacement of the loaded face on a lognormal Tet10 cube (lambda != u)."""
    p = mg.mixed_tet10(4)
    top = np.nonzero(np.abs(p.coords[:, 2] - 1.0) < 1e-12)[0]
    g = np.zeros(3 * p.n_nodes)
    g[3 * top + 2] = 1.0 / top.size
    h = handle_of(p)
    try:
        fld = h.solve()
        dJdE, lam = h.backward(g)
        # a second backward with the same g gives bit-identical results (deterministic adjoint)
        dJdE2, lam2 = h.backward(g)
    finally:
        h.close()
    assert np.array_equal(dJdE, dJdE2) and np.array_equal(lam, lam2)
    r = oracle_lib.model_solve(p, solver=2, tol=1e-13)
    g_ref, lam_ref, _ = oracle_lib.adjoint_gradient(p, r["u"], g, tol=1e-13)
    assert rel(lam, lam_ref) < 1e-10
    assert rel(dJdE, g_ref) < 1e-9
    assert np.all(lam[np.nonzero(p.fixed)[0]] == 0.0)


def test_compliance_gradient_agrees_with_central_differences(gpu, oracle_lib):
    p, rho = mg.simp_tet4(8)
    h = handle_of(p)
    try:
        h.solve()
        dJdE, _ = h.backward(h._f)
        grad = dJdE * 3 * E0 * rho ** 2
        el = np.random.default_rng(8).choice(p.n_elems, 16, replace=False)
        fd = compliance_fd(oracle_lib, h, p, rho, el)
    finally:
        h.close()
    err = np.abs(fd - grad[el]) / np.abs(grad[el])
    assert err.max() <= 1e-6, err


def test_mixed_precision_gradient(gpu, oracle_lib):
    p, rho = mg.simp_tet4(8)
    h = handle_of(p, tol=1e-11, precision=MAILLE_MIXED)
    try:
        h.solve()
        dJdE, _ = h.backward(h._f)
    finally:
        h.close()
    r = oracle_lib.model_solve(p, solver=2, tol=1e-13)
    g_ref = oracle_lib.adjoint_gradient(p, r["u"], r["f"], tol=1e-13)[0]
    assert rel(dJdE, g_ref) < 1e-7


def test_backward_needs_a_solve_and_finite_input(gpu):
    p, _ = mg.simp_tet4(3)
    h = handle_of(p)
    try:
        with pytest.raises(mb.MailleError):
            h.backward(np.zeros(3 * p.n_nodes))
        h.solve()
        g = np.zeros(3 * p.n_nodes)
        g[5] = np.nan
        with pytest.raises(mb.MailleError):
            h.backward(g)
        # a zero objective has a zero gradient
        dJdE, lam = h.backward(np.zeros(3 * p.n_nodes))
        assert not dJdE.any() and not lam.any()
    finally:
        h.close()


def test_full_size_simp48_gradient(gpu, oracle_lib):
    """Tet4 48^3 SIMP compliance (345 744 free DOF, 663 552 elements): the gradient against the
    oracle's full-size adjoint (tests/golden/simp48_oracle_gradient.json: 64 seeded elements and
    the sum and norm of the whole gradient), and central differences on the same 64 elements."""
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "simp48_oracle_gradient.json")))
    p, rho = mg.simp_tet4(48)
    h = handle_of(p)
    try:
        fld = h.solve()
        assert fld.info["free_dofs"] == g["free_dofs"] == 345744
        J = float(h._f @ fld.displacements)
        assert abs(J - g["compliance"]) <= 1e-11 * g["compliance"]
        dJdE, _ = h.backward(h._f)
        grad = dJdE * 3 * E0 * rho ** 2
        el = np.array(g["elements"])
        assert rel(grad[el], np.array(g["grad"])) < 1e-9
        assert abs(grad.sum() - g["grad_sum"]) <= 1e-9 * abs(g["grad_sum"])
        assert abs(np.linalg.norm(grad) - g["grad_norm"]) <= 1e-9 * g["grad_norm"]
        fd = compliance_fd(oracle_lib, h, p, rho, el)
    finally:
        h.close()
    err = np.abs(fd - grad[el]) / np.abs(grad[el])
    assert err.max() <= 1e-6, err
