"""The oracle's adjoint gradient against central finite differences (CPU, skyline solves).

The reference has no gradients, so the oracle's adjoint (K_ff lambda_f = (dJ/du)_f, then
dJ/dE_e = -lambda_e^T K_e u_e / E_e) is pinned by central differences of J through the oracle's
own direct solver. Two forms of the difference: the plain one, J(rho + h) - J(rho - h) from two
compliances (limited by cancellation, about 1e-8 of J per element here), and the same difference
written without cancellation through the identity, for J = g.u and K(+) u(+) = K(-) u(-) = f,

    J(+) - J(-) = g.(u(+) - u(-)) = -lambda(+)^T (K(+) - K(-)) u(-),   K(+) lambda(+) = g,

where K(+) - K(-) touches one element, so the right side is one element's bilinear form.
"""
import copy

import numpy as np
import pytest

from maille_b200 import meshgen as mg


def _unit_young(prob, e):
    """prob restricted to element e with E = 1 (its K_e / E_e)."""
    q = copy.copy(prob)
    q.conn = prob.conn[e:e + 1]
    q.young = np.ones(1)
    q.poisson = np.asarray(prob.poisson, np.float64).reshape(-1)[e:e + 1] \
        if np.ndim(prob.poisson) else np.full(1, float(prob.poisson))
    return q


def _with_rho(prob, rho):
    q = copy.copy(prob)
    q.young = 210000.0 * rho ** 3
    return q


def test_compliance_gradient_matches_central_differences(oracle_lib):
    p, rho = mg.simp_tet4(4)
    r = oracle_lib.model_solve(p, solver=1)
    u, f = r["u"], r["f"]
    grad_e, lam, _ = oracle_lib.adjoint_gradient(p, u, f, tol=1e-15)
    # compliance is self-adjoint: lambda = u
    assert np.linalg.norm(lam - u) <= 1e-11 * np.linalg.norm(u)
    grad = grad_e * 3 * 210000.0 * rho ** 2
    assert np.all(grad < 0)  # stiffening any element lowers the compliance
    for e in np.random.default_rng(3).choice(p.n_elems, 6, replace=False):
        h = 1e-6 * rho[e]
        sol = {}
        for s in (1, -1):
            rr = rho.copy()
            rr[e] += s * h
            sol[s] = oracle_lib.model_solve(_with_rho(p, rr), solver=1)["u"]
        plain = (f @ sol[1] - f @ sol[-1]) / (2 * h)
        assert abs(plain - grad[e]) <= 1e-4 * abs(grad[e])
        # lambda(+) = u(+) for compliance
        b = oracle_lib.element_bilinear(_unit_young(p, e), sol[1], sol[-1])[0]
        exact = -210000.0 * ((rho[e] + h) ** 3 - (rho[e] - h) ** 3) * b / (2 * h)
        assert abs(exact - grad[e]) <= 1e-6 * abs(grad[e]), (e, exact, grad[e])


def test_gradient_of_a_displacement_objective(oracle_lib):
    """J = mean z-displacement of the loaded face (not self-adjoint): lambda != u."""
    p = mg.mixed_tet10(3)
    r = oracle_lib.model_solve(p, solver=1)
    top = np.nonzero(np.abs(p.coords[:, 2] - 1.0) < 1e-12)[0]
    g = np.zeros(3 * p.n_nodes)
    g[3 * top + 2] = 1.0 / top.size
    grad, lam, _ = oracle_lib.adjoint_gradient(p, r["u"], g, tol=1e-15)
    assert np.linalg.norm(lam - r["u"]) > 1e-3 * np.linalg.norm(r["u"])
    young = np.asarray(p.young, np.float64)
    for e in np.random.default_rng(5).choice(p.n_elems, 4, replace=False):
        h = 1e-6 * young[e]
        q = copy.copy(p)
        q.young = young.copy()
        q.young[e] += h
        up = oracle_lib.model_solve(q, solver=1)["u"]
        q.young[e] -= 2 * h
        um = oracle_lib.model_solve(q, solver=1)["u"]
        q.young[e] += h
        # lambda(+) from the adjoint at E + h
        q.young[e] += h
        lp = oracle_lib.adjoint_gradient(q, up, g, tol=1e-15)[1]
        b = oracle_lib.element_bilinear(_unit_young(p, e), lp, um)[0]
        exact = -b  # (K(+) - K(-)) = 2h K_e / E_e
        assert abs(exact - grad[e]) <= 1e-6 * abs(grad[e]), (e, exact, grad[e])
        plain = (g @ up - g @ um) / (2 * h)
        assert abs(plain - grad[e]) <= 1e-3 * abs(grad[e])
