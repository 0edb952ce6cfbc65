"""Runs the CPU oracle on the full adjoint-compliance workload (Tet4 48^3 unit cube, SIMP
densities rho_e ~ U[0.01, 1], E_e = 210000 rho_e^3, 345 744 free DOF) and records a small
summary: the compliance J = f.u, the oracle's adjoint gradient dJ/drho_e on 64 seeded elements
(the elements the finite-difference check uses), and the sum, norm and extreme values of the
whole gradient. The GPU tests compare the full-size GPU backward() with these values.

    python tests/golden/make_simp48_gradient.py      (about a minute on one core)
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from maille_b200 import meshgen as mg  # noqa: E402

TOL = 1e-13


def fd_elements(n_elems, count=64):
    """The seeded elements of the finite-difference check."""
    return np.sort(np.random.default_rng(48).choice(n_elems, count, replace=False))


def main():
    p, rho = mg.simp_tet4(48)
    r = oracle.model_solve(p, solver=2, tol=TOL)
    assert r["status"] == 0, r["status"]
    u, f = r["u"], r["f"]
    grad_e, lam, adj = oracle.adjoint_gradient(p, u, f, tol=TOL)
    assert adj["status"] == 0, adj["status"]
    grad = grad_e * 3.0 * 210000.0 * rho ** 2  # dJ/drho_e = dJ/dE_e dE_e/drho_e
    el = fd_elements(p.n_elems)
    out = dict(workload="simp_tet4_48^3", tol=TOL, iterations=r["iterations"],
               adjoint_iterations=adj["iterations"], free_dofs=r["free_dofs"],
               compliance=float(f @ u), lambda_minus_u=float(np.linalg.norm(lam - u) / np.linalg.norm(u)),
               grad_sum=float(grad.sum()), grad_norm=float(np.linalg.norm(grad)),
               grad_min=float(grad.min()), grad_max=float(grad.max()),
               elements=el.tolist(), rho=rho[el].tolist(), grad=grad[el].tolist(),
               ms_setup=r["ms_setup"], ms_factor=r["ms_factor"], ms_solve=r["ms_solve"])
    path = os.path.join(HERE, "simp48_oracle_gradient.json")
    json.dump(out, open(path, "w"))
    print(path, r["iterations"], adj["iterations"], r["ms_solve"], out["compliance"], out["grad_sum"])


if __name__ == "__main__":
    main()
