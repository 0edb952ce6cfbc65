"""Runs the CPU oracle on the full mixed-precision benchmark workload (Tet10 40^3 unit cube,
lognormal E, 1 574 640 free DOF) and records a small summary: iteration counts and timings at
the given tolerance, the compliance f.u, norms, and the displacements at 2000 seeded DOFs and
the von Mises values at 500 seeded Gauss points. The GPU tests compare full-size GPU solves
with these samples without shipping the 12.7 MB solution.

    python tests/golden/make_tet10_40_summary.py 1e-13     (about 5-10 minutes on one core)
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from maille_b200 import meshgen as mg  # noqa: E402


def main(tol):
    p = mg.mixed_tet10(40)
    r = oracle.model_solve(p, solver=2, tol=tol)
    assert r["status"] == 0, r["status"]
    rng = np.random.default_rng(40)
    dofs = np.sort(rng.choice(np.nonzero(p.fixed == 0)[0], 2000, replace=False))
    gps = np.sort(rng.choice(r["von_mises"].size, 500, replace=False))
    out = dict(workload="tet10_40^3_lognormal", tol=tol, iterations=r["iterations"],
               rel_residual=r["rel_residual"], free_dofs=r["free_dofs"],
               compliance=float(r["f"] @ r["u"]), u_norm=float(np.linalg.norm(r["u"])),
               vm_norm=float(np.linalg.norm(r["von_mises"])),
               reaction_z=float(r["reactions"][2::3].sum()), ms_setup=r["ms_setup"],
               ms_factor=r["ms_factor"], ms_solve=r["ms_solve"], dofs=dofs.tolist(),
               u=r["u"][dofs].tolist(), gauss_points=gps.tolist(),
               von_mises=r["von_mises"].ravel()[gps].tolist())
    path = os.path.join(HERE, f"tet10_40_oracle_tol{tol:.0e}.json")
    json.dump(out, open(path, "w"))
    print(path, r["iterations"], r["ms_setup"], r["ms_factor"], r["ms_solve"])


if __name__ == "__main__":
    main(float(sys.argv[1]) if len(sys.argv) > 1 else 1e-13)
