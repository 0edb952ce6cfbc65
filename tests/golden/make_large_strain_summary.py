"""Runs the CPU oracle on the full large-strain workload (neo-Hookean Tet4 block 4 x 1 x 1 mm,
64 x 16 x 16 cells x 6 tets, mu_e ~ U[60000, 100000] seeded, lambda = 120000, x = 0 clamped, tip
z displacement -0.4 mm over 10 increments, Newton to 1e-8 with IC(0)-PCG inner solves) and
records a small summary: per increment the Newton iterations and the tip reaction force, the
final tip displacement norm, and the adjoint gradient of the final tip reaction force with
respect to mu_e on 64 seeded elements plus the sum and norm of the whole gradient.

    python tests/golden/make_large_strain_summary.py      (several minutes on one core)
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from maille_b200 import meshgen as mg  # noqa: E402


def sample_elements(n_elems, count=64):
    return np.sort(np.random.default_rng(5).choice(n_elems, count, replace=False))


def main():
    p, mu, tip = mg.large_strain_block()
    r = oracle.large_strain_run(p, increments=10)
    assert r["status"] == 0, r["status"]
    W = np.zeros_like(r["reactions"])
    W[-1, tip] = 1.0  # J = final tip reaction force (z)
    s, gmu, glam = oracle.large_strain_gradient(p, r["u_hist"], W)
    assert s == 0, s
    el = sample_elements(p.n_elems)
    out = dict(workload="neo_hookean_tet4_64x16x16", increments=10, newton=r["newton"].tolist(),
               cuts=r["cuts"].tolist(), newton_total=r["newton_total"], pcg_total=r["pcg_total"],
               tip_reaction=r["reactions"][:, tip].sum(axis=1).tolist(),
               u_final_norm=float(np.linalg.norm(r["u_hist"][-1])),
               u_final_sample=r["u_hist"][-1][::997].tolist(),
               elements=el.tolist(), dJdmu=gmu[el].tolist(), dJdmu_sum=float(gmu.sum()),
               dJdmu_norm=float(np.linalg.norm(gmu)), wall_s=r["wall_s"])
    path = os.path.join(HERE, "large_strain_oracle_summary.json")
    json.dump(out, open(path, "w"))
    print(path, r["newton"], r["pcg_total"], r["wall_s"], out["tip_reaction"][-1], out["dJdmu_sum"])


if __name__ == "__main__":
    main()
