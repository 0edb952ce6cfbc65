"""Runs the CPU oracle on the full transient thermal workload (Tet10 unit cube 40^3 x 6 tets,
531 441 nodes, conductivity lognormal seeded, rho c = 1, T = 100 on z = 0, convection h = 10 to
20 on z = 1, a source of 50 in every element, T = 20 at t = 0, 10 backward-Euler increments over
0.1, IC(0)-PCG to 1e-12) and records a small summary: the PCG iterations per increment, the sum
of the reactions and the extreme temperatures of every increment, the final temperatures on every
997th node, and the oracle's wall time.

    python tests/golden/make_thermal_40_summary.py      (about a minute on one core)
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from maille_b200 import meshgen as mg  # noqa: E402


def main():
    p = mg.thermal_cube(40, True, increments=10, time_period=0.1)
    r = oracle.thermal_transient(p, solver=2, fluxes=False)
    assert r["status"] == 0, r["status"]
    out = dict(workload=p.name, increments=p.increments, time_period=p.time_period, theta=p.theta,
               free_nodes=r["free"], iterations=r["iterations"].tolist(),
               total_iterations=r["total_iterations"],
               reaction_sum=r["reactions"].sum(axis=1).tolist(),
               t_min=r["temps"].min(axis=1).tolist(), t_max=r["temps"].max(axis=1).tolist(),
               t_final_stride=997, t_final_sample=r["temps"][-1][::997].tolist(),
               wall_s=r["wall_s"], ms_setup=r["ms_setup"], ms_factor=r["ms_factor"],
               ms_steps=r["ms_steps"])
    with open(os.path.join(HERE, "thermal_40_oracle_summary.json"), "w") as fh:
        json.dump(out, fh)


if __name__ == "__main__":
    main()
