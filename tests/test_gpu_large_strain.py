"""GPU large-strain path (maille_gpu_large_strain_*) against the oracle: Newton histories and
reactions of every increment, the reference's uniaxial closed form, the adjoint gradient of a
reaction force against the oracle's adjoint on the same checkpoints and against central
differences of whole GPU quasi-static runs, and the full 64 x 16 x 16 workload against the
oracle's full-size summary (tests/golden/large_strain_oracle_summary.json)."""
import json
import os

import numpy as np
import pytest

import maille_b200 as mb
from maille_b200 import meshgen as mg
from maille_b200._lib import MAILLE_MIXED
from maille_b200.large_strain import from_lame

import test_oracle_large_strain as ols

pytestmark = pytest.mark.gpu

LAM = 120000.0


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_newton_history_matches_the_oracle(gpu, oracle_lib):
    p, mu, tip = mg.large_strain_block(cells=(8, 2, 2))
    with mb.LargeStrainSolver(p, increments=10, newton_tol=1e-12, tol=1e-14) as s:
        h = s.run()
    r = oracle_lib.large_strain_run(p, increments=10, newton_tol=1e-12, pcg_tol=1e-14)
    assert r["status"] == 0
    assert rel(h.displacements, r["u_hist"]) < 1e-10
    for k in range(10):
        assert rel(h.reactions[k], r["reactions"][k]) < 1e-9
    assert np.array_equal(h.cuts, r["cuts"])
    # default reference tolerances: the same Newton iteration counts
    with mb.LargeStrainSolver(p, increments=10) as s:
        d = s.run()
    r8 = oracle_lib.large_strain_run(p, increments=10)
    assert np.array_equal(d.newton, r8["newton"])
    assert rel(d.reactions[-1], r8["reactions"][-1]) < 1e-7


def test_uniaxial_tension_matches_the_closed_form(gpu):
    stretch = 2.0
    lat, sxx = ols.uniaxial_closed_form(stretch)
    p, xl = ols.tension_block()
    p.imposed[3 * np.nonzero(xl)[0]] = (stretch - 1.0) * ols.L
    with mb.LargeStrainSolver(p, increments=8) as s:
        h = s.run()
    u = h.displacements[-1].reshape(-1, 3)
    x = p.coords
    assert np.abs(u[:, 0] - (stretch - 1) * x[:, 0]).max() < 1e-6 * ols.L
    assert np.abs(u[:, 1] - (lat - 1) * x[:, 1]).max() < 1e-6 * ols.L
    force = h.reactions[-1][3 * np.nonzero(xl)[0]].sum()
    assert abs(force - sxx * lat * lat * ols.W * ols.D) < 1e-6 * sxx


def test_adjoint_matches_the_oracle_and_central_differences(gpu, oracle_lib):
    p, mu, tip = mg.large_strain_block(cells=(8, 2, 2))
    with mb.LargeStrainSolver(p, increments=10, newton_tol=1e-12, tol=1e-14) as s:
        h = s.run()
        w = np.zeros_like(h.reactions)
        w[-1, tip] = 1.0
        w[4, tip] = 0.5  # a second increment in the objective exercises the reverse pass
        gm, gl = s.backward(w)
        st, om, ol = oracle_lib.large_strain_gradient(p, h.displacements, w, pcg_tol=1e-14)
        assert st == 0
        assert rel(gm, om) < 1e-9 and rel(gl, ol) < 1e-9
        # central differences of J = R_10 + 0.5 R_5 through GPU re-runs

        def J(mu_v):
            s.set_materials(*from_lame(LAM, mu_v))
            hh = s.run()
            return hh.reactions[-1, tip].sum() + 0.5 * hh.reactions[4, tip].sum()

        for e in (0, 37, 100, 191):
            step = 1e-4 * mu[e]
            mp, mm = mu.copy(), mu.copy()
            mp[e] += step
            mm[e] -= step
            fd = (J(mp) - J(mm)) / (2 * step)
            assert abs(fd - gm[e]) <= 1e-6 * abs(gm[e]), (e, fd, gm[e])


def test_mixed_precision_inner_solves(gpu, oracle_lib):
    p, mu, tip = mg.large_strain_block(cells=(16, 4, 4))
    with mb.LargeStrainSolver(p, increments=10, precision=MAILLE_MIXED, tol=1e-11) as s:
        h = s.run()
    r = oracle_lib.large_strain_run(p, increments=10)
    assert r["status"] == 0
    assert rel(h.reactions[-1][tip], r["reactions"][-1][tip]) < 1e-7


def test_backward_needs_a_run(gpu):
    p, mu, tip = mg.large_strain_block(cells=(4, 1, 1))
    with mb.LargeStrainSolver(p, increments=2) as s:
        with pytest.raises(mb.MailleError):
            s.backward(np.zeros((2, 3 * p.n_nodes)))
        s.run()
        gm, gl = s.backward(np.zeros((2, 3 * p.n_nodes)))
        assert not gm.any() and not gl.any()


def test_full_size_block_matches_the_oracle_summary(gpu):
    path = os.path.join(os.path.dirname(__file__), "golden", "large_strain_oracle_summary.json")
    g = json.load(open(path))
    p, mu, tip = mg.large_strain_block()
    assert p.n_nodes == 18785 and p.n_elems == 98304
    with mb.LargeStrainSolver(p, increments=10) as s:
        h = s.run()
        tip_r = h.reactions[:, tip].sum(axis=1)
        assert np.allclose(tip_r, g["tip_reaction"], rtol=1e-7, atol=0)
        assert np.array_equal(h.newton, g["newton"])
        assert abs(np.linalg.norm(h.displacements[-1]) - g["u_final_norm"]) < 1e-8 * g["u_final_norm"]
        w = np.zeros_like(h.reactions)
        w[-1, tip] = 1.0
        gm, _ = s.backward(w)
    el = np.array(g["elements"])
    assert rel(gm[el], np.array(g["dJdmu"])) < 1e-6
    assert abs(gm.sum() - g["dJdmu_sum"]) < 1e-6 * abs(g["dJdmu_sum"])


def test_newton_cuts_match_the_oracle(gpu, oracle_lib):
    """A Newton limit too small for the whole increment forces advance's halvings
    (model.rs:820-870): the GPU takes the same cuts as the oracle, with the same Newton counts
    and end state."""
    p, mu, tip = mg.large_strain_block(cells=(8, 2, 2))
    for inc, nmax in ((2, 3), (10, 2)):
        r = oracle_lib.large_strain_run(p, increments=inc, newton_max=nmax)
        assert r["status"] == 0 and r["cuts"].sum() > 0
        with mb.LargeStrainSolver(p, increments=inc, newton_max=nmax) as s:
            h = s.run()
        assert np.array_equal(h.cuts, r["cuts"]), (h.cuts, r["cuts"])
        assert np.array_equal(h.newton, r["newton"])
        assert h.newton_total == r["newton_total"]
        assert rel(h.displacements, r["u_hist"]) < 1e-9
        assert rel(h.reactions[-1], r["reactions"][-1]) < 1e-7


def test_exhausted_cuts_report_not_converged(gpu, oracle_lib):
    p, mu, tip = mg.large_strain_block(cells=(8, 2, 2))
    r = oracle_lib.large_strain_run(p, increments=2, newton_max=2)
    assert r["status"] == 2 and r["stop_cuts"] == 5
    with mb.LargeStrainSolver(p, increments=2, newton_max=2) as s:
        with pytest.raises(mb.MailleError) as e:
            s.run()
    assert e.value.kind == "IterativeNotConverged" or "converge" in str(e.value)
    assert e.value.history.cuts[0] == 5


def test_inner_pcg_cap_fails_without_a_cut(gpu, oracle_lib):
    """An inner PCG at its cap is IterativeNotConverged, passed up with no halving, as in the
    reference (model.rs:839-842) and the oracle."""
    p, mu, tip = mg.large_strain_block(cells=(8, 2, 2))
    r = oracle_lib.large_strain_run(p, increments=10, pcg_max=3)
    assert r["status"] == 2 and r["stop_cuts"] == 0
    with mb.LargeStrainSolver(p, increments=10, max_iter=3) as s:
        with pytest.raises(mb.MailleError) as e:
            s.run()
    assert e.value.kind == "IterativeNotConverged"
    assert e.value.history.cuts[0] == 0
    assert e.value.history.newton_total == r["newton_total"] == 1
    assert e.value.history.pcg_total == r["pcg_total"] == 3


def test_cancel_flag_stops_the_run(gpu, oracle_lib):
    p, mu, tip = mg.large_strain_block(cells=(8, 2, 2))
    with mb.LargeStrainSolver(p, increments=4) as s:
        s.cancel(True)
        with pytest.raises(mb.MailleError) as e:
            s.run()
        assert e.value.kind == "Cancelled"
        assert e.value.history.newton_total == 0 and not e.value.history.cuts.any()
        s.cancel(False)
        h = s.run()
    r = oracle_lib.large_strain_run(p, increments=4)
    assert np.array_equal(h.newton, r["newton"])
    assert rel(h.reactions[-1], r["reactions"][-1]) < 1e-7
