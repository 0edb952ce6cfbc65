"""GPU parity of the transient heat conduction path (maille_gpu_thermal_transient) against the
oracle's restatement of Model::solve_step (model.rs:621-706), and the reference's transient
known-answer tests (tests/transient.rs) run through the GPU path.

Tolerances: the GPU and the oracle both run IC(0)-PCG to ||r|| <= 1e-12 ||b|| per increment but
with different orderings (multicolour vs RCM), so their temperatures agree to the solver
tolerance times the conditioning: 1e-9 relative to the largest temperature; reactions (sums of
element products of those temperatures) to 1e-8 of the largest reaction; Gauss-point fluxes to
1e-8 of the largest flux.
"""
import numpy as np
import pytest

from maille_b200 import meshgen as mg, thermal as th, _lib

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _check(out, ref, t_tol=1e-9, r_tol=1e-8, q_tol=1e-8):
    assert _rel(out["temps"], ref["temps"]) < t_tol, _rel(out["temps"], ref["temps"])
    assert _rel(out["reactions"], ref["reactions"]) < r_tol, _rel(out["reactions"], ref["reactions"])
    if ref["fluxes"] is not None and out["fluxes"] is not None:
        assert _rel(out["fluxes"], ref["fluxes"]) < q_tol, _rel(out["fluxes"], ref["fluxes"])


@pytest.mark.parametrize("quadratic,cells", [(False, 8), (True, 4)])
def test_transient_matches_the_oracle(gpu, oracle_lib, quadratic, cells):
    p = mg.thermal_cube(cells, quadratic, increments=4, time_period=0.04)
    ref = oracle_lib.thermal_transient(p, solver=2)
    assert ref["status"] == 0
    s, out = th.solve_problem(p, f=ref["f"])
    assert s == 0, _lib.last_error()
    _check(out, ref)
    info = out["info"]
    assert info["free_nodes"] == ref["free"]
    assert info["iterations_total"] > 0 and info["max_rel_residual"] <= 1e-12
    assert np.all(out["iterations"] > 0)


def test_crank_nicolson_with_rcm_ordering_and_no_fluxes(gpu, oracle_lib):
    p = mg.thermal_cube(6, False, increments=3, time_period=0.03, theta=0.5)
    ref = oracle_lib.thermal_transient(p, solver=2, fluxes=False)
    s, out = th.solve_problem(p, f=ref["f"], fluxes=False, ordering=_lib.MAILLE_ORDER_RCM)
    assert s == 0, _lib.last_error()
    _check(out, ref)
    assert out["info"]["levels"] > 20  # RCM: level-scheduled, many levels


def test_host_loads_and_device_path_agree_with_the_oracle_end_to_end(gpu, oracle_lib):
    # f assembled by the library's host helper (sources + convection), not taken from the oracle
    p = mg.thermal_cube(4, True, increments=2, time_period=0.05)
    ref = oracle_lib.thermal_transient(p, solver=2)
    s, out = th.solve_problem(p)
    assert s == 0, _lib.last_error()
    _check(out, ref)


def test_repeated_runs_are_bit_identical(gpu):
    p = mg.thermal_cube(5, True, increments=3, time_period=0.03)
    s1, a = th.solve_problem(p)
    s2, b = th.solve_problem(p)
    assert s1 == 0 and s2 == 0
    assert np.array_equal(a["temps"], b["temps"])
    assert np.array_equal(a["reactions"], b["reactions"])
    assert np.array_equal(a["fluxes"], b["fluxes"])


def _slab(name, nx, k=1.0):
    nodes, tets = mg.box_grid((nx, 1, 1), (1.0, 0.25, 0.25))
    conn = tets
    if name == "Tet10":
        nodes, conn = mg.to_quadratic_tet(nodes, tets)
    return nodes, conn, k


def test_quenched_slab_follows_the_fourier_series_on_the_gpu(gpu):
    # transient.rs:281-295 through the GPU path (solver tolerance 1e-12 as the reference's PCG)
    from maille_b200.thermal import Step, ThermalModel
    for name, nx in (("Tet4", 40), ("Tet10", 10)):
        nodes, conn, k = _slab(name, nx)
        ends = np.nonzero((np.abs(nodes[:, 0]) < 1e-12) | (np.abs(nodes[:, 0] - 1.0) < 1e-12))[0]
        model = ThermalModel(nodes, conn, k, 1.0, bcs=[(int(v), 100.0) for v in ends])
        hist = model.solve_step(Step.transient(0.1, 400), np.zeros(nodes.shape[0]), fluxes=False)
        n = 2 * np.arange(500) + 1.0
        for s in (80, 200, 400):
            t = hist[s].time
            exact = 100.0 * (1.0 - (4.0 / (n * np.pi) * np.sin(np.outer(nodes[:, 0], n) * np.pi)
                                    * np.exp(-(n * np.pi) ** 2 * t)).sum(axis=1))
            assert np.max(np.abs(hist[s].temperatures - exact)) / 100.0 < 4e-3


def test_energy_balance_is_exact_on_the_gpu(gpu):
    # transient.rs:445-474 (sum over increments of dt (reactions + sources) = heat stored)
    from maille_b200.thermal import HeatSource, Step, ThermalModel
    for name in ("Tet4", "Tet10"):
        nodes, conn, k = _slab(name, 4)
        left = np.nonzero(np.abs(nodes[:, 0]) < 1e-12)[0]
        model = ThermalModel(nodes, conn, k, 1.0, bcs=[(int(v), 80.0) for v in left])
        model.with_heat_sources([HeatSource(e, 50.0) for e in range(conn.shape[0])])
        step = Step.transient(0.3, 12).with_theta(0.5)
        hist = model.solve_step(step, 20.0 + 5.0 * nodes[:, 0])
        w = np.zeros(nodes.shape[0])  # rho c int N dV
        for e in conn:
            p0 = nodes[e[0]]
            vol = abs(np.dot(nodes[e[1]] - p0, np.cross(nodes[e[2]] - p0, nodes[e[3]] - p0))) / 6.0
            if conn.shape[1] == 4:
                w[e] += vol * 0.25
            else:
                w[e[:4]] += vol * -0.05
                w[e[4:]] += vol * 0.2
        stored = float(np.dot(hist[12].temperatures - hist[0].temperatures, w))
        supplied = sum(step.time_step * (h.reactions.sum() + 50.0 * 0.0625) for h in hist[1:])
        assert abs(stored - supplied) < 1e-9 * abs(stored), (stored, supplied)


def test_iteration_cap_reports_not_converged(gpu):
    p = mg.thermal_cube(4, True, increments=3, time_period=0.3)
    s, out = th.solve_problem(p, max_iter=2)
    assert s == _lib.MAILLE_NOT_CONVERGED
    assert "increment 1" in _lib.last_error()


@pytest.mark.parametrize("precision", [_lib.MAILLE_FP64, _lib.MAILLE_MIXED])
def test_full_size_transient_matches_the_oracle_summary(gpu, precision):
    # the 40^3 Tet10 workload (7.7 M lower slots, more than one thread each in any capped grid):
    # iterations per increment, reaction sums and sampled final temperatures against the
    # oracle's run (tests/golden/make_thermal_40_summary.py), in both precisions
    import json
    import os
    g = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                    "thermal_40_oracle_summary.json")))
    p = mg.thermal_cube(40, True, increments=g["increments"], time_period=g["time_period"])
    s, out = th.solve_problem(p, fluxes=False, precision=precision)
    assert s == 0, _lib.last_error()
    assert out["info"]["free_nodes"] == g["free_nodes"]
    sample = out["temps"][-1][::g["t_final_stride"]]
    assert np.max(np.abs(sample - np.array(g["t_final_sample"]))) < 1e-9 * 100.0
    sums = out["reactions"].sum(axis=1)
    assert np.max(np.abs(sums - np.array(g["reaction_sum"]))) < 1e-7 * np.max(np.abs(g["reaction_sum"]))
    assert np.allclose(out["temps"].min(axis=1), g["t_min"], rtol=0, atol=1e-9 * 100.0)
    assert np.allclose(out["temps"].max(axis=1), g["t_max"], rtol=0, atol=1e-9 * 100.0)


def test_steady_solve_matches_the_oracle_and_keeps_the_linear_field(gpu, oracle_lib):
    # Model::solve with Analysis::Thermal through ThermalModel.solve (the transient path with no
    # capacity, theta = 1, one increment), against the oracle's own steady run, and the slab
    # between two temperatures with a source (transient.rs:196-223's steady state)
    from maille_b200.thermal import HeatSource, ThermalModel
    for name in ("Tet4", "Tet10"):
        nodes, conn, k = _slab(name, 6)
        ends = [(int(v), 100.0) for v in np.nonzero(np.abs(nodes[:, 0]) < 1e-12)[0]]
        ends += [(int(v), 20.0) for v in np.nonzero(np.abs(nodes[:, 0] - 1.0) < 1e-12)[0]]
        model = ThermalModel(nodes, conn, 2.5, 1.0, bcs=ends)
        model.with_heat_sources([HeatSource(e, 300.0) for e in range(conn.shape[0])])
        inc = model.solve()
        p = mg.ThermalProblem(coords=nodes, conn=conn, conductivity=np.full(conn.shape[0], 2.5),
                              rho_c=np.zeros(conn.shape[0]), fixed=model.fixed, imposed=model.imposed,
                              loads=np.zeros(nodes.shape[0]), initial=np.zeros(nodes.shape[0]),
                              s_elem=np.arange(conn.shape[0], dtype=np.int64),
                              s_value=np.full(conn.shape[0], 300.0))
        ref = oracle_lib.thermal_transient(p, solver=1)
        assert ref["status"] == 0
        assert _rel(inc.temperatures, ref["temps"][1]) < 1e-9
        assert _rel(inc.reactions, ref["reactions"][1]) < 1e-8
        assert _rel(inc.heat_fluxes, ref["fluxes"][1]) < 1e-8
        # without the source the field is linear and the flux uniform: q = -k dT/dx = 2.5 * 80
        model.with_heat_sources([])
        lin = model.solve()
        assert np.max(np.abs(lin.temperatures - (100.0 - 80.0 * nodes[:, 0]))) < 1e-8
        assert np.max(np.abs(lin.heat_fluxes[..., 3] - 200.0)) < 1e-6


def test_steady_known_answers_of_the_reference_through_the_gpu(gpu):
    # tests/thermal.rs:424-456 (convection-cooled wall, exact) and 472-505 (thin Tet10 fin vs fin
    # theory) through ThermalModel.solve, with the convection loads from the library's helper
    import math
    from maille_b200.thermal import Convection, ThermalModel
    from test_oracle_thermal import face_positions
    K, T, L, H = 50.0, 2.0, 4.0, 1.0

    def faces(nodes, conn, on):
        return [(e, f) for e in range(conn.shape[0]) for f in range(4)
                if all(on(nodes[v]) for v in conn[e, face_positions(conn.shape[1], f)])]

    t1, h, sink = 20.0, 30.0, 300.0
    for quadratic in (False, True):
        nodes, tets = mg.box_grid((4, 1, 2), (L, H, T))
        conn = tets
        if quadratic:
            nodes, conn = mg.to_quadratic_tet(nodes, tets)
        left = np.nonzero(np.abs(nodes[:, 0]) < 1e-12)[0]
        model = ThermalModel(nodes, conn, K, 1.0, bcs=[(int(v), t1) for v in left])
        model.with_convection([Convection(e, f, h, sink)
                               for e, f in faces(nodes, conn, lambda q: abs(q[0] - L) < 1e-12)])
        inc = model.solve()
        exact = t1 + (sink - t1) * h * nodes[:, 0] / (K + h * L)
        assert np.max(np.abs(inc.temperatures - exact)) < 1e-9
        power = H * T * K * h * (sink - t1) / (K + h * L)
        assert abs(inc.reactions[left].sum() + power) < 1e-8 * power
    hf, length = 0.1, 16.0
    nodes, tets = mg.box_grid((16, 1, 1), (length, H, T))
    nodes, conn = mg.to_quadratic_tet(nodes, tets)
    side = lambda c, lim: abs(c) < 1e-12 or abs(c - lim) < 1e-12  # noqa: E731
    base = np.nonzero(np.abs(nodes[:, 0]) < 1e-12)[0]
    model = ThermalModel(nodes, conn, K, 1.0, bcs=[(int(v), 100.0) for v in base])
    model.with_convection([Convection(e, f, hf, 20.0)
                           for e, f in faces(nodes, conn, lambda q: side(q[1], H) or side(q[2], T))])
    inc = model.solve(fluxes=False)
    m = math.sqrt(hf * 2.0 * (H + T) / (K * H * T))
    exact = 20.0 + 80.0 * np.cosh(m * (length - nodes[:, 0])) / math.cosh(m * length)
    assert np.max(np.abs(inc.temperatures - exact)) / 80.0 < 0.002


def test_cancel_flag_stops_the_step(gpu, oracle_lib):
    """The observer's Flow::Stop role (solve_step_with, model.rs:628, 1203-1218): a raised flag
    stops the step before its first increment with MAILLE_CANCELLED; cleared, the same step runs
    to the oracle's history."""
    p = mg.thermal_cube(4, False, increments=3, time_period=0.03)
    ref = oracle_lib.thermal_transient(p, solver=2)
    th.cancel(True, device=0)
    try:
        s, out = th.solve_problem(p, f=ref["f"])
    finally:
        th.cancel(False, device=0)
    assert s == 5, (s, _lib.last_error())
    assert "Cancelled before increment 1" in _lib.last_error()
    assert not out["iterations"].any()
    s, out = th.solve_problem(p, f=ref["f"])
    assert s == 0, _lib.last_error()
    _check(out, ref)


def test_cancel_rejects_a_device_out_of_range(gpu):
    with pytest.raises(th.MailleError):
        th.cancel(True, device=64)


@pytest.mark.parametrize("ordering", [_lib.MAILLE_ORDER_MULTICOLOR_BFS, _lib.MAILLE_ORDER_MULTICOLOR,
                                      _lib.MAILLE_ORDER_RCM, _lib.MAILLE_ORDER_MULTICOLOR_ITERATED])
def test_device_ordering_equals_the_host_ordering(gpu, monkeypatch, ordering):
    """The thermal step orders its free nodes on the device by default; the host analysis
    (MAILLE_HOST_ORDERING=1) runs the same algorithms on the same graph: the same levels,
    iterations and temperatures bit for bit."""
    p = mg.thermal_cube(5, True, increments=2, time_period=0.02)
    monkeypatch.setenv("MAILLE_HOST_ORDERING", "1")
    s1, a = th.solve_problem(p, fluxes=False, ordering=ordering)
    monkeypatch.delenv("MAILLE_HOST_ORDERING")
    s2, b = th.solve_problem(p, fluxes=False, ordering=ordering)
    assert s1 == 0 and s2 == 0, _lib.last_error()
    assert a["info"]["levels"] == b["info"]["levels"]
    assert np.array_equal(a["iterations"], b["iterations"])
    assert np.array_equal(a["temps"], b["temps"])


@pytest.mark.parametrize("quadratic,cells", [(False, 8), (True, 4)])
def test_mixed_precision_transient_matches_the_oracle(gpu, oracle_lib, quadratic, cells):
    """The mixed form (FP32 matrices and vectors, FP64 reliable updates, the stopping test on the
    FP64 true residual) against the oracle's FP64 history, at the FP64 tolerances of this file."""
    p = mg.thermal_cube(cells, quadratic, increments=4, time_period=0.04)
    ref = oracle_lib.thermal_transient(p, solver=2)
    s, out = th.solve_problem(p, f=ref["f"], precision=_lib.MAILLE_MIXED)
    assert s == 0, _lib.last_error()
    _check(out, ref)
    assert out["info"]["max_rel_residual"] <= 1e-12
    s64, out64 = th.solve_problem(p, f=ref["f"])
    assert s64 == 0
    # the same problem in FP64 within the solver tolerance
    assert _rel(out["temps"], out64["temps"]) < 1e-10


def test_mixed_precision_iteration_cap_and_repeatability(gpu):
    p = mg.thermal_cube(6, False, increments=2, time_period=0.02)
    s, out = th.solve_problem(p, max_iter=3, precision=_lib.MAILLE_MIXED)
    assert s == _lib.MAILLE_NOT_CONVERGED and "IterativeNotConverged at increment 1" in _lib.last_error()
    s1, a = th.solve_problem(p, precision=_lib.MAILLE_MIXED)
    s2, b = th.solve_problem(p, precision=_lib.MAILLE_MIXED)
    assert s1 == 0 and s2 == 0
    assert np.array_equal(a["temps"], b["temps"])
