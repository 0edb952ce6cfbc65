"""Pins the oracle's transient heat conduction (the theta-method of Model::solve_step,
model.rs:621-706) to the reference's own known-answer tests (CPU only).

The transient tests restate tests/transient.rs of the reference (crate maille-core) on its Tet4
and Tet10 meshes: the same slab L x H x THICKNESS, material (k = 1, rho = 2, c = 0.5, so the
diffusivity is 1), boundary conditions, steps and tolerances, checked against the same analytic
solutions (Fourier series of the quenched slab, Heisler series, the amplification factor of the
theta-method, exact energy balance). The steady tests restate tests/thermal.rs (imposed-
temperature wall, uniform source, convection-cooled wall, thin fin) on the oracle's steady run
(the step with no capacity, theta = 1, one increment). The quadrature and capacity tests
restate quadrature.rs:240-272 and assembly.rs:880-977.
"""
import math

import numpy as np
import pytest

from maille_b200 import meshgen as mg

K, RHO, C, L, H, THICKNESS = 1.0, 2.0, 0.5, 1.0, 0.25, 0.25
VOLUME = L * H * THICKNESS


def slab(name, nx, k=K):
    nodes, tets = mg.box_grid((nx, 1, 1), (L, H, THICKNESS))
    conn = tets
    if name == "Tet10":
        nodes, conn = mg.to_quadratic_tet(nodes, tets)
    return nodes, conn, k


def problem(mesh, bcs=(), sources=0.0, convection=None, initial=0.0, period=1.0, steps=1, theta=1.0,
            rho_c=RHO * C):
    nodes, conn, k = mesh
    n, ne = nodes.shape[0], conn.shape[0]
    fixed = np.zeros(n, np.uint8)
    imposed = np.zeros(n)
    for x, value in bcs:
        on = np.abs(nodes[:, 0] - x) < 1e-12
        fixed[on] = 1
        imposed[on] = value
    p = mg.ThermalProblem(coords=nodes, conn=conn, conductivity=np.full(ne, k),
                          rho_c=np.full(ne, rho_c), fixed=fixed, imposed=imposed,
                          loads=np.zeros(n), initial=np.broadcast_to(np.asarray(initial, float), (n,)).copy(),
                          time_period=period, increments=steps, theta=theta)
    if sources:
        p.s_elem = np.arange(ne, dtype=np.int64)
        p.s_value = np.full(ne, float(sources))
    if convection is not None:
        x, film, sink = convection
        ce, cf = mg.faces_on(nodes, conn, 0, x)
        p.c_elem, p.c_face = ce, cf
        p.c_film = np.full(ce.size, film)
        p.c_sink = np.full(ce.size, sink)
    return p


def steady(oracle_lib, p):
    """Model::solve of the thermal model: the oracle's run with rho_c = 0, theta = 1, one step."""
    q = mg.ThermalProblem(**{**p.__dict__, "rho_c": np.zeros_like(p.rho_c), "theta": 1.0,
                             "increments": 1, "time_period": 1.0})
    out = oracle_lib.thermal_transient(q)
    assert out["status"] == 0
    return out["temps"][1], out["reactions"][1]


def weights(mesh):
    """rho c int N_i dV per node (transient.rs:138-170): V/4 at Tet4 vertices; -V/20 at Tet10
    vertices and V/5 at mid-edge nodes."""
    nodes, conn, _ = mesh
    w = np.zeros(nodes.shape[0])
    for e in conn:
        p0 = nodes[e[0]]
        vol = abs(np.dot(nodes[e[1]] - p0, np.cross(nodes[e[2]] - p0, nodes[e[3]] - p0))) / 6.0
        if conn.shape[1] == 4:
            w[e] += RHO * C * vol * 0.25
        else:
            w[e[:4]] += RHO * C * vol * -0.05
            w[e[4:]] += RHO * C * vol * 0.2
    return w


def mean(temps, w):
    return float(np.dot(temps, w)) / (RHO * C * VOLUME)


# --- quadrature.rs:240-272 and assembly.rs:880-977 ---------------------------------------------

def test_tetra14_is_exact_to_degree_five_with_positive_weights(oracle_lib):
    rule = oracle_lib.tetra14()
    assert np.all(rule[:, 3] > 0.0)
    for a in range(6):
        for b in range(6 - a):
            for c in range(6 - a - b):
                got = float(np.sum(rule[:, 3] * rule[:, 0] ** a * rule[:, 1] ** b * rule[:, 2] ** c))
                exact = math.factorial(a) * math.factorial(b) * math.factorial(c) / math.factorial(a + b + c + 3)
                assert abs(got - exact) < 1e-15, (a, b, c)
    got6 = float(np.sum(rule[:, 3] * rule[:, 0] ** 6))
    assert abs(got6 - math.factorial(6) / math.factorial(9)) > 1e-7


def _h(p, c):
    """complete homogeneous symmetric polynomial h_p(c_1..c_4)"""
    total = 0.0
    for a in range(p + 1):
        for b in range(p + 1 - a):
            for d in range(p + 1 - a - b):
                e = p - a - b - d
                total += c[0] ** a * c[1] ** b * c[2] ** d * c[3] ** e
    return total


@pytest.mark.parametrize("npe", [4, 10])
def test_capacity_matrices_are_exact(oracle_lib, npe):
    # the tetrahedron of assembly.rs:962-975 (volume 1); integral of (sum c_k lambda_k)^p over it
    # is 6 V p! / (p + 3)! h_p(c)
    tet = np.array([[0.0, 0, 0], [2, 0, 0], [0, 3, 0], [0, 0, 1]])
    coords = tet if npe == 4 else np.concatenate([tet, (tet[mg.TET10_EDGES[:, 0]] + tet[mg.TET10_EDGES[:, 1]]) / 2])
    rho_c = 1.7
    ke, ce = oracle_lib.thermal_element(coords, 1.3, rho_c)
    volume = 1.0
    assert abs(ce.sum() - rho_c * volume) < 1e-13 * volume
    assert np.allclose(ce, ce.T, rtol=0, atol=1e-15)
    corners = np.array([0.3, -1.1, 2.0, 0.7])      # a linear field s by its vertex values
    lam = np.linalg.solve(np.c_[tet, np.ones(4)].T, np.r_[coords.T, np.ones((1, npe))])  # (4, npe)
    lin = corners @ lam
    power = 1 if npe == 4 else 2                  # s = lin (Tet4) or lin^2 (Tet10), interpolated exactly
    s = lin ** power
    energy = float(s @ ce @ s)
    p = 2 * power
    expected = rho_c * 6.0 * volume * math.factorial(p) / math.factorial(p + 3) * _h(p, corners)
    assert abs(energy - expected) < 1e-12 * expected
    # conduction: a constant field carries no heat, K is symmetric
    assert np.allclose(ke.sum(axis=1), 0.0, atol=1e-13)
    assert np.allclose(ke, ke.T, rtol=0, atol=1e-15)


# --- tests/transient.rs ---------------------------------------------------------------------------

def test_increments_start_from_the_initial_field_at_regular_times(oracle_lib):
    # transient.rs:172-194 (on the Tet4 slab)
    mesh = slab("Tet4", 4)
    nodes = mesh[0]
    p = problem(mesh, bcs=[(0.0, 30.0)], initial=10.0 * nodes[:, 0], period=0.5, steps=4)
    assert abs(p.time_step - 0.125) < 1e-15
    out = oracle_lib.thermal_transient(p)
    assert out["status"] == 0
    assert out["temps"].shape == (5, nodes.shape[0])
    expected = np.where(np.abs(nodes[:, 0]) < 1e-12, 30.0, 10.0 * nodes[:, 0])
    assert np.all(np.abs(out["temps"][0] - expected) < 1e-15)
    assert np.all(np.abs(out["reactions"][0]) < 1e-15)


@pytest.mark.parametrize("name", ["Tet4", "Tet10"])
def test_starting_from_the_steady_state_stays_there(oracle_lib, name):
    # transient.rs:196-223
    mesh = slab(name, 4)
    base = problem(mesh, bcs=[(0.0, 100.0), (L, 20.0)], sources=300.0)
    t_ss, r_ss = steady(oracle_lib, base)
    p = problem(mesh, bcs=[(0.0, 100.0), (L, 20.0)], sources=300.0, initial=t_ss, period=1.0,
                steps=5, theta=0.5)
    out = oracle_lib.thermal_transient(p)
    assert out["status"] == 0
    for s in range(1, 6):
        assert np.max(np.abs(out["temps"][s] - t_ss)) < 1e-10
        assert np.max(np.abs(out["reactions"][s] - r_ss)) < 1e-9


@pytest.mark.parametrize("name", ["Tet4", "Tet10"])
def test_long_time_reaches_the_steady_state(oracle_lib, name):
    # transient.rs:225-251
    mesh = slab(name, 4)
    base = problem(mesh, bcs=[(0.0, 100.0), (L, 20.0)], sources=300.0)
    t_ss, _ = steady(oracle_lib, base)
    p = problem(mesh, bcs=[(0.0, 100.0), (L, 20.0)], sources=300.0, initial=0.0, period=40.0, steps=40)
    out = oracle_lib.thermal_transient(p, fluxes=False)
    assert out["status"] == 0
    assert np.max(np.abs(out["temps"][40] - t_ss)) < 1e-8


def fourier(x, t, ts):
    alpha = K / (RHO * C)
    n = 2 * np.arange(500) + 1.0
    terms = 4.0 / (n * np.pi) * np.sin(np.outer(x, n) * np.pi / L) * np.exp(-alpha * (n * np.pi / L) ** 2 * t)
    return ts * (1.0 - terms.sum(axis=1))


def quench_errors(oracle_lib, name, nx, increments):
    ts = 100.0
    mesh = slab(name, nx)
    p = problem(mesh, bcs=[(0.0, ts), (L, ts)], initial=0.0, period=0.1, steps=increments)
    out = oracle_lib.thermal_transient(p, fluxes=False)
    assert out["status"] == 0
    x = mesh[0][:, 0]
    errs = []
    for s in (increments // 5, increments // 2, increments):
        t = s * p.time_step
        errs.append(float(np.max(np.abs(out["temps"][s] - fourier(x, t, ts)) / ts)))
    return errs


@pytest.mark.parametrize("name,nx", [("Tet4", 40), ("Tet10", 10)])
def test_quenched_slab_follows_the_fourier_series(oracle_lib, name, nx):
    # transient.rs:281-295
    errors = quench_errors(oracle_lib, name, nx, 400)
    assert all(e < 4e-3 for e in errors), errors


def test_quenched_slab_converges_in_time_and_space(oracle_lib):
    # transient.rs:297-312 (the Tet10 and Tet4 halves)
    ratio = quench_errors(oracle_lib, "Tet10", 20, 100)[2] / quench_errors(oracle_lib, "Tet10", 20, 400)[2]
    assert 3.4 < ratio < 4.4, ratio
    ratio = quench_errors(oracle_lib, "Tet4", 10, 400)[2] / quench_errors(oracle_lib, "Tet4", 20, 400)[2]
    assert 2.9 < ratio < 4.2, ratio


@pytest.mark.parametrize("name", ["Tet4", "Tet10"])
def test_small_biot_cooling_follows_the_discrete_amplification_factor(oracle_lib, name):
    # transient.rs:314-349
    film, sink, t0 = 0.4, 20.0, 100.0
    tau = RHO * C * VOLUME / (film * H * THICKNESS)
    mesh = slab(name, 2, k=1e7 * film * L)
    w = weights(mesh)
    for theta in (1.0, 0.75, 0.5):
        p = problem(mesh, convection=(L, film, sink), initial=t0, period=tau, steps=8, theta=theta)
        r = p.time_step / tau
        g = (1.0 - (1.0 - theta) * r) / (1.0 + theta * r)
        out = oracle_lib.thermal_transient(p, fluxes=False)
        assert out["status"] == 0
        for s in range(9):
            expected = sink + (t0 - sink) * g ** s
            got = mean(out["temps"][s], w)
            assert abs(got - expected) < 1e-5 * (t0 - sink), (theta, s, got, expected)
            assert np.max(np.abs(out["temps"][s] - got)) < 1e-5 * (t0 - sink)


def heisler_roots(biot, count):
    roots = []
    for n in range(count):
        f = lambda z: z * math.sin(z) - biot * math.cos(z)  # noqa: E731
        a, b = n * math.pi, n * math.pi + math.pi / 2
        for _ in range(100):
            m = (a + b) / 2
            if f(a) * f(m) <= 0.0:
                b = m
            else:
                a = m
        roots.append((a + b) / 2)
    return np.array(roots)


def heisler(x, t, roots):
    fo = K / (RHO * C) * t / (L * L)
    z = roots
    coef = 4.0 * np.sin(z) / (2.0 * z + np.sin(2.0 * z))
    return (coef * np.exp(-z * z * fo) * np.cos(np.outer(x, z) / L)).sum(axis=1)


@pytest.mark.parametrize("name,nx,tolerance", [("Tet4", 40, 4e-3), ("Tet10", 5, 5e-4)])
def test_convective_cooling_at_finite_biot_follows_heisler(oracle_lib, name, nx, tolerance):
    # transient.rs:393-402
    biot, t0, sink = 1.0, 100.0, 20.0
    roots = heisler_roots(biot, 200)
    assert abs(roots[0] - 0.860333589) < 1e-9
    mesh = slab(name, nx)
    p = problem(mesh, convection=(L, biot * K / L, sink), initial=t0, period=0.5, steps=200, theta=0.5)
    out = oracle_lib.thermal_transient(p, fluxes=False)
    assert out["status"] == 0
    x = mesh[0][:, 0]
    for s in (20, 80, 200):
        err = np.max(np.abs((out["temps"][s] - sink) / (t0 - sink) - heisler(x, s * p.time_step, roots)))
        assert err < tolerance, (s, err)


def test_time_order_is_one_for_euler_and_two_for_crank_nicolson(oracle_lib):
    # transient.rs:420-443 (on the Tet4 slab)
    film, sink, t0 = 0.4, 20.0, 100.0
    tau = RHO * C * VOLUME / (film * H * THICKNESS)
    mesh = slab("Tet4", 2, k=1e7 * film * L)
    w = weights(mesh)
    exact = sink + (t0 - sink) * math.exp(-1.0)

    def error(theta, n):
        p = problem(mesh, convection=(L, film, sink), initial=t0, period=tau, steps=n, theta=theta)
        out = oracle_lib.thermal_transient(p, fluxes=False)
        return abs(mean(out["temps"][n], w) - exact)

    euler = error(1.0, 10) / error(1.0, 20)
    crank = error(0.5, 10) / error(0.5, 20)
    assert 1.9 < euler < 2.1, euler
    assert 3.9 < crank < 4.1, crank


@pytest.mark.parametrize("name", ["Tet4", "Tet10"])
def test_energy_balance_is_exact(oracle_lib, name):
    # transient.rs:445-474
    q = 50.0
    mesh = slab(name, 4)
    w = weights(mesh)
    nodes = mesh[0]
    p = problem(mesh, bcs=[(0.0, 80.0)], sources=q, initial=20.0 + 5.0 * nodes[:, 0], period=0.3,
                steps=12, theta=0.5)
    out = oracle_lib.thermal_transient(p, fluxes=False)
    assert out["status"] == 0
    stored = RHO * C * VOLUME * (mean(out["temps"][12], w) - mean(out["temps"][0], w))
    supplied = sum(p.time_step * (out["reactions"][s].sum() + q * VOLUME) for s in range(1, 13))
    assert abs(stored - supplied) < 1e-10 * abs(stored), (stored, supplied)


def test_linear_field_gives_the_exact_flux_and_the_iterative_solver_agrees(oracle_lib):
    # a steady slab between two temperatures: T linear in x, q = -k dT/dx at every Gauss point
    # (heat_fluxes, element.rs:480-506), the same with the IC(0)-PCG as with the direct solver
    for name in ("Tet4", "Tet10"):
        mesh = slab(name, 6, k=2.5)
        p = problem(mesh, bcs=[(0.0, 100.0), (L, 40.0)], initial=0.0, period=1.0, steps=1)
        q = mg.ThermalProblem(**{**p.__dict__, "rho_c": np.zeros_like(p.rho_c)})
        direct = oracle_lib.thermal_transient(q, solver=1)
        pcg = oracle_lib.thermal_transient(q, solver=2)
        assert direct["status"] == 0 and pcg["status"] == 0
        x = mesh[0][:, 0]
        assert np.max(np.abs(direct["temps"][1] - (100.0 - 60.0 * x))) < 1e-9
        assert np.max(np.abs(pcg["temps"][1] - direct["temps"][1])) < 1e-8
        qx = direct["fluxes"][1][..., 3]
        assert np.max(np.abs(qx - 2.5 * 60.0)) < 1e-8
        assert np.max(np.abs(direct["fluxes"][1][..., 4:])) < 1e-8


# --- tests/thermal.rs: steady conduction (Model::solve, Analysis::Thermal) -----------------------

KS, TS, LS, HS = 50.0, 2.0, 4.0, 1.0  # tests/thermal.rs:13-17: k, thickness (z), length (x), height (y)


def steady_mesh(n, quadratic):
    nodes, tets = mg.box_grid(n, (LS, HS, TS))
    conn = tets
    if quadratic:
        nodes, conn = mg.to_quadratic_tet(nodes, tets)
    return nodes, conn


def face_positions(npe, face):
    """Element node positions of a face (mesh.rs:184-198): its corners, then for Tet10 the
    mid-edge nodes of its edges a-b, b-c, c-a."""
    a, b, c = (int(v) for v in mg.TET_FACES[face])
    if npe == 4:
        return [a, b, c]
    edges = [tuple(e) for e in mg.TET10_EDGES.tolist()]
    mid = lambda p, q: 4 + (edges.index((p, q)) if (p, q) in edges else edges.index((q, p)))  # noqa: E731
    return [a, b, c, mid(a, b), mid(b, c), mid(c, a)]


def steady_problem(nodes, conn, bcs=(), source=0.0, convection=None):
    n, ne = nodes.shape[0], conn.shape[0]
    fixed = np.zeros(n, np.uint8)
    imposed = np.zeros(n)
    for x, value in bcs:
        on = np.abs(nodes[:, 0] - x) < 1e-12
        fixed[on] = 1
        imposed[on] = value
    p = mg.ThermalProblem(coords=nodes, conn=conn, conductivity=np.full(ne, KS), rho_c=np.zeros(ne),
                          fixed=fixed, imposed=imposed, loads=np.zeros(n), initial=np.zeros(n))
    if source:
        p.s_elem = np.arange(ne, dtype=np.int64)
        p.s_value = np.full(ne, float(source))
    if convection is not None:
        on_face, film, sink = convection
        ce, cf = [], []
        for e in range(ne):
            for f in range(4):
                # every node of the face (Element::face_nodes: Tet10 faces include their mid-edge
                # nodes), so an interior face whose corners all lie on the sides is left out
                if all(on_face(nodes[v]) for v in conn[e, face_positions(conn.shape[1], f)]):
                    ce.append(e)
                    cf.append(f)
        p.c_elem = np.array(ce, np.int64)
        p.c_face = np.array(cf, np.int32)
        p.c_film = np.full(len(ce), film)
        p.c_sink = np.full(len(ce), sink)
    return p


def run_steady(oracle_lib, p):
    out = oracle_lib.thermal_transient(p, solver=1)
    assert out["status"] == 0
    return out["temps"][1], out["reactions"][1], out["fluxes"][1]


@pytest.mark.parametrize("quadratic", [False, True])
def test_wall_with_imposed_temperatures_is_exact_with_the_right_heat_flow(oracle_lib, quadratic):
    # tests/thermal.rs:99-137 (Tet4 / Tet10 [4, 1, 2])
    t1, t2 = 100.0, 20.0
    q = -KS * (t2 - t1) / LS
    power = q * HS * TS
    nodes, conn = steady_mesh((4, 1, 2), quadratic)
    t, r, fl = run_steady(oracle_lib, steady_problem(nodes, conn, bcs=[(0.0, t1), (LS, t2)]))
    assert np.max(np.abs(t - (t1 + (t2 - t1) * nodes[:, 0] / LS))) < 1e-10
    assert np.max(np.abs(fl[..., 3] - q)) < 1e-9 * q
    assert np.max(np.abs(fl[..., 4:])) < 1e-9 * q
    at = lambda x: np.abs(nodes[:, 0] - x) < 1e-12  # noqa: E731
    assert abs(r[at(0.0)].sum() - power) < 1e-9 * power
    assert abs(r[at(LS)].sum() + power) < 1e-9 * power


def slab_errors(oracle_lib, nodes, conn):
    # tests/thermal.rs:286-318: uniform source q, T = 0 on x = 0 and x = L
    q = 1e3
    t, r, fl = run_steady(oracle_lib, steady_problem(nodes, conn, bcs=[(0.0, 0.0), (LS, 0.0)], source=q))
    produced = q * LS * HS * TS
    assert abs(r.sum() + produced) < 1e-9 * produced
    x = nodes[:, 0]
    terr = np.max(np.abs(t - q * x * (LS - x) / (2.0 * KS)))
    qerr = np.max(np.abs(fl[..., 3] - q * (fl[..., 0] - LS / 2.0)))
    return terr / (q * LS * LS / (8.0 * KS)), qerr / (q * LS / 2.0)


def test_quadratic_elements_are_exact_for_a_uniform_heat_source(oracle_lib):
    # tests/thermal.rs:320-327 (the Tet10 half)
    t, q = slab_errors(oracle_lib, *steady_mesh((2, 1, 1), True))
    assert t < 1e-10 and q < 1e-10, (t, q)


def test_linear_elements_are_exact_at_the_nodes_and_their_flux_converges(oracle_lib):
    # tests/thermal.rs:329-358 (the Tet4 half)
    errors = [slab_errors(oracle_lib, *steady_mesh((nx, 1, 1), False)) for nx in (4, 8, 16)]
    for t, q in errors:
        assert t < 1e-10 and q > 1e-3, errors
    for a, b in zip(errors, errors[1:]):
        assert 1.8 < a[1] / b[1] < 2.2, errors


@pytest.mark.parametrize("quadratic", [False, True])
def test_wall_cooled_by_convection_is_exact(oracle_lib, quadratic):
    # tests/thermal.rs:424-456 (Tet4 / Tet10 [4, 1, 2])
    t1, h, sink = 20.0, 30.0, 300.0
    power = HS * TS * KS * h * (sink - t1) / (KS + h * LS)
    nodes, conn = steady_mesh((4, 1, 2), quadratic)
    p = steady_problem(nodes, conn, bcs=[(0.0, t1)], convection=(lambda q: abs(q[0] - LS) < 1e-12, h, sink))
    assert p.c_elem.size > 0
    t, r, _ = run_steady(oracle_lib, p)
    assert np.max(np.abs(t - (t1 + (sink - t1) * h * nodes[:, 0] / (KS + h * LS)))) < 1e-10
    out = r[np.abs(nodes[:, 0]) < 1e-12].sum()
    assert abs(out + power) < 1e-9 * power


def test_thin_fins_match_fin_theory(oracle_lib):
    # tests/thermal.rs:472-505 (the Tet10 bar: 16 x 1 x 1 cells of 16 x H x T, four lateral faces)
    h, length = 0.1, 16.0
    nodes, tets = mg.box_grid((16, 1, 1), (length, HS, TS))
    nodes, conn = mg.to_quadratic_tet(nodes, tets)
    m = math.sqrt(h * 2.0 * (HS + TS) / (KS * HS * TS))
    side = lambda c, lim: abs(c) < 1e-12 or abs(c - lim) < 1e-12  # noqa: E731
    t0, sink = 100.0, 20.0
    p = steady_problem(nodes, conn, bcs=[(0.0, t0)],
                       convection=(lambda q: side(q[1], HS) or side(q[2], TS), h, sink))
    t, _, _ = run_steady(oracle_lib, p)
    exact = sink + (t0 - sink) * np.cosh(m * (length - nodes[:, 0])) / math.cosh(m * length)
    assert np.max(np.abs(t - exact)) / (t0 - sink) < 0.002
