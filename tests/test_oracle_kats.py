"""Pins the CPU oracle to the reference's own known-answer tests for this path (CPU only).

Each test restates a reference test (paths relative to crates/maille-core of the reference) and
runs it on the oracle, so a GPU result compared with the oracle is compared with something that
already passes the reference's checks.
"""
import numpy as np
import pytest

import cases


# --- solve.rs / iterative.rs unit tests ---------------------------------------------------------

def test_dot_matches_the_plain_sum_for_every_length_around_the_chunk_size(oracle_lib):
    # solve.rs:349-359
    for n in range(40):
        a = 0.5 + np.arange(n, dtype=float)
        b = 2.0 - 0.25 * np.arange(n, dtype=float)
        plain = float(sum(x * y for x, y in zip(a, b)))
        assert abs(oracle_lib.dot(a, b) - plain) <= 1e-12 * (1 + abs(plain))


def test_graph_lists_each_neighbour_once(oracle_lib):
    # iterative.rs:286-293
    off, tgt = oracle_lib.graph_from_elements(4, [[0, 1, 2], [1, 2, 3]])
    assert sorted(tgt[off[1]:off[2]]) == [0, 2, 3]
    assert off[1] - off[0] == 2


def _profile(adj, order):
    rank = np.empty(len(order), int)
    rank[np.asarray(order)] = np.arange(len(order))
    return sum(rank[v] - min([rank[w] for w in adj[v]] + [rank[v]]) + 1 for v in range(len(adj)))


def _csr(adj):
    off = np.zeros(len(adj) + 1, np.int64)
    for v, a in enumerate(adj):
        off[v + 1] = off[v] + len(a)
    return off, np.array([w for a in adj for w in a], np.int64)


def test_rcm_is_a_permutation_that_shrinks_the_profile_of_a_shuffled_grid(oracle_lib):
    # solve.rs:387-416
    side, shuffle = 6, [3, 0, 5, 1, 4, 2]
    idx = lambda i, j: shuffle[i] * side + shuffle[j]  # noqa: E731
    adj = [[] for _ in range(side * side)]
    for i in range(side):
        for j in range(side):
            if i + 1 < side:
                adj[idx(i, j)].append(idx(i + 1, j))
                adj[idx(i + 1, j)].append(idx(i, j))
            if j + 1 < side:
                adj[idx(i, j)].append(idx(i, j + 1))
                adj[idx(i, j + 1)].append(idx(i, j))
    order = oracle_lib.rcm(*_csr(adj))
    assert sorted(order) == list(range(side * side))
    before, after = _profile(adj, range(side * side)), _profile(adj, order)
    assert after <= side * side * (side + 1)
    assert after < before


def test_rcm_handles_disconnected_graphs_and_isolated_vertices(oracle_lib):
    # solve.rs:418-425
    order = oracle_lib.rcm(*_csr([[2], [3], [0], [1], []]))
    assert sorted(order) == [0, 1, 2, 3, 4]


def _grid_system(oracle_lib, n):
    """iterative.rs:256-283: (4 + degree, -1) Laplacian of an n x n grid, RCM numbered."""
    elements = cases.grid_laplacian_elements(n)
    off, tgt = oracle_lib.graph_from_elements(n * n, elements)
    order = oracle_lib.rcm(off, tgt)
    rank = np.empty(n * n, np.int64)
    rank[order] = np.arange(n * n)
    trip = []
    for v in range(n * n):
        nb = tgt[off[v]:off[v + 1]]
        trip.append((rank[v], rank[v], 1.0 + len(nb)))
        trip += [(rank[v], rank[w], -1.0) for w in nb if w < v]
    x = np.sin(np.arange(n * n) * 0.37)
    s, b, _ = oracle_lib.csr_run(off, tgt, trip, x, mode=2, order=order)
    assert s == 0
    return off, tgt, order, trip, x, b


def test_pcg_recovers_the_chosen_solution(oracle_lib):
    # iterative.rs:302-309 (b = A x in the renumbered space, x chosen there)
    off, tgt, order, trip, x, b = _grid_system(oracle_lib, 30)
    s, got, _ = oracle_lib.csr_run(off, tgt, trip, b, mode=0, order=order)
    assert s == 0
    assert np.abs(got - x).max() < 1e-8


def test_pcg_solves_several_right_hand_sides_and_a_zero_one(oracle_lib):
    # iterative.rs:311-324
    off, tgt, order, trip, _, b = _grid_system(oracle_lib, 10)
    s, z, it = oracle_lib.csr_run(off, tgt, trip, np.zeros(100), mode=0, order=order)
    assert s == 0 and np.all(z == 0.0) and it == 0
    s, x, _ = oracle_lib.csr_run(off, tgt, trip, b, mode=0, order=order)
    _, ax, _ = oracle_lib.csr_run(off, tgt, trip, x, mode=2, order=order)
    assert np.abs(ax - b).max() < 1e-8


def test_incomplete_cholesky_of_a_tridiagonal_matrix_is_exact(oracle_lib):
    # iterative.rs:326-346
    off, tgt = oracle_lib.graph_from_elements(4, [[0, 1], [1, 2], [2, 3]])
    trip = [(i, i, 2.0) for i in range(4)] + [(i, i - 1, -1.0) for i in range(1, 4)]
    s, z, _ = oracle_lib.csr_run(off, tgt, trip, np.array([1.0, 0, 0, 1.0]), mode=1)
    assert s == 0
    _, back, _ = oracle_lib.csr_run(off, tgt, trip, z, mode=2)
    assert np.abs(back - [1.0, 0, 0, 1.0]).max() < 1e-13


def test_singular_matrix_is_reported(oracle_lib):
    # iterative.rs:348-362
    off, tgt = oracle_lib.graph_from_elements(3, [[0, 1], [1, 2]])
    trip = [(0, 0, 1.0), (1, 1, 2.0), (2, 2, 1.0), (1, 0, -1.0), (2, 1, -1.0)]
    s, _, _ = oracle_lib.csr_run(off, tgt, trip, np.ones(3), mode=0)
    assert s != 0


# --- element kernels, face loads, von Mises ----------------------------------------------------

VERTICES = np.array([[1.0, 0.5, 0.0], [3.0, 1.0, 0.5], [1.5, 2.5, 0.0], [1.2, 1.0, 2.0]])
EDGES = [(0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3)]


def element_coords(quadratic):
    """element.rs:716-730: a general tet, plus its mid-edge nodes for Tet10."""
    c = [v for v in VERTICES]
    if quadratic:
        c += [(VERTICES[a] + VERTICES[b]) / 2 for a, b in EDGES]
    return np.array(c)


def volume():
    e = VERTICES[1:] - VERTICES[0]
    return np.dot(e[0], np.cross(e[1], e[2])) / 6


def uniform_strain(c, eps):
    return np.stack([eps[0] * c[:, 0] + eps[5] / 2 * c[:, 1] + eps[4] / 2 * c[:, 2],
                     eps[5] / 2 * c[:, 0] + eps[1] * c[:, 1] + eps[3] / 2 * c[:, 2],
                     eps[4] / 2 * c[:, 0] + eps[3] / 2 * c[:, 1] + eps[2] * c[:, 2]], 1).ravel()


@pytest.mark.parametrize("quadratic", [False, True])
def test_tet_stiffness_is_symmetric_and_ignores_the_six_rigid_motions(oracle_lib, quadratic):
    # element.rs:782-817
    c = element_coords(quadratic)
    k = oracle_lib.element_stiffness(c, 210e3, 0.3)
    scale = k[0, 0]
    assert np.abs(k - k.T).max() < 1e-9 * scale
    motions = []
    for axis in range(3):
        t = np.zeros((len(c), 3))
        t[:, axis] = 1
        motions.append(t.ravel())
    x, y, z = c[:, 0], c[:, 1], c[:, 2]
    zero = np.zeros_like(x)
    motions += [np.stack([zero, -z, y], 1).ravel(), np.stack([z, zero, -x], 1).ravel(),
                np.stack([-y, x, zero], 1).ravel()]
    for u in motions:
        assert np.abs(k @ u).max() < 1e-9 * scale


@pytest.mark.parametrize("quadratic", [False, True])
def test_tet_strain_energy_of_a_uniform_strain_is_v_eps_d_eps(oracle_lib, quadratic):
    # element.rs:819-843
    c = element_coords(quadratic)
    k = oracle_lib.element_stiffness(c, 210e3, 0.3)
    d = cases.d_matrix()
    for eps in ([1e-3, 0, 0, 0, 0, 0], [0, 0, 1e-3, 0, 0, 0], [0, 0, 0, 1e-3, 0, 0],
                [0, 0, 0, 0, 0, 1e-3], [1e-3, -2e-3, 0.5e-3, 3e-3, -1e-3, 2e-3]):
        eps = np.array(eps, float)
        u = uniform_strain(c, eps)
        expected = volume() * eps @ d @ eps
        assert abs(u @ k @ u - expected) < 1e-9 * expected


@pytest.mark.parametrize("quadratic", [False, True])
def test_tet_stresses_of_a_uniform_strain_are_d_eps_at_every_gauss_point(oracle_lib, quadratic):
    # element.rs:845-862
    eps = cases.EPS
    c = element_coords(quadratic)
    d = cases.d_matrix()
    sigma = d @ eps
    out = oracle_lib.element_stresses(c, 210e3, 0.3, uniform_strain(c, eps))
    for p in out:
        got = np.array([p[3], p[4], p[5], p[7], p[8], p[6]])  # to Voigt xx yy zz yz xz xy
        assert np.abs(got - sigma).max() < 1e-9 * d[0, 0] * 1e-3


def unit_tet(quadratic):
    v = np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    if quadratic:
        v = np.concatenate([v, [(v[a] + v[b]) / 2 for a, b in EDGES]])
    return v


def test_tet4_face_load_is_a_third_of_the_resultant_at_each_node(oracle_lib):
    # assembly.rs:1296-1302
    pos, f = oracle_lib.face_pressure(unit_tet(False), 0, 6.0)
    assert list(pos) == [0, 1, 2]
    assert np.abs(f - [0, 0, 1, 0, 0, 1, 0, 0, 1]).max() < 1e-12


def test_tet10_face_load_goes_to_the_mid_nodes_only(oracle_lib):
    # assembly.rs:1304-1314
    pos, f = oracle_lib.face_pressure(unit_tet(True), 0, 6.0)
    assert list(pos) == [0, 1, 2, 4, 5, 6]
    assert np.abs(f - np.array([0.0] * 9 + [0, 0, 1, 0, 0, 1, 0, 0, 1])).max() < 1e-12


def test_a_slanted_face_gets_the_outward_resultant(oracle_lib):
    # assembly.rs:1316-1325
    _, f = oracle_lib.face_pressure(unit_tet(False), 2, 6.0)
    assert np.abs(f.reshape(3, 3).sum(0) + 3.0).max() < 1e-12


def test_missing_faces_give_nothing(oracle_lib):
    # assembly.rs:1327-1340 (the tet part)
    pos, f = oracle_lib.face_pressure(unit_tet(False), 4, 1.0)
    assert len(pos) == 0 and len(f) == 0


def _s(sxx=0, syy=0, szz=0, txy=0, tyz=0, txz=0):
    return np.array([0, 0, 0, sxx, syy, szz, txy, tyz, txz], float)


def test_von_mises_known_answers(oracle_lib):
    # results.rs:339-370
    assert abs(oracle_lib.von_mises(_s(sxx=100)) - 100) < 1e-12
    assert abs(oracle_lib.von_mises(_s(txy=50)) - 50 * 3 ** 0.5) < 1e-12
    assert abs(oracle_lib.von_mises(_s(80, 80, 80))) < 1e-12
    assert abs(oracle_lib.von_mises(_s(tyz=30, txz=40)) - 50 * 3 ** 0.5) < 1e-12
    nu = 0.3
    assert abs(oracle_lib.von_mises(_s(sxx=100, szz=nu * 100)) - 100 * (1 - nu + nu * nu) ** 0.5) < 1e-12


# --- whole solves (tests/solid.rs, tests/pressure.rs, tests/iterative.rs) ---------------------

def voigt(g):
    """(.., 9) Gauss records -> Voigt (xx, yy, zz, yz, xz, xy)."""
    return np.stack([g[..., 3], g[..., 4], g[..., 5], g[..., 7], g[..., 8], g[..., 6]], -1)


def test_tet10_extrapolation_reproduces_a_linear_function_at_the_ten_nodes(oracle_lib):
    # results.rs:258-278 through the oracle's smoothing: one reference Tet10 whose Gauss values are a
    # linear f at the TETRA_4 points (point g near vertex g: barycentric a on it, b on the others)
    # must give f at the ten nodes
    from types import SimpleNamespace
    f = lambda x, y, z: 2.0 + 3.0 * x - 5.0 * y + 7.0 * z  # noqa: E731
    a, b = (5.0 + 3.0 * 5 ** 0.5) / 20.0, (5.0 - 5 ** 0.5) / 20.0
    nodes = np.array([(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (.5, 0, 0), (.5, .5, 0), (0, .5, 0),
                      (0, 0, .5), (.5, 0, .5), (0, .5, .5)], float)
    gauss = np.zeros((1, 4, 9))
    for g in range(4):
        lam = np.full(4, b)
        lam[g] = a
        x, y, z = lam[1], lam[2], lam[3]
        gauss[0, g, 3:] = f(x, y, z)
    prob = SimpleNamespace(coords=nodes, conn=np.arange(10, dtype=np.int64).reshape(1, 10))
    out = oracle_lib.nodal_stresses(prob, gauss)
    for k in range(10):
        assert np.abs(out[k] - f(*nodes[k])).max() < 1e-12, k


def test_nodal_smoothing_averages_over_the_elements_of_a_node(oracle_lib):
    # smooth, results.rs:198-230: component-wise mean over the elements sharing a node; an
    # isolated node gets 0 (two Tet4 sharing the face 1-2-3, node 5 touched by no element)
    from types import SimpleNamespace
    prob = SimpleNamespace(coords=np.zeros((6, 3)), conn=np.array([[0, 1, 2, 3], [1, 2, 3, 4]], np.int64))
    gauss = np.zeros((2, 1, 9))
    gauss[0, 0, 3:] = [1, 2, 3, 4, 5, 6]
    gauss[1, 0, 3:] = [3, 4, 5, 6, 7, 8]
    out = oracle_lib.nodal_stresses(prob, gauss)
    assert np.array_equal(out[0], [1, 2, 3, 4, 5, 6]) and np.array_equal(out[4], [3, 4, 5, 6, 7, 8])
    for k in (1, 2, 3):
        assert np.array_equal(out[k], [2, 3, 4, 5, 6, 7])
    assert np.array_equal(out[5], np.zeros(6))


@pytest.mark.parametrize("solver", [1, 2])
@pytest.mark.parametrize("quadratic", [False, True])
def test_uniform_strain_patch_is_exact(oracle_lib, quadratic, solver):
    # tests/solid.rs:52-116 (Auto = Direct at this size; the iterative solver must agree)
    p = cases.patch(quadratic)
    r = oracle_lib.model_solve(p, solver=solver)
    assert r["status"] == 0
    assert np.abs(r["u"].reshape(-1, 3) - cases.uniform_field(p.coords)).max() < 1e-12
    sigma = cases.d_matrix() @ cases.EPS
    scale = np.abs(sigma).max()
    assert np.abs(voigt(r["gauss"]) - sigma).max() <= 1e-9 * scale
    nodal = oracle_lib.nodal_stresses(p, r["gauss"])  # sxx syy szz txy tyz txz
    nv = np.stack([nodal[:, 0], nodal[:, 1], nodal[:, 2], nodal[:, 4], nodal[:, 5], nodal[:, 3]], 1)
    assert np.abs(nv - sigma).max() <= 1e-9 * scale


@pytest.mark.parametrize("quadratic", [False, True])
def test_uniaxial_traction_gives_e_delta_over_l_and_poisson_contraction(oracle_lib, quadratic):
    # tests/solid.rs:118-175
    L, delta = 4.0, 0.01
    p = cases.uniaxial(quadratic, L, delta)
    r = oracle_lib.model_solve(p, solver=1)
    strain = delta / L
    g = r["gauss"]
    assert np.abs(g[..., 3] - cases.E * strain).max() <= 1e-9 * cases.E * strain
    assert np.abs(g[..., 4]).max() < 1e-9 * cases.E * strain
    u = r["u"].reshape(-1, 3)
    assert np.abs(u[:, 1] + cases.NU * strain * p.coords[:, 1]).max() < 1e-12
    assert np.abs(u[:, 2] + cases.NU * strain * p.coords[:, 2]).max() < 1e-12
    pull = r["reactions"][0::3][np.abs(p.coords[:, 0] - L) < 1e-12].sum()
    assert abs(pull - cases.E * strain) <= 1e-9 * cases.E * strain


@pytest.mark.parametrize("quadratic", [False, True])
def test_cube_under_hydrostatic_pressure_shrinks_uniformly(oracle_lib, quadratic):
    # tests/pressure.rs:194-224
    p = cases.hydrostatic(quadratic)
    r = oracle_lib.model_solve(p, solver=1)
    strain = -50.0 * (1 - 2 * cases.NU) / cases.E
    assert np.abs(r["u"].reshape(-1, 3) - strain * p.coords).max() < 1e-12
    g = r["gauss"]
    assert np.abs(g[..., 3] + 50.0).max() < 1e-6 and np.abs(g[..., 6]).max() < 1e-6


def test_tet10_cantilever_matches_beam_theory(oracle_lib):
    # tests/solid.rs:259-270 (first size)
    p, tip = cases.cantilever((10, 2, 2), True)
    r = oracle_lib.model_solve(p, solver=1)
    assert abs(r["u"][3 * tip + 2] / cases.timoshenko() - 1) < 0.02


def test_iterative_static_solution_matches_the_direct_one(oracle_lib):
    # tests/iterative.rs:68-83 (max-norm relative gaps)
    p = cases.iterative_cantilever()
    d = oracle_lib.model_solve(p, solver=1)
    i = oracle_lib.model_solve(p, solver=2)
    gap = lambda a, b: np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)  # noqa: E731
    assert gap(i["u"], d["u"]) < 1e-8
    assert gap(i["reactions"], d["reactions"]) < 1e-8
    assert gap(i["gauss"][..., 3], d["gauss"][..., 3]) < 1e-7


@pytest.mark.parametrize("quadratic,cells,nu", [(True, 2, 0.49), (False, 4, 0.4999)])
def test_shift_ladder_rescues_a_failed_factorisation(oracle_lib, quadratic, cells, nu):
    # Pcg::new (iterative.rs:201-207): IC(0) of a nearly incompressible block meets a pivot
    # <= 1e-12 a_ii (iterative.rs:160-163) at shifts 0, 1e-3 and 1e-2 and succeeds at 0.1; the
    # shifted preconditioner still converges to the direct solution (tests/iterative.rs:68-83)
    p = cases.nearly_incompressible((cells,) * 3, quadratic, nu)
    d = oracle_lib.model_solve(p, solver=1)
    i = oracle_lib.model_solve(p, solver=2, tol=1e-14)
    assert i["status"] == 0 and i["shift"] == 0.1
    assert np.abs(i["u"] - d["u"]).max() < 1e-8 * np.abs(d["u"]).max()
    # the same matrix at nu = 0.3 factors without a shift
    q = cases.nearly_incompressible((cells,) * 3, quadratic, 0.3)
    assert oracle_lib.model_solve(q, solver=2)["shift"] == 0.0


def test_iterative_solver_reports_an_unconstrained_structure(oracle_lib):
    # tests/iterative.rs:199-224
    r = oracle_lib.model_solve(cases.unconstrained(), solver=2)
    assert r["status"] in (1, 2)


def test_cube_example_follows_the_analytic_field(oracle_lib):
    # crates/maille-cli/tests/examples.rs:669-681 on examples/cube
    p = cases.cube_example()
    r = oracle_lib.model_solve(p, solver=1)
    x = p.coords
    u = r["u"].reshape(-1, 3)
    assert np.abs(u[:, 0] - 0.01 * x[:, 0]).max() < 1e-12
    assert np.abs(u[:, 1] + 0.25 * 0.01 * x[:, 1]).max() < 1e-12
    assert np.abs(u[:, 2] + 0.25 * 0.01 * x[:, 2]).max() < 1e-12


def test_pressure_resultant_of_the_plain_config(oracle_lib):
    # 10 MPa on the unit face z = 1: the loads sum to -10 along z and the reactions balance them
    from maille_b200 import meshgen as mg
    p = mg.plain_tet4(6)
    r = oracle_lib.model_solve(p, solver=2)
    assert abs(r["f"][2::3].sum() + 10.0) < 1e-12
    assert abs(r["reactions"][2::3].sum() - 10.0) < 1e-9
