"""The oracle's large-strain path (neo-Hookean Tet4, quasi-static Newton, adjoint) on the CPU:
the element response against the linear stiffness in the small-displacement limit (the
reference's assembly.rs:1195-1210 check) and against finite differences of itself, the
reference's uniaxial-tension closed form (tests/finite_strain.rs: neo_hookean uniaxial tension
with free lateral sides) restated on displacements and reactions, and the adjoint gradient of a
reaction force against central differences of whole quasi-static runs."""
import copy

import numpy as np
import pytest

from maille_b200 import meshgen as mg
from maille_b200.large_strain import from_lame, lame

E, NU = 210e3, 0.3
L, W, D = 2.0, 1.0, 1.0


def tet():
    return np.array([[0.1, 0.0, 0.0], [1.2, 0.1, 0.0], [0.0, 0.9, 0.2], [0.1, 0.1, 1.1]])


def test_small_displacements_give_the_linear_response(oracle_lib):
    lam, mu = lame(E, NU)
    u = 1e-7 * np.random.default_rng(0).standard_normal(12)
    s, fe, ke, _, _ = oracle_lib.neo_hookean_tet4(tet(), lam, mu, u)
    assert s == 0
    k = oracle_lib.element_stiffness(tet(), E, NU)
    assert np.abs(fe - k @ u).max() <= 1e-5 * np.abs(k @ u).max()
    assert np.abs(ke - k).max() <= 1e-5 * np.abs(k).max()


def test_tangent_and_parameter_derivatives_match_differences(oracle_lib):
    lam, mu = 120000.0, 80000.0
    u = 0.05 * np.random.default_rng(1).standard_normal(12)
    _, fe, ke, dm, dl = oracle_lib.neo_hookean_tet4(tet(), lam, mu, u)
    assert np.abs(ke - ke.T).max() <= 1e-14 * np.abs(ke).max()
    h = 1e-7
    fd = np.zeros((12, 12))
    for k in range(12):
        up, um = u.copy(), u.copy()
        up[k] += h
        um[k] -= h
        fd[:, k] = (oracle_lib.neo_hookean_tet4(tet(), lam, mu, up)[1]
                    - oracle_lib.neo_hookean_tet4(tet(), lam, mu, um)[1]) / (2 * h)
    assert np.abs(fd - ke).max() <= 1e-7 * np.abs(ke).max()
    for which, d, ref in ((0, mu, dm), (1, lam, dl)):
        args_p = (lam, mu * (1 + 1e-6)) if which == 0 else (lam * (1 + 1e-6), mu)
        args_m = (lam, mu * (1 - 1e-6)) if which == 0 else (lam * (1 - 1e-6), mu)
        fd = (oracle_lib.neo_hookean_tet4(tet(), *args_p, u)[1]
              - oracle_lib.neo_hookean_tet4(tet(), *args_m, u)[1]) / (2e-6 * d)
        assert np.abs(fd - ref).max() <= 1e-7 * np.abs(ref).max()


def uniaxial_closed_form(stretch):
    """Free lateral sides: lateral stretch l with sigma_yy(l, J = stretch l^2) = 0 (bisection),
    then sigma_xx (finite_strain.rs tests, neo_hooke::uniaxial)."""
    lam, mu = lame(E, NU)

    def principal(s, j):
        return (mu * (s * s - 1.0) + lam * np.log(j)) / j

    lo, hi = 0.01, 10.0
    sign = np.sign(principal(lo, stretch * lo * lo))
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if np.sign(principal(mid, stretch * mid * mid)) == sign:
            lo = mid
        else:
            hi = mid
    lat = 0.5 * (lo + hi)
    return lat, principal(stretch, stretch * lat * lat)


def tension_block():
    """box_grid([3, 2, 2], [L, W, D]) Tet4 with free_lateral_tension's constraints."""
    nodes, tets = mg.box_grid((3, 2, 2), (L, W, D))
    n = nodes.shape[0]
    fixed = np.zeros(3 * n, np.uint8)
    imposed = np.zeros(3 * n)
    x0 = np.abs(nodes[:, 0]) < 1e-9
    xl = np.abs(nodes[:, 0] - L) < 1e-9
    fixed[3 * np.nonzero(x0 | xl)[0]] = 1
    fixed[3 * np.nonzero(np.abs(nodes[:, 1]) < 1e-9)[0] + 1] = 1
    fixed[3 * np.nonzero(np.abs(nodes[:, 2]) < 1e-9)[0] + 2] = 1
    return mg.Problem(coords=nodes, conn=tets, young=np.full(tets.shape[0], E),
                      poisson=np.full(tets.shape[0], NU), fixed=fixed, imposed=imposed,
                      loads=np.zeros(3 * n)), xl


def test_uniaxial_tension_matches_the_closed_form(oracle_lib):
    stretch = 2.0
    lat, sxx = uniaxial_closed_form(stretch)
    p, xl = tension_block()
    p.imposed[3 * np.nonzero(xl)[0]] = (stretch - 1.0) * L
    r = oracle_lib.large_strain_run(p, increments=8)
    assert r["status"] == 0
    u = r["u_hist"][-1].reshape(-1, 3)
    x = p.coords
    assert np.abs(u[:, 0] - (stretch - 1) * x[:, 0]).max() < 1e-6 * L
    assert np.abs(u[:, 1] - (lat - 1) * x[:, 1]).max() < 1e-6 * L
    assert np.abs(u[:, 2] - (lat - 1) * x[:, 2]).max() < 1e-6 * L
    # axial force on the x = L face: first Piola stress P_xx = sigma_xx l^2 on the initial area
    force = r["reactions"][-1][3 * np.nonzero(xl)[0]].sum()
    assert abs(force - sxx * lat * lat * W * D) < 1e-6 * sxx * W * D
    assert (r["newton"] <= 8).all()


def test_adjoint_reaction_gradient_matches_central_differences(oracle_lib):
    p, mu, tip = mg.large_strain_block(cells=(8, 2, 2))
    lam = 120000.0
    r = oracle_lib.large_strain_run(p, increments=10, newton_tol=1e-12, pcg_tol=1e-15)
    assert r["status"] == 0
    w = np.zeros_like(r["reactions"])
    w[-1, tip] = 1.0
    s, gm, gl = oracle_lib.large_strain_gradient(p, r["u_hist"], w, pcg_tol=1e-15)
    assert s == 0

    def J(mu_v):
        q = copy.copy(p)
        q.young, q.poisson = from_lame(lam, mu_v)
        rr = oracle_lib.large_strain_run(q, increments=10, newton_tol=1e-12, pcg_tol=1e-15)
        assert rr["status"] == 0
        return rr["reactions"][-1, tip].sum()

    for e in (0, 37, 100):
        h = 1e-4 * mu[e]
        mp, mm = mu.copy(), mu.copy()
        mp[e] += h
        mm[e] -= h
        fd = (J(mp) - J(mm)) / (2 * h)
        assert abs(fd - gm[e]) <= 1e-6 * abs(gm[e]), (e, fd, gm[e])


def test_newton_failures_halve_the_increment(oracle_lib):
    """advance (model.rs:820-870): a Newton that needs more than newton_max corrections is
    retried on two halves of the interval, up to five halvings deep (MAX_CUTS, model.rs:1224)."""
    p, mu, tip = mg.large_strain_block(cells=(8, 2, 2))
    full = oracle_lib.large_strain_run(p, increments=2)
    assert full["status"] == 0 and not full["cuts"].any()
    cut = oracle_lib.large_strain_run(p, increments=2, newton_max=3)
    assert cut["status"] == 0 and (cut["cuts"] == 1).all()
    # the same end state at the Newton tolerance
    assert np.linalg.norm(cut["u_hist"][-1] - full["u_hist"][-1]) < 1e-7 * np.linalg.norm(full["u_hist"][-1])
    # every halving exhausted: NotConverged after MAX_CUTS = 5 cuts of the first increment
    out = oracle_lib.large_strain_run(p, increments=2, newton_max=2)
    assert out["status"] == 2 and out["stop_increment"] == 1 and out["stop_cuts"] == 5


def test_inner_pcg_cap_ends_the_run_without_a_cut(oracle_lib):
    """An inner solve at its iteration cap is IterativeNotConverged (error.rs:226-229), which
    advance passes up unchanged: no halving (model.rs:839-842 cuts on NotConverged, Singular and
    PlasticCollapse only)."""
    p, mu, tip = mg.large_strain_block(cells=(8, 2, 2))
    out = oracle_lib.large_strain_run(p, increments=10, pcg_max=3)
    assert out["status"] == 2 and out["stop_increment"] == 1 and out["stop_cuts"] == 0
    assert out["pcg_total"] == 3 and out["newton_total"] == 1
