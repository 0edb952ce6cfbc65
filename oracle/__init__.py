"""ctypes wrapper of the CPU oracle (oracle/maille_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the checker, and by
bench.py's cpu_baseline / reference legs. The product package (maille_b200) never imports it.
"""
from __future__ import annotations

import copy
import ctypes
import os
import subprocess
import time

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_d = ctypes.POINTER(ctypes.c_double)
_i64 = ctypes.POINTER(ctypes.c_int64)
_i32 = ctypes.POINTER(ctypes.c_int32)
_u8 = ctypes.POINTER(ctypes.c_uint8)
_ip = ctypes.POINTER(ctypes.c_int)

STATUS = {0: "OK", 1: "SINGULAR", 2: "NOT_CONVERGED", 3: "INVALID"}


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++ only, no GPU needed)."""
    src = os.path.join(_HERE, "maille_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.oracle_element_stiffness.argtypes = [ctypes.c_int, _d, ctypes.c_double, ctypes.c_double, _d]
        L.oracle_element_stresses.argtypes = [ctypes.c_int, _d, ctypes.c_double, ctypes.c_double, _d, _d]
        L.oracle_von_mises.argtypes = [_d]
        L.oracle_von_mises.restype = ctypes.c_double
        L.oracle_face_pressure.argtypes = [ctypes.c_int, _d, ctypes.c_int, ctypes.c_double, _ip, _d]
        L.oracle_face_pressure.restype = ctypes.c_int
        L.oracle_dot.argtypes = [_d, _d, ctypes.c_int64]
        L.oracle_dot.restype = ctypes.c_double
        L.oracle_graph_from_elements.argtypes = [ctypes.c_int64, ctypes.c_int64, _i64, _i64, _i64, _i64]
        L.oracle_graph_from_elements.restype = ctypes.c_int64
        L.oracle_rcm.argtypes = [ctypes.c_int64, _i64, _i64, _i64]
        L.oracle_csr_run.argtypes = [ctypes.c_int64, _i64, _i64, _i64, ctypes.c_int64, _i64, _i64, _d,
                                     _d, ctypes.c_int, ctypes.c_double, _d, _i64]
        L.oracle_csr_run.restype = ctypes.c_int
        L.oracle_model_solve.argtypes = [
            ctypes.c_int64, _d, ctypes.c_int, ctypes.c_int64, _i64, _d, _d, _u8, _d, _d,
            ctypes.c_int64, _i64, _i32, _d, ctypes.c_int, ctypes.c_double, ctypes.c_int64, _i64,
            _d, _d, _d, _d, _d, _d]
        L.oracle_model_solve.restype = ctypes.c_int
        L.oracle_energy.argtypes = [ctypes.c_int64, _d, ctypes.c_int, ctypes.c_int64, _i64, _d, _d, _d]
        L.oracle_energy.restype = ctypes.c_double
        L.oracle_element_bilinear.argtypes = [ctypes.c_int64, _d, ctypes.c_int, ctypes.c_int64, _i64,
                                               _d, _d, _d, _d, _d]
        L.oracle_element_bilinear.restype = None
        L.oracle_large_strain_run.argtypes = [ctypes.c_int64, _d, ctypes.c_int64, _i64, _d, _d, _u8, _d, _d,
                                              ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                              ctypes.c_int64, _d, _d, _i32, _i32, _d]
        L.oracle_large_strain_run.restype = ctypes.c_int
        L.oracle_large_strain_gradient.argtypes = [ctypes.c_int64, _d, ctypes.c_int64, _i64, _d, _d, _u8,
                                                   ctypes.c_int, _d, _d, ctypes.c_double, ctypes.c_int64,
                                                   _d, _d]
        L.oracle_large_strain_gradient.restype = ctypes.c_int
        L.oracle_neo_hookean_tet4.argtypes = [_d, ctypes.c_double, ctypes.c_double, _d, _d, _d, _d, _d]
        L.oracle_neo_hookean_tet4.restype = ctypes.c_int
        L.oracle_nodal_stresses.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_int64, _i64, _d, _d]
        L.oracle_thermal_transient.argtypes = [
            ctypes.c_int64, _d, ctypes.c_int, ctypes.c_int64, _i64, _d, _d, _u8, _d, _d,
            ctypes.c_int64, _i64, _d, ctypes.c_int64, _i64, _i32, _d, _d, _d,
            ctypes.c_double, ctypes.c_double, ctypes.c_int64, ctypes.c_int, ctypes.c_double,
            ctypes.c_int64, _d, _d, _d, _d, _i64, _d]
        L.oracle_thermal_transient.restype = ctypes.c_int
        L.oracle_tetra14.argtypes = [_d]
        L.oracle_thermal_element.argtypes = [ctypes.c_int, _d, ctypes.c_double, ctypes.c_double, _d, _d]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def element_stiffness(coords, young, nu):
    c = _c(coords, np.float64)
    npe = c.shape[0]
    ke = np.zeros((3 * npe, 3 * npe))
    lib().oracle_element_stiffness(npe, _p(c, _d), young, nu, _p(ke, _d))
    return ke


def element_stresses(coords, young, nu, u_e):
    c = _c(coords, np.float64)
    npe = c.shape[0]
    out = np.zeros((1 if npe == 4 else 4, 9))
    u = _c(u_e, np.float64)
    lib().oracle_element_stresses(npe, _p(c, _d), young, nu, _p(u, _d), _p(out, _d))
    return out


def von_mises(s9):
    s = _c(s9, np.float64)
    return lib().oracle_von_mises(_p(s, _d))


def face_pressure(coords, face, value):
    c = _c(coords, np.float64)
    pos = np.zeros(6, np.int32)
    forces = np.zeros(18)
    nn = lib().oracle_face_pressure(c.shape[0], _p(c, _d), face, value,
                                    pos.ctypes.data_as(_ip), _p(forces, _d))
    return pos[:nn].copy(), forces[:3 * nn].copy()


def dot(a, b):
    a = _c(a, np.float64)
    b = _c(b, np.float64)
    return lib().oracle_dot(_p(a, _d), _p(b, _d), a.size)


def graph_from_elements(n, elements):
    eoff = np.zeros(len(elements) + 1, np.int64)
    for k, e in enumerate(elements):
        eoff[k + 1] = eoff[k] + len(e)
    eidx = np.array([v for e in elements for v in e], np.int64)
    if eidx.size == 0:
        eidx = np.zeros(1, np.int64)
    off = np.zeros(n + 1, np.int64)
    cnt = lib().oracle_graph_from_elements(n, len(elements), _p(eoff, _i64), _p(eidx, _i64), _p(off, _i64), None)
    tgt = np.zeros(max(cnt, 1), np.int64)
    lib().oracle_graph_from_elements(n, len(elements), _p(eoff, _i64), _p(eidx, _i64), _p(off, _i64), _p(tgt, _i64))
    return off, tgt[:cnt]


def rcm(offsets, targets):
    off = _c(offsets, np.int64)
    tgt = _c(targets, np.int64) if len(targets) else np.zeros(1, np.int64)
    n = off.size - 1
    order = np.zeros(n, np.int64)
    lib().oracle_rcm(n, _p(off, _i64), _p(tgt, _i64), _p(order, _i64))
    return order


def csr_run(offsets, targets, triplets, b, mode=0, order=None, tol=1e-12):
    """Csr on the graph (numbered by `order`), filled by Csr::add(i, j, v) triplets.
    mode 0: Pcg solve, 1: IC(0) precondition, 2: multiply. Returns (status, x, iterations)."""
    off = _c(offsets, np.int64)
    tgt = _c(targets, np.int64) if len(targets) else np.zeros(1, np.int64)
    n = off.size - 1
    ti = np.array([t[0] for t in triplets], np.int64)
    tj = np.array([t[1] for t in triplets], np.int64)
    tv = np.array([t[2] for t in triplets], np.float64)
    bb = _c(b, np.float64)
    x = np.zeros(n)
    it = np.zeros(1, np.int64)
    o = _c(order, np.int64) if order is not None else None
    s = lib().oracle_csr_run(n, _p(off, _i64), _p(tgt, _i64), _p(o, _i64), ti.size, _p(ti, _i64),
                             _p(tj, _i64), _p(tv, _d), _p(bb, _d), mode, tol, _p(x, _d), _p(it, _i64))
    return s, x, int(it[0])


def model_solve(prob, solver: int = 2, tol: float = 1e-12, max_iter: int = 10000, dof_order=None):
    """Model::solve of a meshgen.Problem on the CPU. solver: 0 Auto, 1 Direct, 2 Iterative.

    Returns a dict with status, u, reactions, gauss (E, ngp, 9), von_mises (E, ngp), f,
    iterations, rel_residual, shift, free_dofs, nnz, ms_setup, ms_factor, ms_solve, wall_s.
    """
    L = lib()
    coords = _c(prob.coords, np.float64)
    conn = _c(prob.conn, np.int64)
    npe = conn.shape[1]
    ne = conn.shape[0]
    ng = 1 if npe == 4 else 4
    n = 3 * coords.shape[0]
    u = np.zeros(n)
    r = np.zeros(n)
    g = np.zeros((ne, ng, 9))
    vm = np.zeros((ne, ng))
    f = np.zeros(n)
    info = np.zeros(8)
    pe = _c(prob.p_elem, np.int64)
    pf = _c(prob.p_face, np.int32)
    pv = _c(prob.p_value, np.float64)
    order = _c(dof_order, np.int64) if dof_order is not None else None
    t0 = time.perf_counter()
    s = L.oracle_model_solve(
        coords.shape[0], _p(coords, _d), npe, ne, _p(conn, _i64), _p(_c(prob.young, np.float64), _d),
        _p(_c(prob.poisson, np.float64), _d), _p(_c(prob.fixed, np.uint8), _u8),
        _p(_c(prob.imposed, np.float64), _d), _p(_c(prob.loads, np.float64), _d),
        pe.size, _p(pe, _i64), _p(pf, _i32), _p(pv, _d), solver, tol, max_iter, _p(order, _i64),
        _p(u, _d), _p(r, _d), _p(g, _d), _p(vm, _d), _p(f, _d), _p(info, _d))
    wall = time.perf_counter() - t0
    return dict(status=s, u=u, reactions=r, gauss=g, von_mises=vm, f=f, iterations=int(info[0]),
                rel_residual=info[1], shift=info[2], free_dofs=int(info[3]), nnz=int(info[4]),
                ms_setup=info[5], ms_factor=info[6], ms_solve=info[7], wall_s=wall)


def energy(prob, v):
    """v^T K v summed element by element."""
    coords = _c(prob.coords, np.float64)
    conn = _c(prob.conn, np.int64)
    vv = _c(v, np.float64)
    return lib().oracle_energy(coords.shape[0], _p(coords, _d), conn.shape[1], conn.shape[0],
                               _p(conn, _i64), _p(_c(prob.young, np.float64), _d),
                               _p(_c(prob.poisson, np.float64), _d), _p(vv, _d))


def element_bilinear(prob, a, b):
    """a_e^T K_e b_e for every element (K_e of the element's own E and nu)."""
    coords = _c(prob.coords, np.float64)
    conn = _c(prob.conn, np.int64)
    out = np.zeros(conn.shape[0])
    lib().oracle_element_bilinear(coords.shape[0], _p(coords, _d), conn.shape[1], conn.shape[0],
                                  _p(conn, _i64), _p(_c(prob.young, np.float64), _d),
                                  _p(_c(prob.poisson, np.float64), _d), _p(_c(a, np.float64), _d),
                                  _p(_c(b, np.float64), _d), _p(out, _d))
    return out


def adjoint_gradient(prob, u, dJdu, tol: float = 1e-13, max_iter: int = 100000):
    """dJ/dE_e of a linear static solve u for an objective with gradient dJdu: the adjoint system
    K_ff lambda_f = (dJ/du)_f solved by the oracle's IC(0)-PCG (lambda = 0 on fixed DOFs, no
    pressure, no imposed values), then -lambda_e^T K_e u_e / E_e. Returns (gradient, lambda, info)."""
    adj = copy.copy(prob)
    adj.loads = np.ascontiguousarray(dJdu, np.float64).reshape(prob.loads.shape)
    adj.imposed = np.zeros_like(prob.imposed)
    adj.p_elem = np.zeros(0, np.int64)
    adj.p_face = np.zeros(0, np.int32)
    adj.p_value = np.zeros(0)
    res = model_solve(adj, solver=2, tol=tol, max_iter=max_iter)
    lam = res["u"]
    grad = -element_bilinear(prob, lam, u) / np.asarray(prob.young, np.float64)
    return grad, lam, res


def neo_hookean_tet4(coords, lam, mu, ue):
    """One neo-Hookean Tet4 response: (status, fe [12], ke [12, 12], dfe/dmu, dfe/dlambda)."""
    fe, ke, dm, dl = np.zeros(12), np.zeros((12, 12)), np.zeros(12), np.zeros(12)
    s = lib().oracle_neo_hookean_tet4(_p(_c(coords, np.float64), _d), lam, mu, _p(_c(ue, np.float64), _d),
                                      _p(fe, _d), _p(ke, _d), _p(dm, _d), _p(dl, _d))
    return s, fe, ke, dm, dl


def large_strain_run(prob, increments: int = 10, newton_tol: float = 1e-8, newton_max: int = 25,
                     pcg_tol: float = 1e-12, pcg_max: int = 10000):
    """Model::solve_quasi_static of a neo-Hookean Tet4 Problem (Kinematics::Large, linear ramp of
    the loads and imposed values over `increments` equal increments). Returns a dict: status,
    u_hist (increments, 3N) checkpoints, reactions (increments, 3N), newton (increments,), cuts,
    newton_total, pcg_total, wall_s, and for the increment the run stopped at (the last one on
    success): stop_increment and stop_cuts (its interval halvings)."""
    coords = _c(prob.coords, np.float64)
    conn = _c(prob.conn, np.int64)
    n = coords.size
    uh = np.zeros((increments, n))
    rh = np.zeros((increments, n))
    it = np.zeros(increments, np.int32)
    cuts = np.zeros(increments, np.int32)
    info = np.zeros(4)
    t0 = time.perf_counter()
    s = lib().oracle_large_strain_run(
        coords.shape[0], _p(coords, _d), conn.shape[0], _p(conn, _i64), _p(_c(prob.young, np.float64), _d),
        _p(_c(prob.poisson, np.float64), _d), _p(_c(prob.fixed, np.uint8), _u8),
        _p(_c(prob.imposed, np.float64), _d), _p(_c(prob.loads, np.float64), _d), increments, newton_tol,
        newton_max, pcg_tol, pcg_max, _p(uh, _d), _p(rh, _d), _p(it, _i32), _p(cuts, _i32), _p(info, _d))
    return dict(status=s, u_hist=uh, reactions=rh, newton=it, cuts=cuts, newton_total=int(info[0]),
                pcg_total=int(info[1]), stop_cuts=int(info[2]), stop_increment=int(info[3]),
                wall_s=time.perf_counter() - t0)


def large_strain_gradient(prob, u_hist, dJdR, pcg_tol: float = 1e-12, pcg_max: int = 10000):
    """dJ/dmu_e and dJ/dlambda_e of J = sum_k dJdR[k] . R_k over the checkpoints u_hist."""
    coords = _c(prob.coords, np.float64)
    conn = _c(prob.conn, np.int64)
    gm = np.zeros(conn.shape[0])
    gl = np.zeros(conn.shape[0])
    uh = _c(u_hist, np.float64)
    s = lib().oracle_large_strain_gradient(
        coords.shape[0], _p(coords, _d), conn.shape[0], _p(conn, _i64), _p(_c(prob.young, np.float64), _d),
        _p(_c(prob.poisson, np.float64), _d), _p(_c(prob.fixed, np.uint8), _u8), uh.shape[0], _p(uh, _d),
        _p(_c(dJdR, np.float64), _d), pcg_tol, pcg_max, _p(gm, _d), _p(gl, _d))
    return s, gm, gl


def nodal_stresses(prob, gauss):
    conn = _c(prob.conn, np.int64)
    g = _c(gauss, np.float64)
    out = np.zeros((prob.coords.shape[0], 6))
    lib().oracle_nodal_stresses(prob.coords.shape[0], conn.shape[1], conn.shape[0], _p(conn, _i64),
                                _p(g, _d), _p(out, _d))
    return out


def tetra14():
    """TETRA_14 as a (14, 4) array of (xi, eta, zeta, weight)."""
    out = np.zeros((14, 4))
    lib().oracle_tetra14(_p(out, _d))
    return out


def thermal_element(coords, k, rho_c):
    """(conduction K_e, capacity C_e) of one Tet4/Tet10 element (coords (npe, 3))."""
    c = _c(coords, np.float64)
    npe = c.shape[0]
    ke = np.zeros((npe, npe))
    ce = np.zeros((npe, npe))
    lib().oracle_thermal_element(npe, _p(c, _d), k, rho_c, _p(ke, _d), _p(ce, _d))
    return ke, ce


def thermal_transient(prob, solver: int = 0, tol: float = 1e-12, max_iter: int = 10000,
                      fluxes: bool = True):
    """Model::solve_step of a meshgen.ThermalProblem on the CPU. solver: 0 Auto, 1 Direct,
    2 Iterative. Returns a dict with status, temps (S + 1, N), reactions (S + 1, N), fluxes
    (S + 1, E, ngp, 6) or None, f, iterations (S,), total_iterations, rel_residual, shift,
    free, nnz, ms_setup, ms_factor, ms_steps, wall_s."""
    L = lib()
    coords = _c(prob.coords, np.float64)
    conn = _c(prob.conn, np.int64)
    n, (ne, npe) = coords.shape[0], conn.shape
    ng = 1 if npe == 4 else 4
    steps = int(prob.increments)
    temps = np.zeros((steps + 1, n))
    reac = np.zeros((steps + 1, n))
    flux = np.zeros((steps + 1, ne, ng, 6)) if fluxes else None
    f = np.zeros(n)
    its = np.zeros(max(steps, 1), np.int64)
    info = np.zeros(8)
    se, sv = _c(prob.s_elem, np.int64), _c(prob.s_value, np.float64)
    ce, cf = _c(prob.c_elem, np.int64), _c(prob.c_face, np.int32)
    ch, cs = _c(prob.c_film, np.float64), _c(prob.c_sink, np.float64)
    t0 = time.perf_counter()
    s = L.oracle_thermal_transient(
        n, _p(coords, _d), npe, ne, _p(conn, _i64), _p(_c(prob.conductivity, np.float64), _d),
        _p(_c(prob.rho_c, np.float64), _d), _p(_c(prob.fixed, np.uint8), _u8),
        _p(_c(prob.imposed, np.float64), _d), _p(_c(prob.loads, np.float64), _d),
        se.size, _p(se, _i64), _p(sv, _d), ce.size, _p(ce, _i64), _p(cf, _i32), _p(ch, _d), _p(cs, _d),
        _p(_c(prob.initial, np.float64), _d), prob.time_step, prob.theta, steps, solver, tol,
        max_iter, _p(temps, _d), _p(reac, _d), _p(flux, _d), _p(f, _d), _p(its, _i64), _p(info, _d))
    wall = time.perf_counter() - t0
    return dict(status=s, temps=temps, reactions=reac, fluxes=flux, f=f, iterations=its[:steps],
                total_iterations=int(info[0]), rel_residual=info[1], shift=info[2],
                free=int(info[3]), nnz=int(info[4]), ms_setup=info[5], ms_factor=info[6],
                ms_steps=info[7], wall_s=wall)
