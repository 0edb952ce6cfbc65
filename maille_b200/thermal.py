"""Host-side mirror of maille-core's transient thermal interface for the GPU path.

Names and argument meaning follow the reference (crates/maille-core/src/model.rs): `Step` with
`transient`, `with_theta`, `time_step` (model.rs:119-173), `HeatSource` and `Convection`
(model.rs:44-66), `Model::solve_step` (model.rs:621-706) returning one `Increment` per step
after the t = 0 one (results.rs). `ThermalModel.solve_step` sends the whole step to the CUDA
library (maille_gpu_thermal_transient); the heat-source and convection loads of the reference's
`assemble` are added on the host by the library's helper (maille_gpu_thermal_loads).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import MAILLE_ORDER_AUTO, ThermalProblem, ThermalResult, ptr
from .model import MailleError, _STATUS_KIND, _raise_for


@dataclass
class Step:
    """A transient step: `time_period` in `increments` equal steps, theta-method with theta in
    [1/2, 1] (1: backward Euler, the default; 1/2: Crank-Nicolson)."""
    time_period: float
    increments: int
    theta: float = 1.0

    @staticmethod
    def transient(time_period: float, increments: int) -> "Step":
        if not (math.isfinite(time_period) and time_period > 0.0):
            raise MailleError("InvalidProperty", f"time period {time_period}")
        if increments <= 0:
            raise MailleError("NoIncrements")
        return Step(float(time_period), int(increments), 1.0)

    def with_theta(self, theta: float) -> "Step":
        if not (0.5 <= theta <= 1.0):
            raise MailleError("ThetaOutOfRange", f"theta {theta}")
        return Step(self.time_period, self.increments, float(theta))

    @property
    def time_step(self) -> float:
        return self.time_period / self.increments


@dataclass
class HeatSource:
    """Uniform heat source `value` (power per volume) in element `element`."""
    element: int
    value: float


@dataclass
class Convection:
    """h (T - T_inf) on face `face` (0-1-2, 0-3-1, 1-3-2, 2-3-0) of element `element`."""
    element: int
    face: int
    film: float
    sink: float


@dataclass
class Increment:
    """One increment of a transient step: time, nodal temperatures, reactions (heat supplied at
    imposed nodes) and Gauss-point heat fluxes (E, ngp, 6) of x, y, z, qx, qy, qz."""
    time: float
    temperatures: np.ndarray
    reactions: np.ndarray
    heat_fluxes: np.ndarray | None
    iterations: int = 0


def thermal_loads(coords, conn, sources=(), convection=()) -> np.ndarray:
    """Heat-source and convection loads of the reference's assemble (model.rs:1110-1140) as a
    nodal vector: sources as (element, q) pairs, convection as (element, face, film, sink)."""
    L = _lib.load()
    coords = np.ascontiguousarray(coords, np.float64)
    conn = np.ascontiguousarray(conn, np.int64)
    se = np.ascontiguousarray([s[0] for s in sources], np.int64)
    sv = np.ascontiguousarray([s[1] for s in sources], np.float64)
    ce = np.ascontiguousarray([c[0] for c in convection], np.int64)
    cf = np.ascontiguousarray([c[1] for c in convection], np.int32)
    ch = np.ascontiguousarray([c[2] for c in convection], np.float64)
    cs = np.ascontiguousarray([c[3] for c in convection], np.float64)
    f = np.zeros(coords.shape[0])
    s = L.maille_gpu_thermal_loads(coords.shape[0], ptr(coords, _lib._d), conn.shape[1], conn.shape[0],
                                   ptr(conn, _lib._i64), se.size, ptr(se, _lib._i64),
                                   ptr(sv, _lib._d), ce.size, ptr(ce, _lib._i64), ptr(cf, _lib._i32),
                                   ptr(ch, _lib._d), ptr(cs, _lib._d), ptr(f, _lib._d))
    if s != 0:
        raise MailleError(_STATUS_KIND.get(s, "Unknown"), _lib.last_error())
    return f


def thermal_problem_struct(coords, conn, conductivity, rho_c, fixed, imposed, f, initial, time_step,
                           theta, increments, conv_elem=None, conv_face=None, conv_film=None,
                           tol=1e-12, max_iter=10000, ordering=MAILLE_ORDER_AUTO, device=0, precision=0):
    """ThermalProblem over numpy arrays (kept alive in the returned dict)."""
    conn_a = np.asarray(conn)
    keep = dict(coords=np.ascontiguousarray(coords, np.float64).ravel(),
                conn=np.ascontiguousarray(conn, np.int64).ravel(),
                k=np.ascontiguousarray(conductivity, np.float64),
                rc=np.ascontiguousarray(rho_c, np.float64),
                fixed=np.ascontiguousarray(fixed, np.uint8),
                imposed=np.ascontiguousarray(imposed, np.float64),
                f=np.ascontiguousarray(f, np.float64) if f is not None else None,
                initial=np.ascontiguousarray(initial, np.float64),
                ce=np.ascontiguousarray(conv_elem if conv_elem is not None else [], np.int64),
                cf=np.ascontiguousarray(conv_face if conv_face is not None else [], np.int32),
                ch=np.ascontiguousarray(conv_film if conv_film is not None else [], np.float64))
    p = ThermalProblem(
        n_nodes=keep["coords"].size // 3, coords=ptr(keep["coords"], _lib._d), nodes_per_elem=conn_a.shape[1],
        n_elems=conn_a.shape[0], conn=ptr(keep["conn"], _lib._i64), conductivity=ptr(keep["k"], _lib._d),
        rho_c=ptr(keep["rc"], _lib._d), fixed=ptr(keep["fixed"], _lib._u8), imposed=ptr(keep["imposed"], _lib._d),
        f=ptr(keep["f"], _lib._d), n_convection=keep["ce"].size, conv_elem=ptr(keep["ce"], _lib._i64),
        conv_face=ptr(keep["cf"], _lib._i32), conv_film=ptr(keep["ch"], _lib._d),
        initial=ptr(keep["initial"], _lib._d), time_step=time_step, theta=theta, increments=increments,
        rel_tol=tol, max_iter=max_iter, ordering=ordering, device=device, precision=precision)
    return p, keep


def solve_problem(prob, f=None, tol=1e-12, max_iter=10000, fluxes=True, device=0,
                  ordering=MAILLE_ORDER_AUTO, out=None, precision=0):
    """The transient step of a meshgen.ThermalProblem on the GPU. `f` is the assembled heat-load
    vector (None: nodal loads plus the problem's sources and convection through
    thermal_loads). `out` may hold preallocated result arrays (temps, reactions, fluxes,
    iterations; pinned host memory makes the copies back faster). Returns (status, dict of temps
    (S + 1, N), reactions (S + 1, N), fluxes (S + 1, E, ngp, 6) or None, iterations (S,),
    info)."""
    L = _lib.load()
    n, ne, npe = prob.n_nodes, prob.n_elems, prob.npe
    ng = 1 if npe == 4 else 4
    steps = int(prob.increments)
    if f is None:
        f = np.asarray(prob.loads, np.float64) + thermal_loads(
            prob.coords, prob.conn, list(zip(prob.s_elem, prob.s_value)),
            list(zip(prob.c_elem, prob.c_face, prob.c_film, prob.c_sink)))
    p, keep = thermal_problem_struct(prob.coords, prob.conn, prob.conductivity, prob.rho_c, prob.fixed,
                                     prob.imposed, f, prob.initial, prob.time_step, prob.theta, steps,
                                     prob.c_elem, prob.c_face, prob.c_film, tol, max_iter, ordering, device,
                                     precision)
    if out is None:
        out = dict(temps=np.zeros((steps + 1, n)), reactions=np.zeros((steps + 1, n)),
                   fluxes=np.zeros((steps + 1, ne, ng, 6)) if fluxes else None,
                   iterations=np.zeros(steps, np.int32))
    r = ThermalResult(temperatures=ptr(out["temps"], _lib._d), reactions=ptr(out["reactions"], _lib._d),
                      heat_fluxes=ptr(out["fluxes"], _lib._d), iterations=ptr(out["iterations"], _lib._i32))
    s = L.maille_gpu_thermal_transient(ctypes.byref(p), ctypes.byref(r))
    out["info"] = {k: getattr(r, k) for k, _ in ThermalResult._fields_
                   if k not in ("temperatures", "reactions", "heat_fluxes", "iterations")}
    return s, out


def cancel(flag: bool = True, device: int = 0):
    """Raises (or clears) the thermal cancel flag of `device`: every transient step on that device
    stops before its next increment and returns status MAILLE_CANCELLED (MailleError("Cancelled")
    from ThermalModel.solve_step), with the increments completed before it. The flag stays raised
    until cleared."""
    _raise_for(_lib.load().maille_gpu_thermal_cancel(device, 1 if flag else 0))


class ThermalModel:
    """Model with Analysis::Thermal (one DOF T per node) on a Tet4/Tet10 mesh, restricted to the
    transient path: coords (N, 3), conn (E, 4|10), per-element conductivity k and rho_c
    (density x specific heat); bcs as (node, value) imposed temperatures, loads as (node, value)
    nodal heat loads."""

    def __init__(self, coords, conn, conductivity, rho_c, bcs=(), loads=()):
        self.coords = np.ascontiguousarray(coords, np.float64).reshape(-1, 3)
        self.conn = np.ascontiguousarray(conn, np.int64)
        ne = self.conn.shape[0]
        self.conductivity = np.ascontiguousarray(np.broadcast_to(np.asarray(conductivity, np.float64), (ne,)))
        self.rho_c = np.ascontiguousarray(np.broadcast_to(np.asarray(rho_c, np.float64), (ne,)))
        n = self.coords.shape[0]
        self.fixed = np.zeros(n, np.uint8)
        self.imposed = np.zeros(n)
        self.loads = np.zeros(n)
        for node, value in bcs:
            if not 0 <= node < n:
                raise MailleError("UnknownNode", f"node {node}")
            self.fixed[node] = 1
            self.imposed[node] = value
        for node, value in loads:
            if not 0 <= node < n:
                raise MailleError("UnknownNode", f"node {node}")
            self.loads[node] += value
        self.sources: list[HeatSource] = []
        self.convection: list[Convection] = []
        self.tolerance = 1e-12
        self.max_iterations = 10000

    def with_heat_sources(self, sources) -> "ThermalModel":
        self.sources = list(sources)
        return self

    def with_convection(self, convection) -> "ThermalModel":
        for c in convection:
            if not (c.film > 0.0 and math.isfinite(c.film)) or not math.isfinite(c.sink):
                raise MailleError("InvalidProperty", f"film {c.film}, sink {c.sink}")
        self.convection = list(convection)
        return self

    def solve(self, device: int = 0, fluxes: bool = True) -> Increment:
        """Model::solve of the thermal model (model.rs:548-610): K T = F with the imposed
        temperatures, reactions K T - F on the imposed nodes and the heat fluxes. It is the
        transient step with no capacity, theta = 1 and one increment (left matrix K, right
        matrix 0), so it runs on the same device path."""
        steady = ThermalModel.__new__(ThermalModel)
        steady.__dict__.update(self.__dict__)
        steady.rho_c = np.zeros_like(self.rho_c)
        hist = steady.solve_step(Step(1.0, 1, 1.0), np.zeros(self.coords.shape[0]), device=device, fluxes=fluxes)
        return hist[1]

    def solve_step(self, step: Step, initial, device: int = 0, fluxes: bool = True) -> list[Increment]:
        """Model::solve_step (model.rs:621-706): the t = 0 increment, then one per step."""
        initial = np.asarray(initial, np.float64)
        n = self.coords.shape[0]
        if initial.shape != (n,):
            raise MailleError("TemperatureCount", f"expected {n}, got {initial.size}")
        if not np.isfinite(initial).all():
            raise MailleError("NonFiniteTemperature", f"node {int(np.nonzero(~np.isfinite(initial))[0][0])}")
        f = self.loads + thermal_loads(self.coords, self.conn, [(s.element, s.value) for s in self.sources],
                                       [(c.element, c.face, c.film, c.sink) for c in self.convection])
        from .meshgen import ThermalProblem as _TP
        prob = _TP(coords=self.coords, conn=self.conn, conductivity=self.conductivity, rho_c=self.rho_c,
                   fixed=self.fixed, imposed=self.imposed, loads=self.loads, initial=initial,
                   time_period=step.time_period, increments=step.increments, theta=step.theta,
                   c_elem=np.array([c.element for c in self.convection], np.int64),
                   c_face=np.array([c.face for c in self.convection], np.int32),
                   c_film=np.array([c.film for c in self.convection], np.float64),
                   c_sink=np.array([c.sink for c in self.convection], np.float64))
        s, out = solve_problem(prob, f=f, tol=self.tolerance, max_iter=self.max_iterations, fluxes=fluxes,
                               device=device)
        if s != 0:
            raise MailleError(_STATUS_KIND.get(s, "Unknown"), _lib.last_error())
        hist = []
        for k in range(step.increments + 1):
            hist.append(Increment(time=k * step.time_step, temperatures=out["temps"][k],
                                  reactions=out["reactions"][k],
                                  heat_fluxes=out["fluxes"][k] if fluxes else None,
                                  iterations=int(out["iterations"][k - 1]) if k > 0 else 0))
        return hist
