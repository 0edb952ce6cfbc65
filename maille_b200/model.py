"""Host-side mirror of maille-core's solve interface for the GPU path.

Names and argument meaning follow the reference (crates/maille-core/src): `SolverKind` and
`ITERATIVE_FROM` (solve.rs:170-195), `Model::new / with_solver / with_pressures / solve`
(model.rs:251-610), `Field` and `Stress` (results.rs:6-76), the `MailleError` variants on this path
(error.rs:156, 224-229). `Model.solve` sends the iterative branch (`SolverKind.is_iterative`) to the
CUDA library through its C ABI; the skyline direct solver is not part of this library and stays in
the host program, so a model that selects it raises `MailleError("DirectSolverOnHost")`.
"""
from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import (ElasticProblem, ElasticResult, MAILLE_CANCELLED, MAILLE_FP64, MAILLE_MIXED,
                   MAILLE_NOT_CONVERGED, MAILLE_OK, MAILLE_ORDER_AUTO, MAILLE_SINGULAR, ptr)

ITERATIVE_FROM = 100_000  # solve.rs:185


class SolverKind(enum.Enum):
    """solve.rs:170-195: Auto picks the iterative solver from ITERATIVE_FROM free DOFs."""
    AUTO = 0
    DIRECT = 1
    ITERATIVE = 2

    def is_iterative(self, free_dofs: int) -> bool:
        if self is SolverKind.AUTO:
            return free_dofs >= ITERATIVE_FROM
        return self is SolverKind.ITERATIVE


class Dof(enum.IntEnum):
    UX = 0
    UY = 1
    UZ = 2


class MailleError(Exception):
    """Errors of this path: Singular, IterativeNotConverged{iterations, residual}, Cancelled,
    InvalidInput (mesh/model validation), Cuda, DirectSolverOnHost."""

    def __init__(self, kind: str, message: str = "", iterations: int = 0, residual: float = 0.0):
        super().__init__(f"{kind}: {message}" if message else kind)
        self.kind = kind
        self.iterations = iterations
        self.residual = residual


_STATUS_KIND = {1: "Singular", 2: "IterativeNotConverged", 3: "InvalidInput", 4: "Cuda",
                5: "Cancelled"}


def _raise_for(status: int, res: ElasticResult | None = None):
    if status == MAILLE_OK:
        return
    kind = _STATUS_KIND.get(status, "Unknown")
    it = res.iterations if res is not None else 0
    rr = res.final_rel_residual if res is not None else 0.0
    raise MailleError(kind, _lib.last_error(), iterations=it, residual=rr)


@dataclass
class Material:
    young: float
    poisson: float

    @staticmethod
    def with_poisson(young: float, poisson: float) -> "Material":
        if not (young > 0 and -1.0 < poisson < 0.5):
            raise MailleError("InvalidMaterial", f"E={young}, nu={poisson}")
        return Material(float(young), float(poisson))


@dataclass
class Bc:
    node: int
    dof: Dof
    value: float


@dataclass
class Load:
    node: int
    dof: Dof
    value: float


@dataclass
class Pressure:
    """Pressure `value` on face `face` (0-1-2, 0-3-1, 1-3-2, 2-3-0) of element `element`;
    positive compresses (assembly.rs:650-674)."""
    element: int
    face: int
    value: float


class Mesh:
    """Tet4 or Tet10 solid mesh held as arrays: coords (N, 3), conn (E, 4|10) in Maille node order,
    per-element young and poisson (each Tet carries its Material, mesh.rs:126-149)."""

    def __init__(self, coords, conn, young, poisson):
        self.coords = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
        self.conn = np.ascontiguousarray(conn, dtype=np.int64)
        ne = self.conn.shape[0]
        self.young = np.ascontiguousarray(np.broadcast_to(np.asarray(young, np.float64), (ne,)))
        self.poisson = np.ascontiguousarray(np.broadcast_to(np.asarray(poisson, np.float64), (ne,)))
        self._validate()

    def _validate(self):
        """The checks of Mesh::new on this path (mesh.rs:257-348): non-empty, finite
        coordinates, known nodes, one family, no degenerate or inverted tet, straight Tet10."""
        if self.coords.shape[0] == 0 or self.conn.shape[0] == 0:
            raise MailleError("EmptyMesh")
        if self.conn.ndim != 2 or self.conn.shape[1] not in (4, 10):
            raise MailleError("MixedElementTypes", "Tet4 or Tet10 connectivity expected")
        if not np.isfinite(self.coords).all():
            node = int(np.nonzero(~np.isfinite(self.coords).all(axis=1))[0][0])
            raise MailleError("NonFiniteCoordinate", f"node {node}")
        bad = (self.conn < 0) | (self.conn >= self.coords.shape[0])
        if bad.any():
            raise MailleError("UnknownNode", f"node {int(self.conn[bad][0])}")
        c = self.coords[self.conn[:, :4]]
        e = c[:, 1:] - c[:, :1]
        six_v = np.einsum("ij,ij->i", e[:, 0], np.cross(e[:, 1], e[:, 2]))
        edges = [(0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3)]
        longest = np.max([np.linalg.norm(c[:, a] - c[:, b], axis=1) for a, b in edges], axis=0)
        degenerate = np.abs(six_v) <= 1e-12 * longest ** 3
        if degenerate.any():
            raise MailleError("DegenerateTetrahedron", f"element {int(np.nonzero(degenerate)[0][0])}")
        if (six_v < 0).any():
            raise MailleError("InvertedTetrahedron", f"element {int(np.nonzero(six_v < 0)[0][0])}")
        if self.conn.shape[1] == 10:
            mids = self.coords[self.conn[:, 4:]]
            for k, (a, b) in enumerate(edges):
                m = 0.5 * (c[:, a] + c[:, b])
                off = np.linalg.norm(mids[:, k] - m, axis=1)
                bad = off > 1e-9 * np.linalg.norm(c[:, a] - c[:, b], axis=1)
                if bad.any():
                    raise MailleError("CurvedTetrahedron", f"element {int(np.nonzero(bad)[0][0])}")

    @property
    def npe(self) -> int:
        return int(self.conn.shape[1])


@dataclass
class Field:
    """Results of a static solve (results.rs:51-76): displacements and reactions (3 per node),
    Gauss-point stresses as an array (E, ngp, 9) of x, y, z, sxx, syy, szz, txy, tyz, txz, and
    their von Mises values (E, ngp)."""
    displacements: np.ndarray
    reactions: np.ndarray
    stresses: np.ndarray
    von_mises: np.ndarray
    info: dict = field(default_factory=dict)


def problem_struct(coords, conn, young, poisson, fixed, imposed, f, tol=1e-12, max_iter=10000,
                   precision=MAILLE_FP64, ordering=MAILLE_ORDER_AUTO, device=0):
    """ElasticProblem over numpy arrays (kept alive in the returned tuple)."""
    keep = dict(coords=np.ascontiguousarray(coords, np.float64).ravel(),
                conn=np.ascontiguousarray(conn, np.int64).ravel(),
                young=np.ascontiguousarray(young, np.float64),
                poisson=np.ascontiguousarray(poisson, np.float64),
                fixed=np.ascontiguousarray(fixed, np.uint8),
                imposed=np.ascontiguousarray(imposed, np.float64),
                f=np.ascontiguousarray(f, np.float64) if f is not None else None)
    conn_a = np.asarray(conn)
    p = ElasticProblem(
        n_nodes=keep["coords"].size // 3, coords=ptr(keep["coords"], _lib._d),
        nodes_per_elem=conn_a.shape[1], n_elems=conn_a.shape[0], conn=ptr(keep["conn"], _lib._i64),
        young=ptr(keep["young"], _lib._d), poisson=ptr(keep["poisson"], _lib._d),
        fixed=ptr(keep["fixed"], _lib._u8), imposed=ptr(keep["imposed"], _lib._d),
        f=ptr(keep["f"], _lib._d), rel_tol=tol, max_iter=max_iter, precision=precision,
        ordering=ordering, device=device)
    return p, keep


def face_pressure_loads(coords, conn, pressures) -> np.ndarray:
    """Nodal forces of the face pressures (element, face, value) (assembly.rs:650-674)."""
    L = _lib.load()
    coords = np.ascontiguousarray(coords, np.float64)
    conn = np.ascontiguousarray(conn, np.int64)
    pe = np.ascontiguousarray([p[0] for p in pressures], np.int64)
    pf = np.ascontiguousarray([p[1] for p in pressures], np.int32)
    pv = np.ascontiguousarray([p[2] for p in pressures], np.float64)
    f = np.zeros(coords.size)
    s = L.maille_gpu_face_pressure_loads(coords.shape[0], ptr(coords, _lib._d), conn.shape[1],
                                         conn.shape[0], ptr(conn, _lib._i64), pe.size,
                                         ptr(pe, _lib._i64), ptr(pf, _lib._i32), ptr(pv, _lib._d),
                                         ptr(f, _lib._d))
    _raise_for(s)
    return f


def _result_struct(n_nodes, n_elems, ngp):
    out = dict(u=np.zeros(3 * n_nodes), reactions=np.zeros(3 * n_nodes),
               gauss=np.zeros((n_elems, ngp, 9)), vm=np.zeros((n_elems, ngp)))
    r = ElasticResult(u=ptr(out["u"], _lib._d), reactions=ptr(out["reactions"], _lib._d),
                      gauss_stress=ptr(out["gauss"], _lib._d), von_mises=ptr(out["vm"], _lib._d))
    return r, out


def _info(r: ElasticResult) -> dict:
    return {k: getattr(r, k) for k, _ in ElasticResult._fields_ if k not in
            ("u", "reactions", "gauss_stress", "von_mises")}


class Model:
    """Linear static model (Model::new, model.rs:251-311) restricted to this path."""

    def __init__(self, mesh: Mesh, bcs=(), loads=()):
        self.mesh = mesh
        self.bcs = list(bcs)
        self.loads = list(loads)
        self.pressures: list = []
        self.solver = SolverKind.AUTO
        self.precision = MAILLE_FP64
        self.ordering = MAILLE_ORDER_AUTO
        self.tolerance = 1e-12
        self.max_iterations = 10000
        n = mesh.coords.shape[0]
        for b in self.bcs:
            if not 0 <= b.node < n:
                raise MailleError("UnknownNode", f"node {b.node}")
        for l in self.loads:
            if not 0 <= l.node < n:
                raise MailleError("UnknownNode", f"node {l.node}")

    def with_solver(self, kind: SolverKind) -> "Model":
        self.solver = kind
        return self

    def with_pressures(self, pressures) -> "Model":
        self.pressures = list(pressures)
        return self

    def with_precision(self, precision: int) -> "Model":
        """MAILLE_FP64 (plain form) or MAILLE_MIXED (FP32 PCG in FP64 refinement)."""
        self.precision = precision
        return self

    def with_tolerance(self, tol: float) -> "Model":
        self.tolerance = tol
        return self

    @classmethod
    def from_arrays(cls, coords, conn, young, poisson, fixed, imposed=None, loads=None,
                    pressures=None) -> "Model":
        """Model from whole arrays: fixed (3N) mask, imposed (3N), nodal loads (3N), pressures
        as an (element, face, value) list or a tuple of three arrays."""
        m = cls(Mesh(coords, conn, young, poisson))
        n3 = m.mesh.coords.size
        m._fixed = np.ascontiguousarray(fixed, np.uint8).reshape(n3)
        m._imposed = np.zeros(n3) if imposed is None else np.asarray(imposed, np.float64).reshape(n3)
        m._nodal = np.zeros(n3) if loads is None else np.asarray(loads, np.float64).reshape(n3)
        if pressures is not None:
            if isinstance(pressures, tuple) and len(pressures) == 3 and hasattr(pressures[0], "__len__"):
                pressures = list(zip(*pressures))
            m.pressures = [Pressure(int(e), int(f), float(v)) for e, f, v in pressures]
        return m

    def _arrays(self):
        n3 = self.mesh.coords.size
        if hasattr(self, "_fixed"):
            fixed, imposed, f = self._fixed.copy(), self._imposed.copy(), self._nodal.copy()
        else:
            fixed = np.zeros(n3, np.uint8)
            imposed = np.zeros(n3)
            f = np.zeros(n3)
            for l in self.loads:
                f[3 * l.node + int(l.dof)] += l.value
            for b in self.bcs:
                g = 3 * b.node + int(b.dof)
                imposed[g] = b.value
                fixed[g] = 1
        if self.pressures:
            f = f + face_pressure_loads(self.mesh.coords, self.mesh.conn,
                                        [(p.element, p.face, p.value) for p in self.pressures])
        return fixed, imposed, f

    def free_dofs(self) -> int:
        fixed, _, _ = self._arrays()
        return int(fixed.size - np.count_nonzero(fixed))

    def solve(self, device: int = 0) -> Field:
        """Model::solve (model.rs:548-610) through the GPU path."""
        fixed, imposed, f = self._arrays()
        free = int(fixed.size - np.count_nonzero(fixed))
        if not self.solver.is_iterative(free):
            raise MailleError("DirectSolverOnHost",
                              "the skyline Cholesky solver stays in the host program")
        L = _lib.load()
        mesh = self.mesh
        p, keep = problem_struct(mesh.coords, mesh.conn, mesh.young, mesh.poisson, fixed, imposed,
                                 f, self.tolerance, self.max_iterations, self.precision,
                                 self.ordering, device)
        ngp = 1 if mesh.npe == 4 else 4
        r, out = _result_struct(mesh.coords.shape[0], mesh.conn.shape[0], ngp)
        s = L.maille_gpu_elastic_solve(ctypes.byref(p), ctypes.byref(r))
        _raise_for(s, r)
        return Field(out["u"], out["reactions"], out["gauss"], out["vm"], _info(r))


class SolverHandle:
    """Reusable GPU solve handle (create / solve / backward / destroy of the C ABI): one
    analysis, factorisation and set of device buffers for many right-hand sides and adjoints."""

    def __init__(self, model: Model, device: int = 0):
        self._L = _lib.load()
        self.model = model
        fixed, imposed, f = model._arrays()
        self._f = f
        mesh = model.mesh
        self._p, self._keep = problem_struct(mesh.coords, mesh.conn, mesh.young, mesh.poisson,
                                             fixed, imposed, f, model.tolerance,
                                             model.max_iterations, model.precision,
                                             model.ordering, device)
        self._h = ctypes.c_void_p()
        s = self._L.maille_gpu_create(ctypes.byref(self._p), ctypes.byref(self._h))
        _raise_for(s)
        self.ngp = 1 if mesh.npe == 4 else 4

    def solve(self, f=None) -> Field:
        mesh = self.model.mesh
        r, out = _result_struct(mesh.coords.shape[0], mesh.conn.shape[0], self.ngp)
        fa = None if f is None else np.ascontiguousarray(f, np.float64).ravel()
        s = self._L.maille_gpu_solve(self._h, ptr(fa, _lib._d), ctypes.byref(r))
        _raise_for(s, r)
        return Field(out["u"], out["reactions"], out["gauss"], out["vm"], _info(r))

    def nodal_stresses(self):
        """Smoothed nodal stresses of the last solve (nodal_stresses, results.rs:137-230):
        returns (stress (n, 6) as sxx, syy, szz, txy, tyz, txz; von_mises (n,))."""
        n = self.model.mesh.coords.shape[0]
        st = np.zeros(6 * n)
        vm = np.zeros(n)
        s = self._L.maille_gpu_nodal_stresses(self._h, ptr(st, _lib._d), ptr(vm, _lib._d))
        _raise_for(s)
        return st.reshape(n, 6), vm

    def backward(self, dJdu):
        """dJ/dE per element for J with gradient dJ/du (adjoint of the last solve);
        returns (dJdE, lambda)."""
        g = np.ascontiguousarray(dJdu, np.float64).ravel()
        ne = self.model.mesh.conn.shape[0]
        dJdE = np.zeros(ne)
        lam = np.zeros(g.size)
        s = self._L.maille_gpu_backward(self._h, ptr(g, _lib._d), ptr(dJdE, _lib._d),
                                        ptr(lam, _lib._d))
        _raise_for(s)
        return dJdE, lam

    def refactor(self, young=None, poisson=None):
        """New per-element materials on the same mesh and constraints: element integration,
        assembly and IC(0) again, reusing the ordering and scatter map."""
        ne = self.model.mesh.conn.shape[0]
        ya = None if young is None else np.ascontiguousarray(young, np.float64).ravel()
        pa = None if poisson is None else np.ascontiguousarray(poisson, np.float64).ravel()
        for a in (ya, pa):
            if a is not None and a.size != ne:
                raise MailleError("InvalidInput", f"{a.size} material values for {ne} elements")
        s = self._L.maille_gpu_refactor(self._h, ptr(ya, _lib._d), ptr(pa, _lib._d))
        _raise_for(s)
        if ya is not None:
            self.model.mesh.young = ya.copy()
        if pa is not None:
            self.model.mesh.poisson = pa.copy()

    def cancel(self, flag: bool = True):
        self._L.maille_gpu_cancel(self._h, 1 if flag else 0)

    @property
    def stream(self) -> int:
        return int(self._L.maille_gpu_stream(self._h) or 0)

    def close(self):
        if self._h:
            self._L.maille_gpu_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
