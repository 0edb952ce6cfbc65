"""Large strain (neo-Hookean Tet4) quasi-static solves and their adjoint on the GPU
(maille_gpu_large_strain_* of include/maille_gpu.h).

Mirrors Model::solve_quasi_static with Kinematics::Large and Hyperelasticity::NeoHookean
(crates/maille-core/src/model.rs:720-1022, finite_strain.rs): `LargeStrainSolver(problem,
increments).run()` returns the converged displacements and reactions of every increment;
`backward(dJdR)` returns dJ/dmu_e and dJ/dlambda_e for an objective J = sum_k dJdR[k] . R_k of the
increment reactions (the reference has no gradients).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import MAILLE_FP64, ptr, _d, _i32, _i64, _u8
from .model import MailleError, _raise_for


@dataclass
class LargeStrainHistory:
    displacements: np.ndarray   # (increments, 3 N)
    reactions: np.ndarray       # (increments, 3 N), F_int - lambda F at fixed DOFs
    newton: np.ndarray          # (increments,) residuals of each increment's last equilibrium
    cuts: np.ndarray            # (increments,)
    newton_total: int
    pcg_total: int
    ms_total: float


def lame(young, poisson):
    """(lambda, mu) of E and nu (finite_strain.rs:30-35)."""
    young = np.asarray(young, np.float64)
    poisson = np.asarray(poisson, np.float64)
    return young * poisson / ((1 + poisson) * (1 - 2 * poisson)), young / (2 * (1 + poisson))


def from_lame(lam, mu):
    """(E, nu) with lame(E, nu) = (lambda, mu)."""
    lam = np.asarray(lam, np.float64)
    mu = np.asarray(mu, np.float64)
    return mu * (3 * lam + 2 * mu) / (lam + mu), lam / (2 * (lam + mu))


class LargeStrainSolver:
    def __init__(self, problem, increments: int = 10, newton_tol: float = 1e-8, newton_max: int = 25,
                 tol: float = 1e-12, max_iter: int = 10000, precision: int = MAILLE_FP64, device: int = 0):
        if problem.conn.shape[1] != 4:
            raise MailleError("InvalidInput", "the large-strain path takes Tet4 meshes")
        self._L = _lib.load()
        self.increments = increments
        self.n3 = 3 * problem.coords.shape[0]
        self.n_elems = problem.conn.shape[0]
        self._keep = dict(
            coords=np.ascontiguousarray(problem.coords, np.float64),
            conn=np.ascontiguousarray(problem.conn, np.int64),
            young=np.ascontiguousarray(np.broadcast_to(problem.young, (self.n_elems,)), np.float64),
            poisson=np.ascontiguousarray(np.broadcast_to(problem.poisson, (self.n_elems,)), np.float64),
            fixed=np.ascontiguousarray(problem.fixed, np.uint8),
            imposed=np.ascontiguousarray(problem.imposed, np.float64),
            f=np.ascontiguousarray(problem.loads, np.float64))
        k = self._keep
        self._p = _lib.LargeStrainProblem(
            n_nodes=k["coords"].shape[0], coords=ptr(k["coords"], _d), n_elems=self.n_elems,
            conn=ptr(k["conn"], _i64), young=ptr(k["young"], _d), poisson=ptr(k["poisson"], _d),
            fixed=ptr(k["fixed"], _u8), imposed=ptr(k["imposed"], _d),
            f=ptr(k["f"], _d) if np.any(k["f"]) else None, increments=increments,
            newton_tol=newton_tol, newton_max_iter=newton_max, rel_tol=tol, max_iter=max_iter,
            precision=precision, device=device)
        self._h = ctypes.c_void_p()
        _raise_for(self._L.maille_gpu_large_strain_create(ctypes.byref(self._p), ctypes.byref(self._h)))

    def run(self) -> LargeStrainHistory:
        u = np.zeros((self.increments, self.n3))
        r = np.zeros((self.increments, self.n3))
        it = np.zeros(self.increments, np.int32)
        cuts = np.zeros(self.increments, np.int32)
        res = _lib.LargeStrainResult(u=ptr(u, _d), reactions=ptr(r, _d), newton_iterations=ptr(it, _i32),
                                     cuts=ptr(cuts, _i32))
        status = self._L.maille_gpu_large_strain_run(self._h, ctypes.byref(res))
        history = LargeStrainHistory(u, r, it, cuts, res.newton_total, res.pcg_total, res.ms_total)
        try:
            _raise_for(status)
        except MailleError as e:
            e.history = history  # the counts up to the failing increment, its cuts included
            raise
        return history

    def cancel(self, flag: bool = True):
        """Raises (or clears) the cancel flag: the run stops before its next Newton iteration or
        inner PCG launch with MailleError("Cancelled")."""
        self._L.maille_gpu_large_strain_cancel(self._h, 1 if flag else 0)

    def backward(self, dJdR):
        g = np.ascontiguousarray(dJdR, np.float64).reshape(self.increments, self.n3)
        gm = np.zeros(self.n_elems)
        gl = np.zeros(self.n_elems)
        _raise_for(self._L.maille_gpu_large_strain_backward(self._h, ptr(g, _d), ptr(gm, _d), ptr(gl, _d)))
        return gm, gl

    def set_materials(self, young=None, poisson=None):
        ya = None if young is None else np.ascontiguousarray(young, np.float64)
        pa = None if poisson is None else np.ascontiguousarray(poisson, np.float64)
        _raise_for(self._L.maille_gpu_large_strain_set_materials(self._h, ptr(ya, _d), ptr(pa, _d)))

    def close(self):
        if self._h:
            self._L.maille_gpu_large_strain_destroy(self._h)
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
