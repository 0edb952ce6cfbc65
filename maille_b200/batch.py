"""Batched solves: many independent Tet4/Tet10 models, several load cases each, in one GPU call
(maille_gpu_batch_* of include/maille_gpu.h).

The reference solves one Model (one mesh, one load vector) per Model::solve call
(crates/maille-core/src/model.rs:548-610); a host program with many models loops over them. Here
the loop moves into one persistent GPU kernel: `BatchSolver(problems, loads)` packs the models,
`solve()` returns every instance's displacements for every load case, each converged to its own
IC(0)-PCG stopping test ||r|| <= tol ||b|| (iterative.rs:233).

Across GPUs the batch shards by instance (`partition_lpt`, `solve_sharded`): each rank solves its
own instances, with no collective on the data path.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import MAILLE_BATCH_MAX_RHS, MAILLE_FP64, ptr, _d, _i32, _i64, _u8
from .model import MailleError, _raise_for


@dataclass
class BatchField:
    """Results of a batched solve: per instance a (3 N_k, n_rhs) displacement array."""
    displacements: List[np.ndarray]
    iterations: np.ndarray      # (n_instances, n_rhs)
    rel_residual: np.ndarray    # (n_instances, n_rhs)
    status: np.ndarray          # (n_instances,) MailleStatus per instance
    info: dict = field(default_factory=dict)


def pack(problems: Sequence, loads: Optional[Sequence[np.ndarray]]):
    """Packed arrays of the C ABI: node and element offsets, coordinates, local connectivity,
    materials, constraints and the (n_rhs, 3 N_total) load cases. `loads[k]` is (3 N_k, n_rhs)."""
    if len(problems) == 0:
        raise MailleError("InvalidInput", "empty batch")
    npe = problems[0].conn.shape[1]
    if any(p.conn.shape[1] != npe for p in problems):
        raise MailleError("InvalidInput", "every instance must use the same element family")
    nodes = np.array([p.coords.shape[0] for p in problems], np.int64)
    elems = np.array([p.conn.shape[0] for p in problems], np.int64)
    node_off = np.concatenate([[0], np.cumsum(nodes)]).astype(np.int64)
    elem_off = np.concatenate([[0], np.cumsum(elems)]).astype(np.int64)
    out = dict(
        npe=npe, node_offset=node_off, elem_offset=elem_off,
        coords=np.ascontiguousarray(np.concatenate([p.coords for p in problems]), np.float64),
        conn=np.ascontiguousarray(np.concatenate([p.conn for p in problems]), np.int64),
        young=np.ascontiguousarray(np.concatenate([np.broadcast_to(p.young, (p.conn.shape[0],))
                                                   for p in problems]), np.float64),
        poisson=np.ascontiguousarray(np.concatenate([np.broadcast_to(p.poisson, (p.conn.shape[0],))
                                                     for p in problems]), np.float64),
        fixed=np.ascontiguousarray(np.concatenate([p.fixed for p in problems]), np.uint8),
        imposed=np.ascontiguousarray(np.concatenate([p.imposed for p in problems]), np.float64),
    )
    out["n_rhs"] = 0
    out["f"] = None
    if loads is not None:
        out["f"] = pack_loads(loads, node_off)
        out["n_rhs"] = out["f"].shape[0]
    return out


def pack_loads(loads: Sequence[np.ndarray], node_off: np.ndarray) -> np.ndarray:
    """(n_rhs, 3 N_total) from per-instance (3 N_k, n_rhs) load arrays."""
    n_rhs = {np.asarray(l).reshape(np.asarray(l).shape[0], -1).shape[1] for l in loads}
    if len(n_rhs) != 1:
        raise MailleError("InvalidInput", "every instance needs the same number of load cases")
    n_rhs = n_rhs.pop()
    if not 1 <= n_rhs <= MAILLE_BATCH_MAX_RHS:
        raise MailleError("InvalidInput", f"1..{MAILLE_BATCH_MAX_RHS} load cases per instance")
    f = np.zeros((n_rhs, 3 * int(node_off[-1])))
    for k, l in enumerate(loads):
        a = np.asarray(l, np.float64).reshape(-1, n_rhs)
        if a.shape[0] != 3 * (node_off[k + 1] - node_off[k]):
            raise MailleError("InvalidInput", f"instance {k}: loads have {a.shape[0]} rows")
        f[:, 3 * node_off[k]:3 * node_off[k + 1]] = a.T
    return f


class BatchSolver:
    """GPU handle over a packed batch (create / solve / refactor / cancel / destroy)."""

    def __init__(self, problems: Sequence, loads: Sequence[np.ndarray], tol: float = 1e-12,
                 max_iter: int = 10000, precision: int = MAILLE_FP64, device: int = 0):
        self._L = _lib.load()
        self._pk = pack(problems, loads)
        pk = self._pk
        self.n_instances = len(problems)
        self.n_rhs = pk["n_rhs"]
        self.node_offset = pk["node_offset"]
        self._p = _lib.BatchProblem(
            n_instances=self.n_instances, nodes_per_elem=pk["npe"], n_rhs=self.n_rhs,
            node_offset=ptr(pk["node_offset"], _i64), elem_offset=ptr(pk["elem_offset"], _i64),
            coords=ptr(pk["coords"], _d), conn=ptr(pk["conn"], _i64), young=ptr(pk["young"], _d),
            poisson=ptr(pk["poisson"], _d), fixed=ptr(pk["fixed"], _u8),
            imposed=ptr(pk["imposed"], _d), f=ptr(pk["f"], _d), rel_tol=tol, max_iter=max_iter,
            precision=precision, device=device)
        self._h = ctypes.c_void_p()
        s = self._L.maille_gpu_batch_create(ctypes.byref(self._p), ctypes.byref(self._h))
        _raise_for(s)

    def solve(self, loads: Optional[Sequence[np.ndarray]] = None) -> BatchField:
        f = None if loads is None else np.ascontiguousarray(pack_loads(loads, self.node_offset))
        n3 = 3 * int(self.node_offset[-1])
        u = np.zeros((self.n_rhs, n3))
        it = np.zeros((self.n_instances, self.n_rhs), np.int32)
        rr = np.zeros((self.n_instances, self.n_rhs))
        st = np.zeros(self.n_instances, np.int32)
        res = _lib.BatchResult(u=ptr(u, _d), iterations=ptr(it, _i32), rel_residual=ptr(rr, _d),
                               status=ptr(st, _i32))
        s = self._L.maille_gpu_batch_solve(self._h, ptr(f, _d), ctypes.byref(res))
        info = {k: getattr(res, k) for k, _ in _lib.BatchResult._fields_
                if k not in ("u", "iterations", "rel_residual", "status")}
        if s not in (_lib.MAILLE_OK, _lib.MAILLE_SINGULAR, _lib.MAILLE_NOT_CONVERGED):
            _raise_for(s)
        off = self.node_offset
        disp = [u[:, 3 * off[k]:3 * off[k + 1]].T.copy() for k in range(self.n_instances)]
        return BatchField(disp, it, rr, st, dict(info, status_code=s))

    def refactor(self, young=None, poisson=None):
        ya = None if young is None else np.ascontiguousarray(young, np.float64).ravel()
        pa = None if poisson is None else np.ascontiguousarray(poisson, np.float64).ravel()
        s = self._L.maille_gpu_batch_refactor(self._h, ptr(ya, _d), ptr(pa, _d))
        _raise_for(s)

    def cancel(self, flag: bool = True):
        self._L.maille_gpu_batch_cancel(self._h, 1 if flag else 0)

    @property
    def stream(self) -> int:
        return int(self._L.maille_gpu_batch_stream(self._h) or 0)

    def close(self):
        if self._h:
            self._L.maille_gpu_batch_destroy(self._h)
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


def partition_lpt(costs: Sequence[float], parts: int) -> List[List[int]]:
    """Longest-processing-time partition: instances by decreasing cost, each to the currently
    lightest part (ties to the lowest part index); instances keep ascending order in a part."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    load = [0.0] * parts
    out: List[List[int]] = [[] for _ in range(parts)]
    for k in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        j = min(range(parts), key=lambda q: (load[q], q))
        out[j].append(k)
        load[j] += float(costs[k])
    return [sorted(o) for o in out]


def instance_cost(problem) -> float:
    """Work estimate of one instance: node-pair blocks of its stiffness pattern (about the
    matrix bytes an iteration streams) times the square root of its node count (PCG iterations
    grow with the mesh diameter)."""
    n = problem.coords.shape[0]
    npe = problem.conn.shape[1]
    blocks = n + problem.conn.shape[0] * npe * (npe - 1) / 2.0
    return float(blocks * np.sqrt(n))


def solve_sharded(problems: Sequence, loads: Sequence[np.ndarray], rank: int, world: int,
                  device: int = 0, **kw):
    """This rank's share of a batch (LPT by instance cost): returns (instance ids, BatchField)."""
    shares = partition_lpt([instance_cost(p) for p in problems], world)
    mine = shares[rank]
    if not mine:
        return mine, None
    with BatchSolver([problems[k] for k in mine], [loads[k] for k in mine], device=device, **kw) as b:
        return mine, b.solve()


def gather_sharded(mine: List[int], part: Optional[BatchField], n_instances: int, n_rhs: int,
                   dst: int = 0, group=None) -> Optional[BatchField]:
    """Collects every rank's (instance ids, BatchField) of solve_sharded on rank `dst` through
    torch.distributed (any backend; one gather of host objects after the solves, not on the data
    path) and returns the whole batch's BatchField in instance order there, None on the other
    ranks. Every rank of the group must call it."""
    import torch.distributed as dist
    item = (list(mine), None if part is None else (part.displacements, part.iterations, part.rel_residual,
                                                  part.status))
    world = dist.get_world_size(group)
    out = [None] * world if dist.get_rank(group) == dst else None
    dist.gather_object(item, out, dst=dst, group=group)
    if out is None:
        return None
    disp: List[Optional[np.ndarray]] = [None] * n_instances
    it = np.zeros((n_instances, n_rhs), np.int32)
    rr = np.zeros((n_instances, n_rhs))
    st = np.zeros(n_instances, np.int32)
    seen = 0
    for ids, fields in out:
        if fields is None:
            continue
        d, i, r, s = fields
        for j, k in enumerate(ids):
            disp[k] = d[j]
            it[k], rr[k], st[k] = i[j], r[j], s[j]
            seen += 1
    if seen != n_instances:
        raise MailleError("InvalidInput", f"the ranks returned {seen} of {n_instances} instances")
    return BatchField(disp, it, rr, st, {"ranks": world})
