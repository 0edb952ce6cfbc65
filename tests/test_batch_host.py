"""CPU tests of the batched path's host logic: packing into the C ABI's arrays, input checks
before any device work, and the instance sharding across ranks (longest-processing-time
partition, checked for consistency over gloo with world size 2). No GPU compute runs here."""
import ctypes
import os

import numpy as np
import pytest

import maille_b200 as mb
from maille_b200 import _lib, batch, build, meshgen as mg


def small_batch(count=5, lo=2, hi=4, load_cases=3):
    return mg.batched_tet4(count=count, lo=lo, hi=hi, load_cases=load_cases)


def test_pack_offsets_and_local_connectivity():
    probs, loads = small_batch()
    pk = batch.pack(probs, loads)
    assert pk["node_offset"][0] == 0 and pk["node_offset"][-1] == sum(p.n_nodes for p in probs)
    assert pk["elem_offset"][-1] == sum(p.n_elems for p in probs)
    for k, p in enumerate(probs):
        e0, e1 = pk["elem_offset"][k], pk["elem_offset"][k + 1]
        assert np.array_equal(pk["conn"][e0:e1], p.conn)  # local ids
        n0, n1 = pk["node_offset"][k], pk["node_offset"][k + 1]
        assert np.array_equal(pk["coords"][n0:n1], p.coords)
        # load case j of instance k sits at f[j, 3 n0 : 3 n1]
        assert np.array_equal(pk["f"][:, 3 * n0:3 * n1], loads[k].T)
    assert pk["f"].shape == (3, 3 * pk["node_offset"][-1])


def test_traction_loads_resultant_is_traction_times_area():
    """The vector face traction of the batched workload has no reference counterpart; its
    resultant over the unit top face equals the traction itself."""
    probs, loads = small_batch(count=3, load_cases=4)
    for k, (p, f) in enumerate(zip(probs, loads)):
        res = f.reshape(p.n_nodes, 3, -1).sum(axis=0).T  # (L, 3)
        u = mg.uniform(stream=5000 + k, count=3 * 4).reshape(4, 3)
        cos_t = 2 * u[:, 0] - 1
        phi = 2 * np.pi * u[:, 1]
        sin_t = np.sqrt(1 - cos_t ** 2)
        t = np.stack([sin_t * np.cos(phi), sin_t * np.sin(phi), cos_t], 1) * (1 + 19 * u[:, 2])[:, None]
        assert np.allclose(res, t, rtol=1e-13, atol=1e-13)
        assert np.allclose(np.linalg.norm(t, axis=1), 1 + 19 * u[:, 2])


def test_pack_rejects_bad_batches():
    probs, loads = small_batch(count=2)
    with pytest.raises(mb.MailleError):
        batch.pack([], None)
    with pytest.raises(mb.MailleError):
        batch.pack(probs, [loads[0], loads[1][:, :2]])  # different load-case counts
    with pytest.raises(mb.MailleError):
        batch.pack(probs, [np.zeros((3 * probs[0].n_nodes, 9))] * 2)  # more than 8 load cases
    with pytest.raises(mb.MailleError):
        batch.pack(probs, [loads[0][:-3], loads[1]])  # wrong row count
    q = mg.mixed_tet10(1)
    with pytest.raises(mb.MailleError):
        batch.pack([probs[0], q], None)  # mixed element families


def test_batch_inputs_are_checked_before_any_device_work():
    build.build()
    lib = _lib.load()
    probs, loads = small_batch(count=2)
    pk = batch.pack(probs, loads)

    def status(**over):
        d = dict(pk)
        d.update(over)
        p = _lib.BatchProblem(
            n_instances=over.get("n_instances", 2), nodes_per_elem=over.get("npe", 4),
            n_rhs=over.get("n_rhs", 3), node_offset=_lib.ptr(d["node_offset"], _lib._i64),
            elem_offset=_lib.ptr(d["elem_offset"], _lib._i64), coords=_lib.ptr(d["coords"], _lib._d),
            conn=_lib.ptr(d["conn"], _lib._i64), young=_lib.ptr(d["young"], _lib._d),
            poisson=_lib.ptr(d["poisson"], _lib._d), fixed=_lib.ptr(d["fixed"], _lib._u8),
            imposed=_lib.ptr(d["imposed"], _lib._d), f=_lib.ptr(d["f"], _lib._d), rel_tol=1e-10,
            max_iter=100, precision=over.get("precision", 0), device=0)
        h = ctypes.c_void_p()
        s = lib.maille_gpu_batch_create(ctypes.byref(p), ctypes.byref(h))
        if h:
            lib.maille_gpu_batch_destroy(h)
        return s, _lib.last_error()

    bad_conn = pk["conn"].copy()
    bad_conn[0, 0] = probs[0].n_nodes  # a node id of the next instance, not local
    s, msg = status(conn=bad_conn)
    assert s == _lib.MAILLE_INVALID_INPUT and "unknown node" in msg
    s, msg = status(n_rhs=9)
    assert s == _lib.MAILLE_INVALID_INPUT and "n_rhs" in msg
    s, _ = status(npe=6)
    assert s == _lib.MAILLE_INVALID_INPUT
    s, _ = status(precision=7)
    assert s == _lib.MAILLE_INVALID_INPUT
    y = pk["young"].copy()
    y[3] = -1.0
    s, msg = status(young=y)
    assert s == _lib.MAILLE_INVALID_INPUT and "material" in msg
    f = pk["f"].copy()
    f[1, 4] = np.inf
    s, msg = status(f=f)
    assert s == _lib.MAILLE_INVALID_INPUT and "load" in msg
    off = pk["node_offset"].copy()
    off[1] = off[0]  # an empty instance
    s, msg = status(node_offset=off)
    assert s == _lib.MAILLE_INVALID_INPUT
    fx = pk["fixed"].copy()
    fx[:3 * probs[0].n_nodes] = 1  # every DOF of instance 0 fixed
    s, msg = status(fixed=fx)
    assert s == _lib.MAILLE_INVALID_INPUT and "instance 0" in msg


def test_partition_lpt_covers_every_instance_once_and_balances():
    rng = np.random.default_rng(0)
    costs = rng.uniform(1, 100, 257)
    for parts in (1, 2, 3, 8):
        shares = batch.partition_lpt(costs, parts)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(257))
        loads = [costs[s].sum() for s in shares]
        # LPT bound: max load <= mean load + largest item
        assert max(loads) <= costs.sum() / parts + costs.max() + 1e-9
        assert batch.partition_lpt(costs, parts) == shares  # deterministic
    assert batch.partition_lpt([5.0], 3) == [[0], [], []]


def _shard_worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    probs, _ = mg.batched_tet4(count=40, lo=2, hi=9, load_cases=2)
    costs = [batch.instance_cost(p) for p in probs]
    mine = batch.partition_lpt(costs, world)[rank]
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as fh:
        fh.write(repr(gathered))
    dist.destroy_process_group()


def test_sharding_is_consistent_across_ranks(tmp_path):
    """Two gloo ranks compute their shares independently; every rank sees the same partition,
    the shares are disjoint and cover the batch (no data-path collective is needed)."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.spawn(_shard_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    views = [eval(open(tmp_path / f"r{r}.txt").read()) for r in range(2)]
    assert views[0] == views[1]
    a, b = views[0]
    assert not set(a) & set(b) and sorted(a + b) == list(range(40))


def _gather_worker(rank, world, port, out_dir):
    """Fake per-rank results (no device): instance k's displacement is filled with k, so the
    gathered batch shows where every instance landed."""
    import pickle
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    costs = [float(c) for c in np.arange(1, 12)]
    mine = batch.partition_lpt(costs, world)[rank]
    part = batch.BatchField([np.full((3 * (k + 1), 2), float(k)) for k in mine],
                            np.array([[k, k + 1] for k in mine], np.int32).reshape(-1, 2),
                            np.array([[k * 1e-13, 0.0] for k in mine]).reshape(-1, 2),
                            np.zeros(len(mine), np.int32))
    whole = batch.gather_sharded(mine, part, len(costs), 2)
    with open(os.path.join(out_dir, f"g{rank}.pkl"), "wb") as fh:
        pickle.dump(whole, fh)
    dist.destroy_process_group()


def test_sharded_results_gather_on_rank_zero(tmp_path):
    """The gather after a sharded solve puts every instance back in batch order on rank 0 and
    returns None on the other ranks (world size 2, gloo)."""
    import pickle
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.spawn(_gather_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    whole = pickle.load(open(tmp_path / "g0.pkl", "rb"))
    assert pickle.load(open(tmp_path / "g1.pkl", "rb")) is None
    assert len(whole.displacements) == 11
    for k in range(11):
        assert whole.displacements[k].shape == (3 * (k + 1), 2) and (whole.displacements[k] == k).all()
        assert list(whole.iterations[k]) == [k, k + 1]
    assert whole.info["ranks"] == 2
