"""GPU tests of the batched solve (maille_gpu_batch_*): every instance and load case against the
oracle's IC(0)-PCG (FP64 within 1e-10 relative L2 once both are converged to 1e-13, mixed within
1e-8), every compiled lane layout, per-instance convergence masks and statuses, determinism,
cancellation, the autotune cache, and the full 256-instance workload."""
import copy
import os

import numpy as np
import pytest

import maille_b200 as mb
from maille_b200 import batch, meshgen as mg
from maille_b200._lib import MAILLE_FP64, MAILLE_MIXED

pytestmark = pytest.mark.gpu

# (R, Q, SUB) lane layouts compiled into the library, by padded load-case count
LAYOUTS = {8: [(8, 1), (8, 2), (4, 1), (4, 2), (2, 1)], 4: [(4, 1), (4, 2), (2, 1)],
           2: [(2, 1), (2, 2), (1, 1)]}


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def oracle_columns(oracle_lib, prob, loads, tol=1e-13):
    out = []
    for j in range(loads.shape[1]):
        q = copy.copy(prob)
        q.loads = np.ascontiguousarray(loads[:, j])
        r = oracle_lib.model_solve(q, solver=2, tol=tol)
        assert r["status"] == 0
        out.append(r["u"])
    return np.stack(out, 1)


def check_against_oracle(oracle_lib, probs, loads, field, tol):
    for k, (p, l) in enumerate(zip(probs, loads)):
        ref = oracle_columns(oracle_lib, p, l)
        for j in range(l.shape[1]):
            assert rel(field.displacements[k][:, j], ref[:, j]) < tol, (k, j)


@pytest.fixture
def env_layout():
    keys = ("MAILLE_BATCH_Q", "MAILLE_BATCH_SUB", "MAILLE_BATCH_THREADS", "MAILLE_BATCH_TASK")
    saved = {k: os.environ.get(k) for k in keys}

    def set_layout(q, sub, threads=256, task=4):
        os.environ.update(MAILLE_BATCH_Q=str(q), MAILLE_BATCH_SUB=str(sub),
                          MAILLE_BATCH_THREADS=str(threads), MAILLE_BATCH_TASK=str(task))
    yield set_layout
    for k, v in saved.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v


@pytest.mark.parametrize("n_rhs", [8, 3, 2])
def test_every_layout_matches_the_oracle(gpu, oracle_lib, env_layout, n_rhs):
    probs, loads = mg.batched_tet4(count=5, lo=2, hi=5, load_cases=n_rhs)
    R = 2 if n_rhs <= 2 else (4 if n_rhs <= 4 else 8)
    refs = [oracle_columns(oracle_lib, p, l) for p, l in zip(probs, loads)]
    for q, sub in LAYOUTS[R]:
        for threads, task in ((256, 1), (128, 16)):
            env_layout(q, sub, threads, task)
            with mb.BatchSolver(probs, loads, tol=1e-13) as b:
                f = b.solve()
            assert f.info["status_code"] == 0 and not f.status.any()
            assert f.info["rhs_per_lane"] == q and f.info["threads"] == threads
            for k in range(len(probs)):
                for j in range(n_rhs):
                    assert rel(f.displacements[k][:, j], refs[k][:, j]) < 1e-10, (q, sub, k, j)
                    assert f.rel_residual[k, j] <= 1e-13


def test_tet10_batch_with_imposed_displacements(gpu, oracle_lib):
    probs = []
    for c in (1, 2, 3):
        p = mg.mixed_tet10(c)
        # pull the top face up by 1e-3 in z on one instance: a non-zero K_fc u_c coupling
        top = np.nonzero(np.abs(p.coords[:, 2] - 1.0) < 1e-12)[0]
        if c == 2:
            p.fixed[3 * top + 2] = 1
            p.imposed[3 * top + 2] = 1e-3
            p.p_elem, p.p_face, p.p_value = p.p_elem[:0], p.p_face[:0], p.p_value[:0]
        probs.append(p)
    loads = []
    for p in probs:
        f0 = mb.face_pressure_loads(p.coords, p.conn, list(zip(p.p_elem, p.p_face, p.p_value)))
        l = np.stack([f0, 0.5 * f0 + 0.1, np.zeros_like(f0)], 1)
        l[np.nonzero(p.fixed)[0]] = 0.0
        loads.append(l)
    with mb.BatchSolver(probs, loads, tol=1e-13) as b:
        f = b.solve()
    assert f.info["status_code"] == 0
    for k, (p, l) in enumerate(zip(probs, loads)):
        q = copy.copy(p)
        q.p_elem, q.p_face, q.p_value = p.p_elem[:0], p.p_face[:0], p.p_value[:0]
        ref = oracle_columns(oracle_lib, q, l)
        for j in range(3):
            assert rel(f.displacements[k][:, j], ref[:, j]) < 1e-10, (k, j)
        fixed = np.nonzero(p.fixed)[0]
        assert np.array_equal(f.displacements[k][fixed, 2], p.imposed[fixed])
    # the zero load case of instances without imposed values is exactly zero, in 0 iterations
    assert not f.displacements[0][:, 2].any() and f.iterations[0, 2] == 0


def test_mixed_precision_batch_reaches_1e8(gpu, oracle_lib):
    probs, loads = mg.batched_tet4(count=6, lo=3, hi=8, load_cases=8)
    with mb.BatchSolver(probs, loads, tol=1e-10, precision=MAILLE_MIXED) as b:
        f = b.solve()
    assert f.info["status_code"] == 0
    check_against_oracle(oracle_lib, probs, loads, f, 1e-8)
    assert (f.rel_residual <= 1e-10).all()


def test_instances_stop_on_their_own(gpu):
    """Small instances converge long before large ones; each reports its own iterations, and the
    per-instance iteration cap turns into that instance's status only."""
    probs, loads = mg.batched_tet4(count=4, lo=2, hi=12, load_cases=4)
    with mb.BatchSolver(probs, loads, tol=1e-12) as b:
        f = b.solve()
    sides = [round(p.n_elems / 6) ** (1 / 3) for p in probs]
    it = f.iterations.max(axis=1)
    assert len(set(it)) > 1
    assert it[int(np.argmin(sides))] < it[int(np.argmax(sides))]
    cap = int(it.min()) + 1
    with mb.BatchSolver(probs, loads, tol=1e-12, max_iter=cap) as b:
        g = b.solve()
    assert g.info["status_code"] == 2
    for k in range(4):
        if it[k] <= cap:
            assert g.status[k] == 0
            assert np.array_equal(g.displacements[k], f.displacements[k])
        else:
            assert g.status[k] == 2


def test_repeated_batched_solves_are_bit_identical(gpu):
    probs, loads = mg.batched_tet4(count=6, lo=3, hi=9, load_cases=8)
    with mb.BatchSolver(probs, loads, tol=1e-11) as b:
        a = b.solve()
        c = b.solve()
        d = b.solve(loads)  # explicit loads equal to the problem's
    for k in range(6):
        assert np.array_equal(a.displacements[k], c.displacements[k])
        assert np.array_equal(a.displacements[k], d.displacements[k])
    assert np.array_equal(a.iterations, c.iterations)


def test_refactor_and_new_loads(gpu, oracle_lib):
    probs, loads = mg.batched_tet4(count=3, lo=2, hi=4, load_cases=2)
    with mb.BatchSolver(probs, loads, tol=1e-13) as b:
        b.solve()
        young = [2.0 * np.asarray(p.young) for p in probs]
        b.refactor(young=np.concatenate(young))
        new = [2.0 * l[:, ::-1].copy() for l in loads]
        f = b.solve(new)
    for k, p in enumerate(probs):
        q = copy.copy(p)
        q.young = young[k]
        ref = oracle_columns(oracle_lib, q, new[k])
        for j in range(2):
            assert rel(f.displacements[k][:, j], ref[:, j]) < 1e-10


def test_cancel_flag_stops_the_batch(gpu):
    probs, loads = mg.batched_tet4(count=3, lo=4, hi=6, load_cases=2)
    with mb.BatchSolver(probs, loads) as b:
        b.cancel(True)
        with pytest.raises(mb.MailleError) as e:
            b.solve()
        assert e.value.kind == "Cancelled"
        b.cancel(False)
        assert b.solve().info["status_code"] == 0


def test_autotuner_runs_once_per_shape(gpu):
    for k in ("MAILLE_BATCH_Q",):
        os.environ.pop(k, None)
    probs, loads = mg.batched_tet4(count=7, lo=3, hi=6, load_cases=8)
    with mb.BatchSolver(probs, loads, tol=1e-10) as b:
        first = b.solve()
    with mb.BatchSolver(probs, loads, tol=1e-10) as b:
        second = b.solve()
    assert first.info["autotuned"] == 1 and second.info["autotuned"] == 0
    for key in ("rhs_per_lane", "lanes_per_row", "threads", "task_slices"):
        assert first.info[key] == second.info[key]
    for k in range(7):
        assert np.array_equal(first.displacements[k], second.displacements[k])


def test_full_batched_workload(gpu, oracle_lib):
    """256 Tet4 cubes of side 6..24 with 8 traction load cases each: every instance converges,
    the reported residuals meet the tolerance, instances up to side 8 match the oracle, and the
    largest instances match single-instance GPU solves (FP64 and mixed)."""
    probs, loads = mg.batched_tet4()
    sides = np.array([round((p.n_elems / 6) ** (1 / 3)) for p in probs])
    assert sides.min() == 6 and sides.max() == 24
    with mb.BatchSolver(probs, loads, tol=1e-10) as b:
        f = b.solve()
    assert f.info["status_code"] == 0 and not f.status.any()
    assert (f.rel_residual <= 1e-10).all()
    small = [k for k in range(256) if sides[k] <= 7][:6]
    for k in small:
        ref = oracle_columns(oracle_lib, probs[k], loads[k], tol=1e-12)
        for j in range(8):
            assert rel(f.displacements[k][:, j], ref[:, j]) < 1e-8
    big = [int(k) for k in np.argsort(-sides)[:2]]
    for k in big:
        p = probs[k]
        for j in (0, 7):
            m = mb.Model.from_arrays(p.coords, p.conn, p.young, p.poisson, p.fixed, p.imposed,
                                     loads[k][:, j])
            m.with_solver(mb.SolverKind.ITERATIVE).with_tolerance(1e-12)
            u = m.solve().displacements
            assert rel(f.displacements[k][:, j], u) < 1e-8
    with mb.BatchSolver(probs, loads, tol=1e-10, precision=MAILLE_MIXED) as b:
        g = b.solve()
    assert g.info["status_code"] == 0
    for k in small + big:
        for j in range(8):
            assert rel(g.displacements[k][:, j], f.displacements[k][:, j]) < 1e-8


def _sharded_worker(rank, world, port, out_dir):
    """One rank of a sharded batch on device 0: its LPT share solved by its own BatchSolver (no
    collective while solving), then the results gathered on rank 0 over gloo."""
    import pickle
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    probs, loads = mg.batched_tet4(count=16, lo=3, hi=8, load_cases=4)
    mine, part = batch.solve_sharded(probs, loads, rank, world, device=0, tol=1e-13)
    whole = batch.gather_sharded(mine, part, len(probs), 4)
    with open(os.path.join(out_dir, f"s{rank}.pkl"), "wb") as fh:
        pickle.dump((mine, whole), fh)
    dist.destroy_process_group()


def test_sharded_batch_gathers_to_the_unsharded_result(gpu, tmp_path):
    """Two ranks (two processes sharing device 0; their kernels never wait on one another) solve
    disjoint LPT shares of a 16-instance batch; the gathered result equals the unsharded
    BatchSolver's instance by instance."""
    import pickle
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.spawn(_sharded_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    (mine0, whole), (mine1, none) = [pickle.load(open(tmp_path / f"s{r}.pkl", "rb")) for r in range(2)]
    assert none is None and mine0 and mine1 and not set(mine0) & set(mine1)
    probs, loads = mg.batched_tet4(count=16, lo=3, hi=8, load_cases=4)
    with batch.BatchSolver(probs, loads, tol=1e-13) as b:
        ref = b.solve()
    assert (whole.status == 0).all()
    for k in range(16):
        assert rel(whole.displacements[k], ref.displacements[k]) < 1e-10, k
        assert whole.rel_residual[k].max() <= 1e-13
