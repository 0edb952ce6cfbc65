#!/usr/bin/env python
"""Benchmark of the B200 linear-elastic solve path (one JSON line on rank 0).

Workload (the mixed-precision configuration): Tet10 unit cube, 40^3 cells x 6 quadratic tets
(531 441 nodes, 384 000 tets, 1 574 640 free DOF), 4-point Gauss rule, per-element E lognormal
(median 210 000 MPa, sigma_log 0.5, seeded), nu = 0.3, z = 0 clamped, 10 MPa pressure on z = 1.
Synthetic data generated in code (maille_b200/meshgen.py).

A step is one full numeric solve on device-resident inputs: element integration, scatter-reduce
assembly, IC(0) factorisation, FP32 inner PCG inside FP64 refinement to the relative residual
`--tol`, reactions, Gauss stresses and von Mises. `value` = free DOF solved per second (all ranks),
checked to reach 1e-8 relative displacement error against a tight FP64 solve. Beside it: the
plain FP64 GPU form on the same workload and tolerance, the live SpMV roofline, the end-to-end
rate through the C ABI with host buffers (`e2e`), and the CPU oracle baseline.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--cells C]
Under torchrun each rank solves its own replica (replicas only: the IC(0) solve does not shard).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DOF/s to 1e-8 rel. error: mixed/batched vs plain FP64 GPU; SpMV HBM GB/s"
UNIT = "DOF/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cells", type=int, default=40)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle baseline")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint cost section")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched section")
    ap.add_argument("--no-large-strain", action="store_true", help="skip the large-strain section")
    ap.add_argument("--no-thermal", action="store_true", help="skip the transient thermal section")
    ap.add_argument("--batch-count", type=int, default=256)
    ap.add_argument("--adjoint-cells", type=int, default=48)
    ap.add_argument("--only", choices=["mixed", "plain", "thermal", "thermal_mixed", "batched", "large_strain"],
                    default=None,
                    help="profiling mode: time one form only (no reference solve, e2e or CPU); "
                         "prints a short line, not the benchmark line")
    ap.add_argument("--thermal-cells", type=int, default=40, help="cube side of the thermal section")
    ap.add_argument("--ordering", choices=sorted(ORDERINGS), default="auto",
                    help="ordering of the elastic solves (MailleOrdering)")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def peaks():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling (200 ms) during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,"
              "utilization.gpu")

    def __init__(self, local_rank):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [v for v in vis.split(",") if v.strip()]
        self.index = ids[local_rank] if local_rank < len(ids) and ids[local_rank].isdigit() else str(local_rank)
        self.proc = None

    def start(self):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.index, f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        rows = [l.split(",") for l in open(self.f.name).read().strip().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 10:
                continue
            try:
                util = float(r[9])
                mx = float(r[2])
                if util > 0:
                    sm.append(float(r[1]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(rows), "samples_under_load": len(sm)}


ORDERINGS = {"auto": 0, "multicolor": 1, "rcm": 2, "multicolor_bfs": 3, "multicolor_iterated": 4}
ORDERING = 0  # --ordering of the elastic solves (MailleOrdering)


def solve_model(mb, p, precision, tol, device):
    m = mb.Model.from_arrays(p.coords, p.conn, p.young, p.poisson, p.fixed, p.imposed, p.loads,
                             (p.p_elem, p.p_face, p.p_value))
    m.with_solver(mb.SolverKind.ITERATIVE).with_tolerance(tol).with_precision(precision)
    m.ordering = ORDERING
    return m


def time_handle(torch, h, steps, warmup, L):
    """W untimed and K timed steps of refactor + solve on device-resident inputs; CUDA events on
    the library's stream. Returns (ms per step, last info, kernel launches per step)."""
    stream = torch.cuda.ExternalStream(h.stream)
    for _ in range(warmup):
        L.maille_gpu_refactor(h._h, None, None)
        h.solve()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k0 = L.maille_gpu_kernel_launches()
    start.record(stream)
    info = None
    for _ in range(steps):
        s = L.maille_gpu_refactor(h._h, None, None)
        if s != 0:
            raise RuntimeError("refactor failed: " + L.maille_gpu_last_error().decode())
        r = h._L  # solve without downloading the results (device-resident)
        from maille_b200._lib import ElasticResult
        res = ElasticResult()
        s = r.maille_gpu_solve(h._h, None, ctypes.byref(res))
        if s != 0:
            raise RuntimeError("solve failed: " + L.maille_gpu_last_error().decode())
        info = {k: getattr(res, k) for k, _ in ElasticResult._fields_
                if k not in ("u", "reactions", "gauss_stress", "von_mises")}
    end.record(stream)
    end.synchronize()
    launches = (L.maille_gpu_kernel_launches() - k0) / steps
    return start.elapsed_time(end) / steps, info, launches


def plain_tet4_section(torch, mb, mg, L, steps, warmup, device, cells=20, tol=1e-10):
    """The plain FP64 Tet4 configuration (unit cube 20^3 x 6 tets, 9 261 nodes, 26 460 free DOF,
    E = 210 000, nu = 0.3, z = 0 clamped, 10 MPa on z = 1, IC(0)-PCG to 1e-10), the reference path
    as it is: device-resident refactor + solve per step (CUDA events), and end to end through the
    C ABI from host buffers (create + solve + results + destroy, wall clock). The matrix is about
    10 MB and stays in L2: a latency-bound size, reported without a roofline."""
    from maille_b200._lib import MAILLE_FP64, ElasticResult, ptr, _d
    from maille_b200.model import problem_struct, face_pressure_loads
    p = mg.plain_tet4(cells)
    p.loads = face_pressure_loads(p.coords, p.conn, list(zip(p.p_elem, p.p_face, p.p_value)))
    p.p_elem, p.p_face, p.p_value = p.p_elem[:0], p.p_face[:0], p.p_value[:0]
    h = mb.SolverHandle(solve_model(mb, p, MAILLE_FP64, tol, device), device=device)
    try:
        ms, info, launches = time_handle(torch, h, max(steps, 5), warmup, L)
    finally:
        h.close()
    prob, keep = problem_struct(p.coords, p.conn.astype(np.int64), p.young, p.poisson, p.fixed, p.imposed,
                                p.loads, tol, 10000, MAILLE_FP64, 0, device)
    outs = dict(u=np.zeros(3 * p.n_nodes), r=np.zeros(3 * p.n_nodes), g=np.zeros(p.n_elems * 9),
                vm=np.zeros(p.n_elems))
    res = ElasticResult(u=ptr(outs["u"], _d), reactions=ptr(outs["r"], _d), gauss_stress=ptr(outs["g"], _d),
                        von_mises=ptr(outs["vm"], _d))
    assert L.maille_gpu_elastic_solve(ctypes.byref(prob), ctypes.byref(res)) == 0
    walls = []
    for _ in range(max(steps, 5)):
        t0 = time.perf_counter()
        if L.maille_gpu_elastic_solve(ctypes.byref(prob), ctypes.byref(res)) != 0:
            raise RuntimeError(L.maille_gpu_last_error().decode())
        walls.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = statistics.median(walls)
    return {"workload": f"tet4_{cells}^3_plain_fp64", "free_dofs": p.free_dofs, "tol": tol,
            "ms_per_step": ms, "value": p.free_dofs / (ms / 1e3), "unit": UNIT,
            "iterations": info["iterations"], "levels": info["levels"], "launches_per_step": launches,
            "e2e_ms": e2e_ms, "e2e_value": p.free_dofs / (e2e_ms / 1e3),
            "note": "the CPU oracle's time for this workload is in the reference arm's line"}


def adjoint_section(torch, mb, mg, L, cells, tol, steps, warmup, device, hbm):
    """Adjoint compliance on the Tet4 SIMP cube (cells^3, E = 210000 rho^3): one forward step
    (element integration, assembly, IC(0), PCG, reactions and stresses, device-resident) against
    one backward() (adjoint PCG with the same factor + the element gradient kernel + the gradient
    download), both with CUDA events on the library's stream; the gradient is checked against the
    oracle's full-size values when the golden summary for this size exists."""
    from maille_b200._lib import MAILLE_FP64, ptr, _d
    p, rho = mg.simp_tet4(cells)
    h = mb.SolverHandle(solve_model(mb, p, MAILLE_FP64, tol, device), device=device)
    try:
        ms_fwd, info, _ = time_handle(torch, h, steps, warmup, L)
        fld = h.solve()
        g = np.ascontiguousarray(h._f)
        dJdE = np.zeros(p.n_elems)
        stream = torch.cuda.ExternalStream(h.stream)
        for _ in range(warmup):
            assert L.maille_gpu_backward(h._h, ptr(g, _d), ptr(dJdE, _d), None) == 0
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(steps):
            s = L.maille_gpu_backward(h._h, ptr(g, _d), ptr(dJdE, _d), None)
            if s != 0:
                raise RuntimeError("backward failed: " + L.maille_gpu_last_error().decode())
        end.record(stream)
        end.synchronize()
        ms_bwd = start.elapsed_time(end) / steps
    finally:
        h.close()
    grad = dJdE * 3 * 210000.0 * rho ** 2
    out = {"workload": f"simp_tet4_{cells}^3_compliance", "free_dofs": p.free_dofs,
           "elements": p.n_elems, "tol": tol, "forward_ms": ms_fwd, "backward_ms": ms_bwd,
           "backward_over_forward": ms_bwd / ms_fwd, "target": 1.5,
           "iterations": info["iterations"], "compliance": float(g @ fld.displacements)}
    it_bytes = pcg_bytes_per_iteration(info["blocks"], info["block_rows"], 8)
    ach = it_bytes * info["iterations"] / (info["ms_solve"] * 1e6)
    out["roofline"] = {"bound": "hbm", "kernel": "k_pcg<double> persistent FP64 PCG of the forward solve",
                       "bytes_per_iteration": it_bytes, "ms_per_iteration": info["ms_solve"] / info["iterations"],
                       "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                       "note": "the backward solve runs the same kernel on the same matrix and factor"}
    path = os.path.join(ROOT, "tests", "golden", f"simp{cells}_oracle_gradient.json")
    if os.path.exists(path):
        ref = json.load(open(path))
        el = np.array(ref["elements"])
        out["grad_rel_err_vs_oracle"] = float(np.linalg.norm(grad[el] - np.array(ref["grad"]))
                                              / np.linalg.norm(ref["grad"]))
    return out


def instance_blocks(p):
    """(kept nodes, 3x3 blocks of the full symmetric pattern incl. the diagonal) of one model: a
    node is kept when one of its DOFs is free; a block couples two kept nodes of one element."""
    n = p.coords.shape[0]
    kept = ~p.fixed.reshape(n, 3).all(axis=1)
    conn = np.asarray(p.conn, np.int64)
    a = np.repeat(conn, conn.shape[1], axis=1).ravel()
    b = np.tile(conn, (1, conn.shape[1])).ravel()
    m = kept[a] & kept[b]
    return int(kept.sum()), int(np.unique(a[m] * n + b[m]).size)


def batched_section(torch, mb, mg, L, count, tol, steps, warmup, device, hbm, rank=0, world=1):
    """Batched Tet4 workload (`count` cubes of side 6..24, 8 traction load cases each; this rank's
    LPT share under torchrun): one step = element integration + assembly + IC(0) of every
    instance and the PCG of every instance and load case (device-resident inputs, CUDA events on
    the batch stream), FP64 and mixed. Against it, the same work as per-instance launches: one
    single-model handle per instance, refactor (element integration, assembly, IC(0)) + one
    device-buffer solve per load case (maille_gpu_solve_device: loads already in device memory,
    displacements written to device memory, no reactions or stresses, as the batch computes
    none), CUDA events around the whole pass. The method is simultaneous independent CG per load
    case sharing the matrix and factor reads, not a block-Krylov method.

    Roofline of the batched PCG: algorithmic bytes = per instance, its iterations (the slowest of
    its load cases) times its matrix bytes per iteration (K once, the strict triangles once each,
    D twice) plus every load case's iterations times its vector passes, over the solve's device
    time (res.ms_solve)."""
    import ctypes as C
    from maille_b200 import batch as mbatch
    from maille_b200._lib import MAILLE_FP64, MAILLE_MIXED, BatchResult
    probs, loads = mg.batched_tet4(count=count)
    mine = mbatch.partition_lpt([mbatch.instance_cost(p) for p in probs], world)[rank]
    probs = [probs[k] for k in mine]
    loads = [loads[k] for k in mine]
    n_rhs = loads[0].shape[1]
    free = sum(p.free_dofs for p in probs)
    out = {"workload": f"batched_tet4_{count}x{n_rhs}rhs", "instances": len(probs), "load_cases": n_rhs,
           "free_dofs": free, "tol": tol}

    def time_batch(precision):
        b = mb.BatchSolver(probs, loads, tol=tol, precision=precision, device=device)
        try:
            first = b.solve()  # runs the autotuner (or hits the cache)
            stream = torch.cuda.ExternalStream(b.stream)
            res = BatchResult()
            for _ in range(warmup):
                L.maille_gpu_batch_refactor(b._h, None, None)
                L.maille_gpu_batch_solve(b._h, None, C.byref(res))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            k0 = L.maille_gpu_kernel_launches()
            e0.record(stream)
            for _ in range(steps):
                if L.maille_gpu_batch_refactor(b._h, None, None) != 0:
                    raise RuntimeError(L.maille_gpu_last_error().decode())
                s = L.maille_gpu_batch_solve(b._h, None, C.byref(res))
                if s != 0:
                    raise RuntimeError(L.maille_gpu_last_error().decode())
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / steps
            launches = (L.maille_gpu_kernel_launches() - k0) / steps
            return ms, first, res, launches
        finally:
            b.close()

    shapes = [instance_blocks(p) for p in probs]
    for name, prec in (("fp64", MAILLE_FP64), ("mixed", MAILLE_MIXED)):
        ms, first, res, launches = time_batch(prec)
        vb = 8 if prec == MAILLE_FP64 else 4
        alg = 0
        for (nb_k, blocks_k), its in zip(shapes, first.iterations):
            mat, vec = pcg_bytes_parts(blocks_k, nb_k, vb)
            alg += int(its.max()) * mat + int(its.sum()) * vec
        out[name] = {"ms_per_step": ms, "value": free * n_rhs / (ms / 1e3),
                     "unit": "DOF*load_cases/s", "max_iterations": res.max_iterations,
                     "mean_iterations": float(first.iterations.mean()),
                     "ms_solve": res.ms_solve, "autotuned_ms": first.info["ms_tune"],
                     "config": {"rhs_per_lane": res.rhs_per_lane, "lanes_per_row": res.lanes_per_row,
                                "threads": res.threads, "task_slices": res.task_slices},
                     "kernel_launches_per_step": launches,
                     "roofline": {"bound": "hbm", "kernel": f"batched persistent PCG ({name})",
                                  "algorithmic_bytes": alg, "ms_solve": res.ms_solve,
                                  "achieved": alg / (res.ms_solve * 1e6), "peak": hbm, "unit": "GB/s",
                                  "frac": alg / (res.ms_solve * 1e6) / hbm}}
        if name == "fp64":
            u_fp64 = first.displacements
        else:
            err = max(float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
                      for a, b in zip(first.displacements, u_fp64))
            out[name]["max_rel_diff_vs_fp64"] = err

    # per-instance launches of the single-model path: refactor + one device-buffer solve per
    # load case, loads resident on the device, no reactions or stresses
    handles = []
    dev = torch.device("cuda", device)
    try:
        for p in probs:
            m = mb.Model.from_arrays(p.coords, p.conn, p.young, p.poisson, p.fixed, p.imposed, None)
            m.with_solver(mb.SolverKind.ITERATIVE).with_tolerance(tol)
            handles.append(mb.SolverHandle(m, device=device))
        d_f = [torch.from_numpy(np.ascontiguousarray(l.T)).to(dev) for l in loads]  # (n_rhs, 3 N)
        d_u = [torch.zeros_like(x) for x in d_f]

        def one_pass():
            for h, F, U in zip(handles, d_f, d_u):
                if L.maille_gpu_refactor(h._h, None, None) != 0:
                    raise RuntimeError(L.maille_gpu_last_error().decode())
                for j in range(n_rhs):
                    if L.maille_gpu_solve_device(h._h, F[j].data_ptr(), U[j].data_ptr()) != 0:
                        raise RuntimeError(L.maille_gpu_last_error().decode())
        one_pass()
        torch.cuda.synchronize()
        k0 = L.maille_gpu_kernel_launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        one_pass()  # every call returns after its stream finished: the pass is serial on the GPU
        e1.record(torch.cuda.ExternalStream(handles[-1].stream))
        e1.synchronize()
        ms_pi = e0.elapsed_time(e1)
        diff = max(float(np.linalg.norm(U.cpu().numpy().T - u) / max(np.linalg.norm(u), 1e-300))
                   for U, u in zip(d_u, u_fp64))
        out["per_instance"] = {"ms_per_step": ms_pi, "value": free * n_rhs / (ms_pi / 1e3),
                               "unit": "DOF*load_cases/s",
                               "kernel_launches_per_step": L.maille_gpu_kernel_launches() - k0,
                               "max_rel_diff_vs_batched_fp64": diff,
                               "includes": "per instance: refactor (element integration, assembly, "
                                           "IC(0)) + one PCG per load case from device-resident "
                                           "loads into device memory",
                               "timing": "CUDA events around the serial pass of synchronous calls"}
        out["batched_includes"] = ("element integration, assembly, IC(0) of every instance, then one "
                                   "persistent PCG launch over every instance and load case, "
                                   "device-resident loads and displacements")
    finally:
        for h in handles:
            h.close()
    for name in ("fp64", "mixed"):
        out[f"speedup_{name}_vs_per_instance"] = out["per_instance"]["ms_per_step"] / out[name]["ms_per_step"]
    return out


def large_strain_section(mb, mg, steps, device):
    """Large-strain neo-Hookean Tet4 block (64 x 16 x 16 cells, 56 355 DOF, 98 304 tets): one
    forward = the whole quasi-static step (10 increments of Newton to 1e-8 with IC(0)-PCG inner
    solves, checkpoints kept on the device); one backward = the gradient of the final tip
    reaction force with respect to every mu_e (reverse pass: tangent at the checkpoint, one
    adjoint PCG solve, element gradient kernel). Host wall clock around the synchronous calls."""
    p, mu, tip = mg.large_strain_block()
    out = {"workload": "neo_hookean_tet4_64x16x16_10inc", "dofs": 3 * p.n_nodes, "elements": p.n_elems}
    with mb.LargeStrainSolver(p, increments=10, device=device) as s:
        h = s.run()  # warm-up
        w = np.zeros_like(h.reactions)
        w[-1, tip] = 1.0
        s.backward(w)
        fw, bw = [], []
        for _ in range(max(1, steps)):
            t0 = time.perf_counter()
            h = s.run()
            fw.append((time.perf_counter() - t0) * 1e3)
            t0 = time.perf_counter()
            gm, _ = s.backward(w)
            bw.append((time.perf_counter() - t0) * 1e3)
    out.update({"forward_ms": statistics.median(fw), "backward_ms": statistics.median(bw),
                "backward_over_forward": statistics.median(bw) / statistics.median(fw),
                "newton_total": int(h.newton_total), "pcg_total": int(h.pcg_total),
                "tip_reaction": float(h.reactions[-1, tip].sum()),
                "ms_per_pcg_iteration": statistics.median(fw) / max(1, int(h.pcg_total)),
                "roofline": None,
                "roofline_note": "no HBM roofline: the tangent matrix and factor (about 19 MB) stay in the "
                                 "126 MB L2, so the inner PCG is bound by the sweeps' latency; the kernel's "
                                 "ncu summary is profiles/k_pcg_large_strain_64x16x16.md"})
    path = os.path.join(ROOT, "tests", "golden", "large_strain_oracle_summary.json")
    if os.path.exists(path):
        g = json.load(open(path))
        el = np.array(g["elements"])
        out["grad_rel_err_vs_oracle"] = float(np.linalg.norm(gm[el] - np.array(g["dJdmu"]))
                                              / np.linalg.norm(g["dJdmu"]))
        out["tip_reaction_rel_err_vs_oracle"] = abs(out["tip_reaction"] - g["tip_reaction"][-1]) / abs(
            g["tip_reaction"][-1])
        out["oracle_cpu_note"] = "the CPU oracle's time for this workload is in the reference arm's line"
    return out


def thermal_section(mg, steps, device, hbm, cells=40, ordering=0):
    """Transient heat conduction on the Tet10 unit cube 40^3 (531 441 nodes, 524 880 free): 10
    backward-Euler increments of (C/dt + K) T_{n+1} = C/dt T_n + F, each solved by IC(0)-PCG from
    zero to 1e-12 (Model::solve_step), in FP64 and in the mixed form (FP32 matrices and vectors,
    FP64 reliable updates). One step = the whole transient through the C ABI from host buffers
    (ordering, element matrices, assembly, IC(0), the increments, the history copied back); the
    device time of the increments comes from the library's CUDA events. Roofline of the
    persistent scalar PCG: algorithmic bytes per iteration = the left matrix (values + int32
    columns) once for the SpMV and its strict triangles once per sweep, plus 16 vector passes
    (values of the storage precision)."""
    import torch
    from maille_b200 import thermal as th
    from maille_b200._lib import MAILLE_FP64, MAILLE_MIXED
    p = mg.thermal_cube(cells, True, increments=10, time_period=0.1)
    f = p.loads + th.thermal_loads(p.coords, p.conn, list(zip(p.s_elem, p.s_value)),
                                   list(zip(p.c_elem, p.c_face, p.c_film, p.c_sink)))
    # inputs and outputs in pinned host memory, as for the elastic end-to-end figure
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    for name in ("coords", "conn", "conductivity", "rho_c", "fixed", "imposed", "initial"):
        setattr(p, name, pin(getattr(p, name)))
    f = pin(f)
    res = dict(temps=pin(np.zeros((p.increments + 1, p.n_nodes))),
               reactions=pin(np.zeros((p.increments + 1, p.n_nodes))), fluxes=None,
               iterations=np.zeros(p.increments, np.int32))
    path = os.path.join(ROOT, "tests", "golden", "thermal_40_oracle_summary.json")
    golden = json.load(open(path)) if cells == 40 and os.path.exists(path) else None
    forms = {}
    for name, prec in (("fp64", MAILLE_FP64), ("mixed", MAILLE_MIXED)):
        kw = dict(f=f, fluxes=False, device=device, out=res, precision=prec, ordering=ordering)
        s, out = th.solve_problem(p, **kw)  # warm-up
        if s != 0:
            forms[name] = {"error": s}
            continue
        walls, dev = [], []
        for _ in range(max(1, steps)):
            t0 = time.perf_counter()
            s, out = th.solve_problem(p, **kw)
            walls.append((time.perf_counter() - t0) * 1e3)
            dev.append(out["info"]["ms_steps"])
        info = out["info"]
        nnz, nb, its = info["nonzeros"], info["free_nodes"], info["iterations_total"]
        vb = 8 if prec == MAILLE_FP64 else 4
        bytes_it = (vb + 4) * nnz + (vb + 4) * (nnz - nb) + 16 * vb * nb
        ms_it = statistics.median(dev) / its
        wall = statistics.median(walls)
        r = {"iterations_total": its, "iterations": out["iterations"].tolist(), "levels": info["levels"],
             "e2e_ms": wall, "e2e_value": nb * p.increments / (wall / 1e3), "unit": "DOF*increments/s",
             "ms_increments_device": statistics.median(dev), "ms_setup": info["ms_setup"],
             "ms_upload": info["ms_upload"], "ms_assembly": info["ms_assembly"], "ms_factor": info["ms_factor"],
             "ms_download": info["ms_download"], "max_rel_residual": info["max_rel_residual"],
             "roofline": {"bound": "hbm", "kernel": f"k_heat_pcg<{'double' if vb == 8 else 'float'}> "
                                                   "(persistent scalar IC(0)-PCG)",
                          "bytes_per_iteration": bytes_it, "ms_per_iteration": ms_it,
                          "achieved": bytes_it / (ms_it * 1e6), "peak": hbm,
                          "frac": bytes_it / (ms_it * 1e6) / hbm}}
        if golden:
            sample = out["temps"][-1][::golden["t_final_stride"]]
            r["max_abs_err_vs_oracle_final_T"] = float(np.max(np.abs(sample - np.array(golden["t_final_sample"]))))
        forms[name] = r
    out = {"workload": p.name + "_10inc", "free_nodes": info["free_nodes"], "nonzeros": info["nonzeros"],
           "increments": p.increments, **forms}
    if golden:
        out["oracle_iterations_total"] = golden["total_iterations"]
        out["oracle_cpu_note"] = "the CPU oracle's time for this workload is in the reference arm's line"
    if "fp64" in forms and "mixed" in forms and "e2e_ms" in forms["mixed"]:
        out["speedup_mixed_vs_fp64_device"] = forms["fp64"]["ms_increments_device"] / forms["mixed"]["ms_increments_device"]
    return out


def spmv_roofline(torch, h, L, precision, blocks, nb, reps=50):
    """Average duration of the PCG SpMV kernel over `reps` launches (CUDA events on the
    library's stream) and its algorithmic bytes: per block 9 values + one int32 column index,
    per row one int64 row pointer, the vector read once and the result written once."""
    stream = torch.cuda.ExternalStream(h.stream)
    L.maille_gpu_spmv_device(h._h, precision, 5)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    L.maille_gpu_spmv_device(h._h, precision, reps)
    end.record(stream)
    end.synchronize()
    ms = start.elapsed_time(end) / reps
    vb = 4 if precision == 1 else 8
    n = 3 * nb
    bytes_ = blocks * (9 * vb + 4) + (nb + 1) * 8 + 2 * n * vb
    return ms, bytes_


def pcg_bytes_parts(blocks, nb, vb):
    """Algorithmic bytes of one PCG iteration (values of `vb` bytes), as (matrix part, vector part
    of one right-hand side): the SpMV reads every block of K (9 values + an int32 column) and
    writes ap; the two sweeps read every strictly lower / upper block once, the diagonal inverses
    D, r, and write y / z; the vector updates read and write x, r, p, ap, z. Each node's 3 vector
    entries are counted once per read or write (the 4th padding entry is not algorithmic)."""
    off_diag = blocks - nb
    matrix = blocks * (9 * vb + 4) + off_diag * (9 * vb + 4) + 2 * nb * 9 * vb
    vec = 3 * nb * vb
    vectors = vec * (2 + 2 + 2 + 3 + 3 + 6 + 3)  # spmv p/ap, fwd r/y, bwd y/z/r, axpy, pupdate
    return matrix, vectors


def pcg_bytes_per_iteration(blocks, nb, vb):
    matrix, vectors = pcg_bytes_parts(blocks, nb, vb)
    return matrix + vectors


# DRAM traffic of the persistent PCG kernel per iteration over its algorithmic bytes, from one ncu
# capture (dram__bytes_read.sum + dram__bytes_write.sum of one 8-iteration launch, Tet10 30^3:
# 0.587 GB against 0.560 GB, kept in the profile summary of k_pcg); traffic grows with the blocks, so
# the ratio scales the capture to the benchmark size.
PCG_TRAFFIC_RATIO = 0.591 / 0.560


def cpu_baseline(p, tol, iterations_needed, max_iter=5):
    """The CPU oracle (single-thread restatement of the reference path) on the full workload:
    element integration + assembly + RCM + IC(0) + `max_iter` PCG iterations timed, the PCG part
    scaled to the oracle's iteration count at `tol` (from its recorded full run)."""
    import oracle
    r = oracle.model_solve(p, solver=2, tol=tol, max_iter=max_iter)
    per_iter = r["ms_solve"] / max(1, r["iterations"])
    total_ms = r["ms_setup"] + r["ms_factor"] + per_iter * iterations_needed
    return {"value": p.free_dofs / (total_ms / 1000.0), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": (f"oracle on the full workload: setup {r['ms_setup']:.0f} ms + IC(0) "
                       f"{r['ms_factor']:.0f} ms + {r['iterations']} PCG iterations timed "
                       f"({per_iter:.1f} ms each), PCG scaled to the oracle's {iterations_needed} "
                       f"iterations to tol {tol:g} (tests/golden summary)"),
            "ms_full_solve_estimate": total_ms}


def oracle_iterations(tol):
    path = os.path.join(ROOT, "tests", "golden", f"tet10_40_oracle_tol{tol:.0e}.json")
    if os.path.exists(path):
        return json.load(open(path))["iterations"], path
    return None, path


def oracle_section(name):
    """One workload on the CPU oracle (the single-thread restatement of the reference path),
    timed in this process: the plain Tet4 20^3 configuration (IC(0)-PCG to 1e-10), the transient
    thermal step on the Tet10 40^3 cube (10 increments, PCG to 1e-12) or the large-strain block
    (10 increments of Newton to 1e-8). Runs in a worker process of the reference arm."""
    import oracle
    from maille_b200 import meshgen as mg
    t0 = time.perf_counter()
    if name in ("plain_tet4_20", "plain_tet4_20_tol1e-12"):
        tol = 1e-12 if name.endswith("1e-12") else 1e-10
        p = mg.plain_tet4(20)
        r = oracle.model_solve(p, solver=2, tol=tol)
        wall = time.perf_counter() - t0
        return {"workload": "tet4_20^3_plain_fp64", "tol": tol, "status": r["status"], "free_dofs": p.free_dofs,
                "iterations": r["iterations"], "wall_s": wall, "value": p.free_dofs / wall, "unit": UNIT}
    if name == "thermal":
        p = mg.thermal_cube(40, True, increments=10, time_period=0.1)
        r = oracle.thermal_transient(p, solver=2, fluxes=False)
        wall = time.perf_counter() - t0
        return {"workload": p.name + "_10inc", "status": r["status"], "free_nodes": int(r["free"]),
                "iterations_total": int(r["total_iterations"]), "wall_s": wall,
                "value": int(r["free"]) * p.increments / wall, "unit": "DOF*increments/s"}
    if name == "large_strain":
        p, mu, tip = mg.large_strain_block()
        r = oracle.large_strain_run(p, increments=10)
        wall = time.perf_counter() - t0
        return {"workload": "neo_hookean_tet4_64x16x16_10inc", "status": r["status"],
                "newton_total": r["newton_total"], "pcg_total": r["pcg_total"], "forward_wall_s": wall}
    raise ValueError(name)


def run_reference(args):
    """The reference arm: the CPU oracle (the reference's IC(0)-PCG path restated in C++, one
    thread: the reference is single-threaded) on the headline workload, measured as ONE full
    solve (element integration, assembly, RCM, IC(0), every PCG iteration to --tol, reactions and
    stresses): at about 3 minutes a solve, that one solve is the whole timed region, so the line
    says steps = 1 whatever --steps asks. Beside it, each in a worker process of its own (one
    thread each, run at the same time as the headline solve on other host cores), the oracle's
    times for the plain Tet4 20^3 configuration, the transient thermal step and the large-strain
    block, which bench.py's own arm reports on the GPU."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from concurrent.futures import ProcessPoolExecutor
    import multiprocessing as mproc
    from maille_b200 import meshgen as mg
    import oracle
    oracle.build()
    p = mg.mixed_tet10(args.cells)
    small = mg.mixed_tet10(4)
    for _ in range(args.warmup):  # untimed warm-up on a small mesh of the same family
        oracle.model_solve(small, solver=2, tol=args.tol)
    sides = ["plain_tet4_20", "plain_tet4_20_tol1e-12", "thermal", "large_strain"]
    cores = os.cpu_count() or 1
    pool = None
    futures = {}
    if cores >= len(sides) + 1 and args.cells == 40:
        pool = ProcessPoolExecutor(max_workers=len(sides), mp_context=mproc.get_context("spawn"))
        futures = {n: pool.submit(oracle_section, n) for n in sides}
    t0 = time.perf_counter()
    r = oracle.model_solve(p, solver=2, tol=args.tol)
    wall = time.perf_counter() - t0
    sections = {}
    if pool is not None:
        for n, fut in futures.items():
            try:
                sections[n] = fut.result(timeout=900)
            except Exception as e:  # a section that failed is reported, not fatal
                sections[n] = {"error": repr(e)}
        pool.shutdown()
    if r["status"] != 0:
        print(json.dumps({"impl": "reference", "unavailable": f"the oracle solve ended with status {r['status']}"}))
        return
    value = p.free_dofs / wall
    sample = (f"one full solve of the workload to tol {args.tol:g}: setup (element integration, assembly, "
              f"RCM) {r['ms_setup']:.0f} ms + IC(0) {r['ms_factor']:.0f} ms + {r['iterations']} PCG iterations "
              f"{r['ms_solve']:.0f} ms, wall {wall:.1f} s")
    need = oracle_iterations(args.tol)[0] if args.cells == 40 else None
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": 1, "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": wall * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"tet10_{args.cells}^3_lognormal_mixed", "free_dofs": p.free_dofs,
                   "tol": args.tol},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample,
                         "iterations": r["iterations"], "recorded_iterations": need,
                         "rel_residual": r["rel_residual"], "shift": r["shift"]},
        "sections": sections,
        "host_cores": cores,
        "note": ("the oracle is single-threaded like the reference; the side sections ran at the same "
                 "time in worker processes, one thread each, on other host cores"),
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def run_only(args):
    """One form, W + K steps of refactor + solve, nothing else (for profiler launch lists); with
    --only thermal, the thermal section's transient (W + K runs of the whole step); with --only
    batched, W + K batched FP64 solves of --batch-count instances (refactor + solve); with --only
    large_strain, W + K runs of the large-strain block (64 x 16 x 16 cells, 10 increments)."""
    if args.only == "batched":
        import torch
        import maille_b200 as mb
        from maille_b200 import meshgen as mg
        probs, loads = mg.batched_tet4(count=args.batch_count)
        with mb.BatchSolver(probs, loads, tol=args.tol) as b:
            for _ in range(args.warmup + args.steps):
                b.refactor()
                fld = b.solve()
        print(json.dumps({"only": "batched", "instances": len(probs), "max_iterations": int(fld.iterations.max()),
                          "ms_solve": fld.info["ms_solve"]}))
        return
    if args.only == "large_strain":
        import maille_b200 as mb
        from maille_b200 import meshgen as mg
        p, mu, tip = mg.large_strain_block()
        with mb.LargeStrainSolver(p, increments=10) as s:
            for _ in range(args.warmup + args.steps):
                h = s.run()
        print(json.dumps({"only": "large_strain", "newton_total": int(h.newton_total),
                          "pcg_total": int(h.pcg_total), "ms_total": h.ms_total}))
        return
    if args.only in ("thermal", "thermal_mixed"):
        from maille_b200 import meshgen as mg, thermal as th
        p = mg.thermal_cube(args.thermal_cells, True, increments=10, time_period=0.1)
        f = p.loads + th.thermal_loads(p.coords, p.conn, list(zip(p.s_elem, p.s_value)),
                                       list(zip(p.c_elem, p.c_face, p.c_film, p.c_sink)))
        prec = 1 if args.only == "thermal_mixed" else 0
        for _ in range(args.warmup + args.steps):
            s, out = th.solve_problem(p, f=f, fluxes=False, precision=prec, ordering=ORDERING)
            if s != 0:
                raise SystemExit(f"thermal transient failed with status {s}")
        print(json.dumps({"only": args.only, "workload": p.name + "_10inc", "ordering": args.ordering,
                          "iterations": out["info"]["iterations_total"], "levels": out["info"]["levels"],
                          "ms_increments_device": out["info"]["ms_steps"],
                          "ms_per_iteration": out["info"]["ms_steps"] / out["info"]["iterations_total"]}))
        return
    import torch
    import maille_b200 as mb
    from maille_b200 import meshgen as mg
    from maille_b200._lib import MAILLE_FP64, MAILLE_MIXED
    from maille_b200.model import face_pressure_loads
    torch.cuda.set_device(0)
    L = mb._lib.load()
    p = mg.mixed_tet10(args.cells)
    p.loads = face_pressure_loads(p.coords, p.conn, list(zip(p.p_elem, p.p_face, p.p_value)))
    p.p_elem, p.p_face, p.p_value = p.p_elem[:0], p.p_face[:0], p.p_value[:0]
    prec = MAILLE_MIXED if args.only == "mixed" else MAILLE_FP64
    h = mb.SolverHandle(solve_model(mb, p, prec, args.tol, 0), device=0)
    ms, info, launches = time_handle(torch, h, args.steps, args.warmup, L)
    h.close()
    print(json.dumps({"only": args.only, "workload": f"tet10_{args.cells}^3", "ordering": args.ordering,
                      "ms_per_step": ms, "iterations": info["iterations"], "updates": info["outer_iterations"],
                      "levels": info["levels"], "ms_solve": info["ms_solve"],
                      "ms_per_iteration": info["ms_solve"] / max(1, info["iterations"]),
                      "launches_per_step": launches}))


def run_ours(args):
    import torch
    import maille_b200 as mb
    from maille_b200 import meshgen as mg
    from maille_b200._lib import MAILLE_FP64, MAILLE_MIXED, ElasticResult
    from maille_b200.model import problem_struct, face_pressure_loads
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    L = mb._lib.load()
    p = mg.mixed_tet10(args.cells)
    f = face_pressure_loads(p.coords, p.conn, list(zip(p.p_elem, p.p_face, p.p_value)))
    p.loads = f
    p.p_elem, p.p_face, p.p_value = p.p_elem[:0], p.p_face[:0], p.p_value[:0]

    # tight FP64 reference solution (untimed) for the accuracy check
    ref = solve_model(mb, p, MAILLE_FP64, 1e-13, local).solve(device=local)
    u_ref = ref.displacements

    hm = mb.SolverHandle(solve_model(mb, p, MAILLE_MIXED, args.tol, local), device=local)
    clocks = Clocks(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ms_mixed, info_m, launches = time_handle(torch, hm, args.steps, args.warmup, L)
    clk = clocks.stop()
    mixed_field = hm.solve()
    err_mixed = float(np.linalg.norm(mixed_field.displacements - u_ref) / np.linalg.norm(u_ref))
    # and against the CPU oracle's own full-size solve at 1e-13 (sampled DOFs and compliance of
    # the committed golden summary), so the accuracy gate does not rest on the GPU alone
    err_oracle = None
    gpath = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden",
                         "tet10_40_oracle_tol1e-13.json")
    if args.cells == 40 and os.path.exists(gpath):
        with open(gpath) as fh:
            gold = json.load(fh)
        dofs, gu = np.array(gold["dofs"]), np.array(gold["u"])
        err_oracle = {
            "rel_err_sampled_dofs": float(np.linalg.norm(mixed_field.displacements[dofs] - gu) / np.linalg.norm(gu)),
            "rel_err_compliance": float(abs(f @ mixed_field.displacements - gold["compliance"]) / abs(gold["compliance"])),
            "samples": int(dofs.size), "oracle_tol": gold["tol"]}

    # max over ranks of the per-step time
    if world > 1:
        t = torch.tensor([ms_mixed], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_mixed = float(t.item())
    free = p.free_dofs
    value = world * free / (ms_mixed / 1000.0)

    # SpMV roofline (FP32 SpMV of the inner PCG, and the FP64 SpMV of the refinement)
    hbm, peak_kind = peaks()
    ms32, bytes32 = spmv_roofline(torch, hm, L, MAILLE_MIXED, info_m["blocks"], info_m["block_rows"])
    ms64, bytes64 = spmv_roofline(torch, hm, L, MAILLE_FP64, info_m["blocks"], info_m["block_rows"])
    gbs32, gbs64 = bytes32 / ms32 / 1e6, bytes64 / ms64 / 1e6
    hm.close()
    it_bytes = pcg_bytes_per_iteration(info_m["blocks"], info_m["block_rows"], 4)
    pcg_gbs = it_bytes * info_m["iterations"] / info_m["ms_solve"] / 1e6

    plain = None
    if not args.no_plain:
        hp = mb.SolverHandle(solve_model(mb, p, MAILLE_FP64, args.tol, local), device=local)
        ms_plain, info_p, _ = time_handle(torch, hp, args.steps, max(1, args.warmup - 1), L)
        plain_field = hp.solve()
        hp.close()
        if world > 1:
            t = torch.tensor([ms_plain], device="cuda")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ms_plain = float(t.item())
        plain = {"value": world * free / (ms_plain / 1000.0), "ms_per_step": ms_plain,
                 "iterations": info_p["iterations"],
                 "rel_err_vs_fp64": float(np.linalg.norm(plain_field.displacements - u_ref) / np.linalg.norm(u_ref)),
                 "ms_assembly": info_p["ms_assembly"], "ms_factor": info_p["ms_factor"],
                 "ms_solve": info_p["ms_solve"]}

    # end to end through the C ABI: host buffers (pinned), create + solve + results + destroy
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    coords, conn, young, poisson = pin(p.coords), pin(p.conn.astype(np.int64)), pin(p.young), pin(p.poisson)
    fixed, imposed, floads = pin(p.fixed), pin(p.imposed), pin(f)
    prob, keep = problem_struct(coords, conn, young, poisson, fixed, imposed, floads, args.tol,
                                10000, MAILLE_MIXED, ORDERING, local)
    ng = 4
    outs = dict(u=pin(np.zeros(3 * p.n_nodes)), r=pin(np.zeros(3 * p.n_nodes)),
                g=pin(np.zeros(p.n_elems * ng * 9)), vm=pin(np.zeros(p.n_elems * ng)))
    from maille_b200._lib import ptr, _d
    res = ElasticResult(u=ptr(outs["u"], _d), reactions=ptr(outs["r"], _d),
                        gauss_stress=ptr(outs["g"], _d), von_mises=ptr(outs["vm"], _d))
    assert L.maille_gpu_elastic_solve(ctypes.byref(prob), ctypes.byref(res)) == 0
    if world > 1:
        torch.distributed.barrier()
    walls = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        t1 = time.perf_counter()
        s = L.maille_gpu_elastic_solve(ctypes.byref(prob), ctypes.byref(res))
        if s != 0:
            raise RuntimeError(L.maille_gpu_last_error().decode())
        walls.append((time.perf_counter() - t1) * 1000.0)
    e2e_ms = (time.perf_counter() - t0) * 1000.0 / args.steps
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())
    h2d = sum(a.nbytes for a in (coords, conn, young, poisson, fixed, imposed, floads))
    d2h = sum(a.nbytes for a in outs.values())
    e2e = {"value": world * free / (e2e_ms / 1000.0), "unit": UNIT, "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms, "step_walls_ms": walls,
           "phases_ms": {k: getattr(res, k) for k in ("ms_setup", "ms_upload", "ms_element",
                                                      "ms_ordering", "ms_symbolic", "ms_buffers",
                                                      "ms_assembly", "ms_factor", "ms_solve", "ms_post",
                                                      "ms_download")},
           "phases_note": ("ms_setup is the host thread (incidence, boundary lists), which runs while the "
                           "device takes the inputs and orders the nodes; the other phases follow one "
                           "another (ms_ordering: the device ordering, wall time)")}

    plain_tet4 = plain_tet4_section(torch, mb, mg, L, args.steps, args.warmup, local)
    # the same configuration at the reference's default tolerance (iterative.rs:9)
    plain_tet4_12 = plain_tet4_section(torch, mb, mg, L, args.steps, args.warmup, local, tol=1e-12)

    batched = None
    if not args.no_batched:
        batched = batched_section(torch, mb, mg, L, args.batch_count, args.tol, args.steps,
                                  args.warmup, local, hbm, rank, world)

    large_strain = None
    if not args.no_large_strain:
        large_strain = large_strain_section(mb, mg, args.steps, local)

    thermal = None
    if not args.no_thermal:
        thermal = thermal_section(mg, args.steps, local, hbm, args.thermal_cells)

    adjoint = None
    if not args.no_adjoint:
        adjoint = adjoint_section(torch, mb, mg, L, args.adjoint_cells, args.tol, args.steps,
                                  args.warmup, local, hbm)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        need, path = oracle_iterations(args.tol)
        if need is not None:
            cpu = cpu_baseline(p, args.tol, need)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64 mixed", "data": "synthetic",
        "config": {"workload": f"tet10_{args.cells}^3_lognormal_mixed", "free_dofs": free,
                   "tol": args.tol, "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2 (matrices > 1 GB)", "ordering": args.ordering,
                   "levels": info_m["levels"], "blocks": info_m["blocks"]},
        "accuracy": {"rel_err_vs_fp64": err_mixed, "target": 1e-8,
                     "ok": err_mixed <= 1e-8 and (err_oracle is None or err_oracle["rel_err_sampled_dofs"] <= 1e-8),
                     "vs_oracle": err_oracle},
        "mixed": {"iterations": info_m["iterations"], "outer": info_m["outer_iterations"],
                  "ms_assembly": info_m["ms_assembly"], "ms_factor": info_m["ms_factor"],
                  "ms_solve": info_m["ms_solve"], "ms_post": info_m["ms_post"]},
        "plain_fp64": plain,
        "speedup_mixed_vs_plain": (plain["ms_per_step"] / ms_mixed) if plain else None,
        "roofline": {"bound": "hbm",
                     "kernel": "k_pcg<float> persistent mixed PCG (SpMV + IC(0) sweeps + updates)",
                     "achieved": pcg_gbs, "peak": hbm, "unit": "GB/s", "frac": pcg_gbs / hbm,
                     "peak_kind": peak_kind, "bytes_per_iteration": it_bytes,
                     "ms_per_iteration": info_m["ms_solve"] / info_m["iterations"],
                     "traffic": PCG_TRAFFIC_RATIO * it_bytes,
                     "traffic_note": "bytes per iteration, ncu DRAM bytes of a Tet10 30^3 launch "
                                     "scaled by blocks (the k_pcg Tet10 30^3 profile summary)"},
        "spmv": {"kernel": "k_spmv<float> (SELL 3x3-block SpMV, FP32, standalone)",
                 "achieved": gbs32, "frac": gbs32 / hbm, "bytes_per_launch": bytes32,
                 "ms_per_launch": ms32,
                 "fp64": {"achieved": gbs64, "frac": gbs64 / hbm, "bytes_per_launch": bytes64,
                          "ms_per_launch": ms64}},
        "plain_tet4_20": plain_tet4,
        "plain_tet4_20_tol1e-12": plain_tet4_12,
        "batched": batched,
        "large_strain": large_strain,
        "adjoint": adjoint,
        "thermal": thermal,
        "e2e": e2e, "cpu_baseline": cpu, "clocks": clk, "gpu_launches": launches,
    }
    print(json.dumps(line))


def main():
    global ORDERING
    args = parse()
    ORDERING = ORDERINGS[args.ordering]
    if args.impl == "reference":
        run_reference(args)
    elif args.only:
        run_only(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
