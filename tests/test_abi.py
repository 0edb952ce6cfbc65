"""CPU tests of the C ABI boundary and the host logic: the library loads, exports every symbol
include/maille_gpu.h declares, validates its inputs before touching a device, and the host-side
helpers agree with the oracle. No GPU compute runs here."""
import ctypes
import os
import re

import numpy as np
import pytest

import cases
import maille_b200 as mb
from maille_b200 import _lib, build, meshgen as mg
from maille_b200.model import problem_struct

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def header_functions():
    text = open(os.path.join(ROOT, "include", "maille_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(maille_gpu_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(lib):
    names = header_functions()
    assert "maille_gpu_elastic_solve" in names and len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_build_recipe_targets_sm100a_only():
    assert "arch=compute_100a,code=sm_100a" in build.FLAGS
    assert sum("arch=" in f for f in build.FLAGS) == 1


def test_version_and_device_count_need_no_gpu(lib):
    assert b"sm_100a" in lib.maille_gpu_version()
    assert lib.maille_gpu_device_count() >= 0


STRUCTS = (("MailleElasticProblem", _lib.ElasticProblem), ("MailleElasticResult", _lib.ElasticResult),
           ("MailleBatchProblem", _lib.BatchProblem), ("MailleBatchResult", _lib.BatchResult),
           ("MailleLargeStrainProblem", _lib.LargeStrainProblem),
           ("MailleLargeStrainResult", _lib.LargeStrainResult),
           ("MailleThermalProblem", _lib.ThermalProblem), ("MailleThermalResult", _lib.ThermalResult))


def test_struct_layouts_match_the_header(tmp_path):
    """Field offsets of the ctypes structs equal those gcc computes from include/maille_gpu.h."""
    import subprocess
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "maille_gpu.h"', "int main(void) {"]
    for cname, py in STRUCTS:
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l}
    for cname, py in STRUCTS:
        assert got[(cname, "size")] == ctypes.sizeof(py)
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def _solve_status(lib, p):
    r = _lib.ElasticResult()
    return lib.maille_gpu_elastic_solve(ctypes.byref(p), ctypes.byref(r))


def test_invalid_inputs_are_rejected_before_any_device_work(lib):
    p0 = mg.plain_tet4(2)
    good = dict(coords=p0.coords, conn=p0.conn, young=p0.young, poisson=p0.poisson,
                fixed=p0.fixed, imposed=p0.imposed, f=p0.loads)

    def status(**kw):
        args = dict(good)
        args.update(kw)
        p, keep = problem_struct(**args)
        return _solve_status(lib, p)

    bad_conn = p0.conn.copy()
    bad_conn[3, 2] = p0.coords.shape[0] + 5
    assert status(conn=bad_conn) == _lib.MAILLE_INVALID_INPUT
    assert "unknown node" in _lib.last_error()
    coords = p0.coords.copy()
    coords[1, 0] = np.nan
    assert status(coords=coords) == _lib.MAILLE_INVALID_INPUT
    assert status(young=-p0.young) == _lib.MAILLE_INVALID_INPUT
    f = p0.loads.copy()
    f[4] = np.inf
    assert status(f=f) == _lib.MAILLE_INVALID_INPUT
    assert status(fixed=np.ones_like(p0.fixed)) == _lib.MAILLE_INVALID_INPUT  # nothing free
    assert lib.maille_gpu_elastic_solve(None, None) == _lib.MAILLE_INVALID_INPUT
    p, keep = problem_struct(**good)
    p.ordering = 5
    assert _solve_status(lib, p) == _lib.MAILLE_INVALID_INPUT and "ordering" in _lib.last_error()
    # wrong element family
    p, keep = problem_struct(**good)
    p.nodes_per_elem = 5
    p.n_elems = p0.conn.size // 5
    assert _solve_status(lib, p) == _lib.MAILLE_INVALID_INPUT


def test_handle_entry_points_reject_null_arguments_without_device_work(lib):
    out = np.zeros(6)
    assert lib.maille_gpu_nodal_stresses(None, _lib.ptr(out, _lib._d), _lib.ptr(out, _lib._d)) == _lib.MAILLE_INVALID_INPUT
    assert lib.maille_gpu_wait_selftest(0, 1, None) == _lib.MAILLE_INVALID_INPUT
    assert "null" in _lib.last_error()
    # cancel flags: a null handle is ignored, a device ordinal out of range is refused
    assert lib.maille_gpu_solve_device(None, None, None) == _lib.MAILLE_INVALID_INPUT
    lib.maille_gpu_large_strain_cancel(None, 1)
    lib.maille_gpu_cancel(None, 1)
    lib.maille_gpu_batch_cancel(None, 1)
    assert lib.maille_gpu_thermal_cancel(64, 1) == _lib.MAILLE_INVALID_INPUT
    assert lib.maille_gpu_thermal_cancel(-1, 0) == _lib.MAILLE_INVALID_INPUT


def test_no_alloc_entry_point_checks_its_arguments_without_device_work(lib):
    # the pointers are never dereferenced: every check runs on the host before the device is used
    f = lib.maille_gpu_bsr3_spmv_dot_noalloc
    base = 1 << 20
    assert f(0, 4, base, base, base, base, base + 8, base + 4096, None) == _lib.MAILLE_INVALID_INPUT
    assert "overlap" in _lib.last_error()
    assert f(0, 4, base, base, base, base, base + 96, base + 100, None) == _lib.MAILLE_INVALID_INPUT
    assert f(0, -1, base, base, base, base, base + 96, base + 200, None) == _lib.MAILLE_INVALID_INPUT
    assert f(0, 4, None, base, base, base, base + 96, base + 200, None) == _lib.MAILLE_INVALID_INPUT
    assert f(64, 4, base, base, base, base, base + 96, base + 200, None) == _lib.MAILLE_INVALID_INPUT


def test_missing_device_is_a_cuda_error_not_a_fallback(lib):
    if lib.maille_gpu_device_count() > 0:
        pytest.skip("a device is visible")
    p0 = mg.plain_tet4(2)
    p, keep = problem_struct(p0.coords, p0.conn, p0.young, p0.poisson, p0.fixed, p0.imposed,
                             p0.loads)
    assert _solve_status(lib, p) == _lib.MAILLE_CUDA_ERROR


@pytest.mark.parametrize("quadratic", [False, True])
def test_face_pressure_helper_matches_the_oracle(lib, oracle_lib, quadratic):
    p = cases.hydrostatic(quadratic)
    f = mb.face_pressure_loads(p.coords, p.conn, list(zip(p.p_elem, p.p_face, p.p_value)))
    r = oracle_lib.model_solve(p, solver=1)
    assert np.abs(f - r["f"]).max() < 1e-13
    # resultant: -p * area on each loaded unit face
    for c in range(3):
        assert abs(f[c::3].sum() + 50.0) < 1e-12


def test_mesh_validation_mirrors_mesh_new():
    # tests/solid.rs bad_tetrahedra_are_refused_with_their_index
    nodes = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0]], float)
    with pytest.raises(mb.MailleError) as e:
        mb.Mesh(nodes, [[0, 1, 2, 3], [0, 2, 1, 3]], 210e3, 0.3)
    assert e.value.kind == "InvertedTetrahedron" and "element 1" in str(e.value)
    with pytest.raises(mb.MailleError) as e:
        mb.Mesh(nodes, [[0, 1, 2, 4]], 210e3, 0.3)
    assert e.value.kind == "DegenerateTetrahedron"
    q_nodes, q_conn = mg.to_quadratic_tet(nodes[:4], np.array([[0, 1, 2, 3]]))
    q_nodes[4] += [0.0, 0.1, 0.0]
    with pytest.raises(mb.MailleError) as e:
        mb.Mesh(q_nodes, q_conn, 210e3, 0.3)
    assert e.value.kind == "CurvedTetrahedron"
    with pytest.raises(mb.MailleError):
        mb.Mesh(nodes, [[0, 1, 2, 9]], 210e3, 0.3)


def test_solver_kind_selection_follows_the_reference():
    # solve.rs:185-195
    assert mb.ITERATIVE_FROM == 100_000
    assert not mb.SolverKind.AUTO.is_iterative(99_999)
    assert mb.SolverKind.AUTO.is_iterative(100_000)
    assert mb.SolverKind.ITERATIVE.is_iterative(1)
    assert not mb.SolverKind.DIRECT.is_iterative(10 ** 7)
    m = mb.Model.from_arrays(*_small_arrays())
    with pytest.raises(mb.MailleError) as e:
        m.solve()  # Auto below the threshold selects the host's skyline solver
    assert e.value.kind == "DirectSolverOnHost"


def _small_arrays():
    p = mg.plain_tet4(2)
    return p.coords, p.conn, p.young, p.poisson, p.fixed


def test_meshgen_matches_the_reference_mesh_sizes():
    # box_grid / to_quadratic_tet node and element counts of the benchmark meshes
    nodes, tets = mg.box_grid((20, 20, 20), (1, 1, 1))
    assert nodes.shape == (9261, 3) and tets.shape == (48000, 4)
    n10, c10 = mg.to_quadratic_tet(*mg.box_grid((6, 6, 6), (1, 1, 1)))
    assert n10.shape[0] == 13 ** 3 and c10.shape == (6 * 216, 10)
    # every tet is positively oriented and Tet10 mids sit at the edge midpoints
    e = nodes[tets[:, 1:]] - nodes[tets[:, :1]]
    assert (np.einsum("ij,ij->i", e[:, 0], np.cross(e[:, 1], e[:, 2])) > 0).all()
    for k, (a, b) in enumerate(mg.TET10_EDGES):
        assert np.allclose(n10[c10[:, 4 + k]], 0.5 * (n10[c10[:, a]] + n10[c10[:, b]]))
    # first-encounter numbering of the mid nodes (the reference's HashMap insertion order)
    first = c10[:, 4:].ravel()
    seen = []
    for v in first:
        if v not in seen:
            seen.append(v)
        if len(seen) > 50:
            break
    assert seen == list(range(7 ** 3, 7 ** 3 + len(seen)))


def test_workload_generators_are_seeded_and_shaped():
    a = mg.uniform(3, 5)
    assert np.array_equal(a, mg.uniform(3, 5)) and (a >= 0).all() and (a < 1).all()
    z = mg.normal(2, 200000)
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1) < 0.01
    p = mg.plain_tet4(20)
    assert p.free_dofs == 26460 and p.p_elem.size == 800
    p, rho = mg.simp_tet4(4)
    assert np.allclose(p.young, 210000 * rho ** 3) and rho.min() >= 0.01 and rho.max() <= 1.0


# --- transient thermal: host helper and input checks ---------------------------------------------

@pytest.mark.parametrize("quadratic", [False, True])
def test_thermal_load_helper_matches_the_oracle(lib, oracle_lib, quadratic):
    from maille_b200 import thermal as th
    p = mg.thermal_cube(3, quadratic, increments=1)
    f = th.thermal_loads(p.coords, p.conn, list(zip(p.s_elem, p.s_value)),
                         list(zip(p.c_elem, p.c_face, p.c_film, p.c_sink)))
    ref = oracle_lib.thermal_transient(p, solver=1, fluxes=False)
    assert ref["status"] == 0
    assert np.abs(f - ref["f"]).max() <= 1e-13 * np.abs(ref["f"]).max()
    # totals: source q V over the unit cube plus h T_inf over the unit top face
    assert abs(f.sum() - (50.0 + 10.0 * 20.0)) < 1e-10


def test_thermal_inputs_are_rejected_before_any_device_work(lib):
    from maille_b200 import thermal as th
    p0 = mg.thermal_cube(2, False, increments=2)
    good = dict(coords=p0.coords, conn=p0.conn, conductivity=p0.conductivity, rho_c=p0.rho_c,
                fixed=p0.fixed, imposed=p0.imposed, f=None, initial=p0.initial, time_step=0.1,
                theta=1.0, increments=2)

    def status(**kw):
        args = dict(good)
        args.update(kw)
        p, keep = th.thermal_problem_struct(**args)
        r = _lib.ThermalResult()
        return lib.maille_gpu_thermal_transient(ctypes.byref(p), ctypes.byref(r))

    assert status(theta=0.4) == _lib.MAILLE_INVALID_INPUT and "theta" in _lib.last_error()
    assert status(precision=7) == _lib.MAILLE_INVALID_INPUT and "precision" in _lib.last_error()
    assert status(precision=1, increments=600000) == _lib.MAILLE_INVALID_INPUT and "32-bit" in _lib.last_error()
    assert status(theta=float("nan")) == _lib.MAILLE_INVALID_INPUT
    assert status(increments=0) == _lib.MAILLE_INVALID_INPUT
    assert status(time_step=0.0) == _lib.MAILLE_INVALID_INPUT
    bad = p0.initial.copy()
    bad[2] = np.nan
    assert status(initial=bad) == _lib.MAILLE_INVALID_INPUT and "node 2" in _lib.last_error()
    conn = p0.conn.copy()
    conn[1, 1] = p0.coords.shape[0]
    assert status(conn=conn) == _lib.MAILLE_INVALID_INPUT and "unknown node" in _lib.last_error()
    assert status(fixed=np.ones_like(p0.fixed)) == _lib.MAILLE_INVALID_INPUT
    assert status(ordering=-1) == _lib.MAILLE_INVALID_INPUT and "ordering" in _lib.last_error()
    assert lib.maille_gpu_thermal_transient(None, None) == _lib.MAILLE_INVALID_INPUT
    if lib.maille_gpu_device_count() == 0:
        assert status() == _lib.MAILLE_CUDA_ERROR  # a valid problem needs a device: no fallback


def test_thermal_step_validation_mirrors_the_reference():
    # tests/transient.rs:476-500
    from maille_b200.thermal import Step
    with pytest.raises(mb.MailleError) as e:
        Step.transient(0.0, 10)
    assert e.value.kind == "InvalidProperty"
    with pytest.raises(mb.MailleError) as e:
        Step.transient(1.0, 0)
    assert e.value.kind == "NoIncrements"
    step = Step.transient(1.0, 10)
    with pytest.raises(mb.MailleError) as e:
        step.with_theta(0.4)
    assert e.value.kind == "ThetaOutOfRange"
    with pytest.raises(mb.MailleError):
        step.with_theta(float("nan"))
    assert abs(step.with_theta(0.5).time_step - 0.1) < 1e-15
    nodes, tets = mg.box_grid((1, 1, 1), (1.0, 1.0, 1.0))
    model = mb.ThermalModel(nodes, tets, 1.0, 1.0)
    with pytest.raises(mb.MailleError) as e:
        model.solve_step(step, [0.0])
    assert e.value.kind == "TemperatureCount"
    t = np.zeros(nodes.shape[0])
    t[2] = np.nan
    with pytest.raises(mb.MailleError) as e:
        model.solve_step(step, t)
    assert e.value.kind == "NonFiniteTemperature"


def test_thermal_load_helper_ignores_out_of_range_items_and_integrates_exactly(lib):
    # face_rule gives None for a face outside 0..3; an unknown element adds nothing either. On a
    # unit top face, sum of h T_inf int N dS is h T_inf (area 1) for Tet4 and Tet10 faces alike,
    # and a uniform source q over the unit cube gives q in total.
    from maille_b200 import thermal as th
    for quadratic in (False, True):
        nodes, tets = mg.box_grid((2, 2, 2), (1.0, 1.0, 1.0))
        conn = tets
        if quadratic:
            nodes, conn = mg.to_quadratic_tet(nodes, tets)
        ce, cf = mg.faces_on(nodes, conn, 2, 1.0)
        conv = [(int(e), int(f), 2.0, 30.0) for e, f in zip(ce, cf)]
        base = th.thermal_loads(nodes, conn, [(e, 5.0) for e in range(conn.shape[0])], conv)
        assert abs(base.sum() - (5.0 + 2.0 * 30.0)) < 1e-12
        noisy = th.thermal_loads(nodes, conn, [(e, 5.0) for e in range(conn.shape[0])] + [(conn.shape[0] + 3, 1.0)],
                                 conv + [(0, 7, 2.0, 30.0), (conn.shape[0], 0, 2.0, 30.0)])
        assert np.array_equal(base, noisy)


def _build_harness(tmp_path):
    import subprocess
    exe = tmp_path / "abi_harness"
    libdir = os.path.join(ROOT, "maille_b200")
    subprocess.run(["gcc", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "abi_harness.c"), "-L", libdir, "-lmaille_gpu",
                    f"-Wl,-rpath,{libdir}", "-lm", "-o", str(exe)], check=True)
    return exe


def test_c_harness_drives_the_abi_without_python(lib, tmp_path):
    # the C ABI from C (as a foreign binding calls it): compiles warning-free against the header,
    # links against the library, and without a device every call reports MAILLE_CUDA_ERROR
    import subprocess
    exe = _build_harness(tmp_path)
    if lib.maille_gpu_device_count() > 0:
        pytest.skip("a device is visible (tests/test_gpu_abi_harness.py runs it)")
    out = subprocess.run([str(exe), "3"], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "elastic status 4" in out.stdout and "thermal status 4" in out.stdout


def _header_text():
    return open(os.path.join(ROOT, "include", "maille_gpu.h")).read()


def test_rust_bindings_mirror_the_header():
    """crates/maille-gpu-sys cannot be compiled here (no Rust toolchain): check its declarations
    against include/maille_gpu.h as text. Every header function is declared with as many
    parameters, and every problem/result struct lists the header's fields in the header's order."""
    import re
    hdr = re.sub(r"/\*.*?\*/", "", _header_text(), flags=re.S)
    rs = open(os.path.join(ROOT, "crates", "maille-gpu-sys", "src", "lib.rs")).read()
    rs = re.sub(r"//[^\n]*", "", rs)

    def nparams(args):
        args = args.strip().rstrip(",")  # rustfmt leaves a trailing comma on multi-line lists
        return 0 if args in ("", "void") else args.count(",") + 1

    hfun = {m.group(1): nparams(m.group(2)) for m in re.finditer(r"\b(maille_gpu_\w+)\s*\(([^)]*)\)\s*;", hdr)}
    block = rs[rs.index('extern "C" {'):]
    block = block[:block.index("\n}\n")]
    rfun = {m.group(1): nparams(m.group(2)) for m in re.finditer(r"pub fn (maille_gpu_\w+)\s*\(([^)]*)\)", block)}
    assert len(hfun) >= 30
    assert hfun == rfun, set(hfun.items()) ^ set(rfun.items())

    for m in re.finditer(r"typedef struct \{(.*?)\}\s*(\w+);", hdr, flags=re.S):
        body, name = m.group(1), m.group(2)
        fields = []
        for decl in re.findall(r"[^;]+;", body):
            parts = [d.strip() for d in decl.strip().rstrip(";").split(",")]
            fields.append(parts[0].split()[-1].lstrip("*"))  # "const double* coords" -> coords
            fields += [d.lstrip("*") for d in parts[1:]]       # "double ms_setup, ms_upload"
        r = re.search(r"pub struct " + name + r" \{(.*?)\n\}", rs, flags=re.S)
        assert r, name
        assert re.findall(r"pub (\w+):", r.group(1)) == fields, name
