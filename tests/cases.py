"""Problem builders restating the setups of the reference's tests for this path (paths relative
to crates/maille-core of the reference): the uniform-strain patch test (tests/solid.rs:52-116),
uniaxial traction (tests/solid.rs:118-175), the cantilever vs beam theory (tests/solid.rs:186-279),
the hydrostatic cube under face pressure (tests/pressure.rs:194-224), the PCG-vs-direct Tet10
cantilever and the unconstrained structure (tests/iterative.rs:45-83, 199-224), the
reference's examples/cube model (tests/golden/cube_example.json), and a nearly incompressible
block on which IC(0) breaks down at the first diagonal shifts (the ladder of Pcg::new,
iterative.rs:14, 201-207)."""
from __future__ import annotations

import json
import os

import numpy as np

from maille_b200 import meshgen as mg
from maille_b200.meshgen import Problem

E = 210e3
NU = 0.3
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def box(n, size, quadratic):
    nodes, tets = mg.box_grid(n, size)
    if quadratic:
        nodes, tets = mg.to_quadratic_tet(nodes, tets)
    return nodes, tets


def problem(nodes, conn, young=E, nu=NU, fixed=None, imposed=None, loads=None, pressures=None,
            name=""):
    n3 = 3 * nodes.shape[0]
    pe = np.array([p[0] for p in pressures or []], np.int64)
    pf = np.array([p[1] for p in pressures or []], np.int32)
    pv = np.array([p[2] for p in pressures or []], np.float64)
    return Problem(coords=nodes, conn=conn, young=np.full(conn.shape[0], young),
                   poisson=np.full(conn.shape[0], nu),
                   fixed=np.zeros(n3, np.uint8) if fixed is None else fixed,
                   imposed=np.zeros(n3) if imposed is None else imposed,
                   loads=np.zeros(n3) if loads is None else loads, p_elem=pe, p_face=pf,
                   p_value=pv, name=name)


EPS = np.array([1e-3, -2e-3, 0.5e-3, 3e-3, -1e-3, 2e-3])  # Voigt xx, yy, zz, yz, xz, xy


def uniform_field(x):
    """u = eps . x for the engineering-shear Voigt strain EPS (tests/solid.rs:56-62)."""
    e = EPS
    return np.stack([e[0] * x[:, 0] + e[5] / 2 * x[:, 1] + e[4] / 2 * x[:, 2],
                     e[5] / 2 * x[:, 0] + e[1] * x[:, 1] + e[3] / 2 * x[:, 2],
                     e[4] / 2 * x[:, 0] + e[3] / 2 * x[:, 1] + e[2] * x[:, 2]], axis=1)


def d_matrix(young=E, nu=NU):
    c = young / ((1 + nu) * (1 - 2 * nu))
    g = young / (2 * (1 + nu))
    d = np.zeros((6, 6))
    d[:3, :3] = c * nu
    for i in range(3):
        d[i, i] = c * (1 - nu)
        d[3 + i, 3 + i] = g
    return d


def patch(quadratic: bool) -> Problem:
    """Box 3x2x2 cells of 2 x 1 x 1.5, u = eps.x imposed on every boundary node."""
    size = (2.0, 1.0, 1.5)
    nodes, conn = box((3, 2, 2), size, quadratic)
    on = np.zeros(nodes.shape[0], bool)
    for c in range(3):
        on |= (np.abs(nodes[:, c]) < 1e-12) | (np.abs(nodes[:, c] - size[c]) < 1e-12)
    fixed = np.zeros(3 * nodes.shape[0], np.uint8)
    imposed = np.zeros(3 * nodes.shape[0])
    ex = uniform_field(nodes)
    for c in range(3):
        fixed[3 * np.nonzero(on)[0] + c] = 1
        imposed[3 * np.nonzero(on)[0] + c] = ex[on, c]
    return problem(nodes, conn, fixed=fixed, imposed=imposed, name=f"patch_q{int(quadratic)}")


def uniaxial(quadratic: bool, length=4.0, delta=0.01) -> Problem:
    """Bar L x 1 x 1 (4x1x1 cells), symmetry planes x, y, z = 0, u_x = delta on x = L."""
    nodes, conn = box((4, 1, 1), (length, 1.0, 1.0), quadratic)
    n = nodes.shape[0]
    fixed = np.zeros(3 * n, np.uint8)
    imposed = np.zeros(3 * n)
    for c in range(3):
        fixed[3 * np.nonzero(np.abs(nodes[:, c]) < 1e-12)[0] + c] = 1
    end = np.nonzero(np.abs(nodes[:, 0] - length) < 1e-12)[0]
    fixed[3 * end] = 1
    imposed[3 * end] = delta
    return problem(nodes, conn, fixed=fixed, imposed=imposed, name=f"uniaxial_q{int(quadratic)}")


def hydrostatic(quadratic: bool, p=50.0) -> Problem:
    """Unit cube 2x2x2 cells, sliding supports on x, y, z = 0, pressure p on x, y, z = 1."""
    nodes, conn = box((2, 2, 2), (1.0, 1.0, 1.0), quadratic)
    n = nodes.shape[0]
    tol = 1e-9 * p / E
    fixed = np.zeros(3 * n, np.uint8)
    for c in range(3):
        fixed[3 * np.nonzero(nodes[:, c] < tol)[0] + c] = 1
    pressures = []
    for c in range(3):
        e, f = mg.faces_on(nodes, conn, c, 1.0, tol)
        pressures += [(int(a), int(b), p) for a, b in zip(e, f)]
    return problem(nodes, conn, fixed=fixed, pressures=pressures, name=f"hydro_q{int(quadratic)}")


# vertices of the tet faces and the mid-edge nodes on them (tests/solid.rs:195-200)
_FACES = [([0, 1, 2], [4, 5, 6]), ([0, 1, 3], [4, 8, 7]), ([1, 2, 3], [5, 9, 8]),
          ([0, 2, 3], [6, 9, 7])]


def cantilever(n, quadratic: bool, L=10.0, B=1.0, H=1.0, P=1.0):
    """Cantilever L x B x H clamped at x = 0, P along z spread on the x = L section by consistent
    nodal forces (A/3 per vertex for Tet4, per mid-edge node for Tet10). Returns (problem, tip
    node at the centre of the end section)."""
    nodes, conn = box(n, (L, B, H), quadratic)
    at_tip = np.abs(nodes[:, 0] - L) < 1e-12
    loads = np.zeros(3 * nodes.shape[0])
    for e in range(conn.shape[0]):
        for verts, mids in _FACES:
            if not all(at_tip[conn[e, v]] for v in verts):
                continue
            p = nodes[conn[e, verts]]
            area = abs((p[1, 1] - p[0, 1]) * (p[2, 2] - p[0, 2])
                       - (p[1, 2] - p[0, 2]) * (p[2, 1] - p[0, 1])) / 2.0
            share = P * area / (B * H) / 3.0
            for k in (mids if quadratic else verts):
                loads[3 * conn[e, k] + 2] += share
    fixed = np.zeros(3 * nodes.shape[0], np.uint8)
    for c in range(3):
        fixed[3 * np.nonzero(np.abs(nodes[:, 0]) < 1e-12)[0] + c] = 1
    tip = int(np.nonzero(at_tip & (np.abs(nodes[:, 1] - B / 2) < 1e-12)
                         & (np.abs(nodes[:, 2] - H / 2) < 1e-12))[0][0])
    return problem(nodes, conn, fixed=fixed, loads=loads, name=f"cantilever_{n}"), tip


def timoshenko(L=10.0, B=1.0, H=1.0, P=1.0):
    """PL^3/3EI + PL/(kappa G A), kappa = 5/6 (tests/solid.rs:181-184)."""
    i, a, g = B * H ** 3 / 12, B * H, E / (2 * (1 + NU))
    return P * L ** 3 / (3 * E * i) + P * L / (5 / 6 * g * a)


def iterative_cantilever() -> Problem:
    """Tet10 10x2x2 cantilever 10 x 1 x 1, clamped x = 0, Uz = 1 on every node of x = 10
    (tests/iterative.rs:45-66)."""
    nodes, conn = box((10, 2, 2), (10.0, 1.0, 1.0), True)
    fixed = np.zeros(3 * nodes.shape[0], np.uint8)
    for c in range(3):
        fixed[3 * np.nonzero(np.abs(nodes[:, 0]) < 1e-12)[0] + c] = 1
    loads = np.zeros(3 * nodes.shape[0])
    loads[3 * np.nonzero(np.abs(nodes[:, 0] - 10.0) < 1e-12)[0] + 2] = 1.0
    return problem(nodes, conn, fixed=fixed, loads=loads, name="iterative_cantilever")


def unconstrained() -> Problem:
    """Tet10 4x1x1 bar without supports, Uz = 1 on node 0 (tests/iterative.rs:199-224)."""
    nodes, conn = box((4, 1, 1), (4.0, 1.0, 1.0), True)
    loads = np.zeros(3 * nodes.shape[0])
    loads[2] = 1.0
    return problem(nodes, conn, loads=loads, name="unconstrained")


def cube_example() -> Problem:
    d = json.load(open(os.path.join(GOLDEN, "cube_example.json")))
    nodes = np.array(d["coords"], np.float64)
    conn = np.array(d["conn"], np.int64)
    n3 = 3 * nodes.shape[0]
    fixed = np.zeros(n3, np.uint8)
    imposed = np.zeros(n3)
    for v, dof, value in d["bcs"]:  # later Bcs overwrite earlier ones (model.rs:1138-1142)
        fixed[3 * v + dof] = 1
        imposed[3 * v + dof] = value
    return problem(nodes, conn, young=d["young"], nu=d["poisson"], fixed=fixed, imposed=imposed,
                   name="cube_example")


def grid_laplacian_elements(n):
    """Quads of the n x n grid of iterative.rs:256-283 (vertex id i + n j)."""
    idx = lambda i, j: i + n * j  # noqa: E731
    return [[idx(i, j), idx(i + 1, j), idx(i + 1, j + 1), idx(i, j + 1)]
            for j in range(n - 1) for i in range(n - 1)]


def nearly_incompressible(cells, quadratic: bool, nu: float, size=(1.0, 1.0, 1.0)) -> Problem:
    """A box clamped on z = 0 under one downward point load at its highest node, every element
    with Poisson ratio `nu` close to 1/2. IC(0) of such a matrix meets a pivot <= 1e-12 a_ii
    (iterative.rs:160-163) at shift 0 and at the first shifts of the ladder, and succeeds later:
    Tet10 2^3 at nu = 0.49 needs shift 0.1 under RCM (1 under multicolouring); Tet4 4^3 at
    nu = 0.4999 needs 0.1 under every ordering tried (scalar and node RCM, multicolour, natural)."""
    nodes, conn = box(cells, size, quadratic)
    n = nodes.shape[0]
    fixed = np.zeros(3 * n, np.uint8)
    bottom = np.nonzero(np.abs(nodes[:, 2]) < 1e-12)[0]
    for c in range(3):
        fixed[3 * bottom + c] = 1
    loads = np.zeros(3 * n)
    loads[3 * int(np.argmax(nodes[:, 2])) + 2] = -1.0
    return problem(nodes, conn, nu=nu, fixed=fixed, loads=loads, name=f"incompressible_{nu}")


def two_blocks(cells=3, quadratic=False) -> Problem:
    """Two separate clamped cubes in one model (two connected components of the node graph), a
    pressure of 10 on the top of each: the orderings treat one component after the other."""
    p = mg.clamped_cube((cells,) * 3, quadratic, E)
    q = mg.clamped_cube((cells + 1, cells, cells), quadratic, 2 * E, size=(1.5, 1.0, 1.0))
    n = p.coords.shape[0]
    coords = np.concatenate([p.coords, q.coords + np.array([3.0, 0.0, 0.0])])
    conn = np.concatenate([p.conn, q.conn + n])
    return Problem(coords=coords, conn=conn, young=np.concatenate([p.young, q.young]),
                   poisson=np.concatenate([p.poisson, q.poisson]), fixed=np.concatenate([p.fixed, q.fixed]),
                   imposed=np.zeros(3 * coords.shape[0]), loads=np.zeros(3 * coords.shape[0]),
                   p_elem=np.concatenate([p.p_elem, q.p_elem + p.conn.shape[0]]),
                   p_face=np.concatenate([p.p_face, q.p_face]),
                   p_value=np.concatenate([p.p_value, q.p_value]), name="two_blocks")
