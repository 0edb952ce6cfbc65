"""Synthetic structured tetrahedral meshes and the benchmark workloads built on them.

`box_grid` and `to_quadratic_tet` restate the reference's bench/test mesh helpers
(crates/maille-core/benches/common/mod.rs:13-53 and 80-104): nx*ny*nz hexahedral cells, each cut
into the 6 Kuhn tetrahedra (the 6 axis paths from (0,0,0) to (1,1,1)), oriented like `Tet4`
(positive signed volume); Tet10 mid-edge nodes are appended in first-encounter order (element
order, then edge order of `TET10_EDGES`, shape.rs:135), which is the order the reference's
HashMap-based helper gives them. Both are vectorised with numpy so the 40^3 Tet10 mesh
(531 441 nodes) builds in about a second.

The random inputs of the workloads (per-element Young's moduli, batched mesh sizes and load
cases) come from a counter-based SplitMix64 stream so that any element's value can be
regenerated without replaying a sequence.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# shape.rs:129 and shape.rs:135
TET_FACES = np.array([[0, 1, 2], [0, 3, 1], [1, 3, 2], [2, 3, 0]], dtype=np.int64)
TET10_EDGES = np.array([[0, 1], [1, 2], [2, 0], [0, 3], [1, 3], [2, 3]], dtype=np.int64)

# benches/common/mod.rs:24-31
_PERMUTATIONS = np.array([[0, 1, 2], [0, 2, 1], [1, 0, 2], [1, 2, 0], [2, 0, 1], [2, 1, 0]])

SEED = 0x6D61696C6C65  # "maille"
_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 output function (Steele, Lea, Flood 2014) on uint64 arrays."""
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform(stream: int, count: int, offset: int = 0, seed: int = SEED) -> np.ndarray:
    """`count` uniforms in [0, 1) from counter-based stream `stream` (53-bit mantissas)."""
    k = np.arange(offset, offset + count, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = (np.uint64(seed) + np.uint64(stream) * np.uint64(0xD1B54A32D192ED03)
             + k * np.uint64(0x9E3779B97F4A7C15))
    return (_splitmix64(x) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normal(stream: int, count: int, seed: int = SEED) -> np.ndarray:
    """Standard normals by Box-Muller in FP64 from pairs of `uniform` draws."""
    u = uniform(stream, 2 * count, seed=seed)
    u1 = 1.0 - u[0::2]  # (0, 1]
    u2 = u[1::2]
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def _signed_volume6(nodes: np.ndarray, tets: np.ndarray) -> np.ndarray:
    """6 x signed volume, benches/common/mod.rs:55-63 (same expression and order)."""
    p0 = nodes[tets[:, 0]]
    a = nodes[tets[:, 1]] - p0
    b = nodes[tets[:, 2]] - p0
    c = nodes[tets[:, 3]] - p0
    return (a[:, 0] * (b[:, 1] * c[:, 2] - b[:, 2] * c[:, 1])
            - a[:, 1] * (b[:, 0] * c[:, 2] - b[:, 2] * c[:, 0])
            + a[:, 2] * (b[:, 0] * c[:, 1] - b[:, 1] * c[:, 0]))


def box_grid(n, size):
    """Box size[0] x size[1] x size[2] of n[0] x n[1] x n[2] cells, 6 Kuhn tets per cell.

    Node (i, j, k) has index i + (nx + 1) (j + (ny + 1) k). Returns (nodes (N, 3) float64,
    tets (6 nx ny nz, 4) int64), cells in k, j, i order and the 6 axis permutations in the
    order of benches/common/mod.rs:24-31.
    """
    nx, ny, nz = (int(v) for v in n)
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    at = lambda c, v: size[c] * v.astype(np.float64) / float(n[c])  # noqa: E731
    nodes = np.stack([at(0, i.ravel()), at(1, j.ravel()), at(2, k.ravel())], axis=1)

    def idx(p):
        return p[..., 0] + (nx + 1) * (p[..., 1] + (ny + 1) * p[..., 2])

    ck, cj, ci = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    base = np.stack([ci.ravel(), cj.ravel(), ck.ravel()], axis=1)  # (cells, 3) as (i, j, k)
    cells = base.shape[0]
    tets = np.empty((cells, 6, 4), dtype=np.int64)
    for t, axes in enumerate(_PERMUTATIONS):
        p = base.copy()
        tets[:, t, 0] = idx(p)
        for v, axis in enumerate(axes):
            p[:, axis] += 1
            tets[:, t, v + 1] = idx(p)
    tets = tets.reshape(-1, 4)
    flip = _signed_volume6(nodes, tets) < 0.0
    tets[flip, 1], tets[flip, 2] = tets[flip, 2].copy(), tets[flip, 1].copy()
    return nodes, tets


def to_quadratic_tet(nodes: np.ndarray, tets: np.ndarray):
    """Tet10 mesh with one node in the middle of every edge, shared between neighbours.

    Mid nodes get indices in first-encounter order over (element, edge), as the reference's
    HashMap helper assigns them (benches/common/mod.rs:80-104).
    """
    a = tets[:, TET10_EDGES[:, 0]]
    b = tets[:, TET10_EDGES[:, 1]]
    lo = np.minimum(a, b).ravel()
    hi = np.maximum(a, b).ravel()
    key = lo * np.int64(nodes.shape[0]) + hi
    uniq, first, inverse = np.unique(key, return_index=True, return_inverse=True)
    by_first = np.argsort(first, kind="stable")
    new_id = np.empty(uniq.shape[0], dtype=np.int64)
    new_id[by_first] = np.arange(uniq.shape[0], dtype=np.int64) + nodes.shape[0]
    mids = new_id[inverse].reshape(-1, 6)
    order_lo = lo[first[by_first]]
    order_hi = hi[first[by_first]]
    mid_coords = (nodes[order_lo] + nodes[order_hi]) / 2.0
    return np.concatenate([nodes, mid_coords]), np.concatenate([tets, mids], axis=1)


def faces_on(nodes: np.ndarray, conn: np.ndarray, axis: int, value: float, tol: float = 1e-12):
    """(element, face) pairs whose three vertices lie on the plane x[axis] = value."""
    verts = conn[:, :4]
    on = np.abs(nodes[verts, axis] - value) < tol  # (E, 4)
    hits = np.stack([on[:, f].all(axis=1) for f in TET_FACES], axis=1)  # (E, 4 faces)
    e, f = np.nonzero(hits)
    return e.astype(np.int64), f.astype(np.int32)


@dataclass
class Problem:
    """A linear static solid problem in the layout of the C ABI (include/maille_gpu.h)."""
    coords: np.ndarray                   # (N, 3) float64
    conn: np.ndarray                     # (E, npe) int64
    young: np.ndarray                    # (E,) float64
    poisson: np.ndarray                  # (E,) float64
    fixed: np.ndarray                    # (3N,) uint8
    imposed: np.ndarray                  # (3N,) float64
    loads: np.ndarray                    # (3N,) float64 nodal loads
    p_elem: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    p_face: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    p_value: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float64))
    name: str = ""

    @property
    def npe(self) -> int:
        return int(self.conn.shape[1])

    @property
    def n_nodes(self) -> int:
        return int(self.coords.shape[0])

    @property
    def n_elems(self) -> int:
        return int(self.conn.shape[0])

    @property
    def free_dofs(self) -> int:
        return int(self.fixed.size - np.count_nonzero(self.fixed))


def clamped_cube(cells, quadratic: bool, young, poisson: float = 0.3, pressure: float = 10.0,
                 size=(1.0, 1.0, 1.0), name: str = "") -> Problem:
    """Box mesh, all DOFs fixed on z = 0, uniform pressure on every tet face lying on z = size_z.

    `young` is a scalar or a per-element array.
    """
    nodes, tets = box_grid(cells, size)
    conn = tets
    if quadratic:
        nodes, conn = to_quadratic_tet(nodes, tets)
    n = nodes.shape[0]
    fixed = np.zeros(3 * n, np.uint8)
    bottom = np.nonzero(np.abs(nodes[:, 2]) < 1e-12)[0]
    for c in range(3):
        fixed[3 * bottom + c] = 1
    pe, pf = faces_on(nodes, conn, 2, size[2])
    e_arr = np.broadcast_to(np.asarray(young, np.float64), (conn.shape[0],)).copy()
    return Problem(coords=nodes, conn=conn, young=e_arr,
                   poisson=np.full(conn.shape[0], poisson), fixed=fixed,
                   imposed=np.zeros(3 * n), loads=np.zeros(3 * n), p_elem=pe, p_face=pf,
                   p_value=np.full(pe.shape[0], pressure), name=name)


# --- the five benchmark configurations -----------------------------------------------------------

def plain_tet4(cells: int = 20) -> Problem:
    """Plain FP64 Tet4: unit cube, cells^3 x 6 tets, E = 210000, nu = 0.3, z = 0 clamped,
    10 MPa pressure on z = 1 (20^3: 9 261 nodes, 48 000 tets, 26 460 free DOF)."""
    return clamped_cube((cells,) * 3, False, 210000.0, name=f"tet4_{cells}^3")


def mixed_tet10(cells: int = 40, sigma_log: float = 0.5) -> Problem:
    """Tet10 unit cube, cells^3 x 6 quadratic tets, per-element E lognormal (median 210000,
    sigma_log 0.5, seeded), nu = 0.3, z = 0 clamped, 10 MPa on z = 1 (40^3: 531 441 nodes,
    384 000 tets, 1 574 640 free DOF)."""
    n_el = 6 * cells ** 3
    young = 210000.0 * np.exp(sigma_log * normal(stream=2, count=n_el))
    return clamped_cube((cells,) * 3, True, young, name=f"tet10_{cells}^3_lognormal")


def simp_tet4(cells: int = 48):
    """Adjoint compliance Tet4: cells^3 cube, rho_e uniform in [0.01, 1] (seeded),
    E_e = 210000 rho_e^3, nu = 0.3, z = 0 clamped, 10 MPa on z = 1. Returns (problem, rho)."""
    n_el = 6 * cells ** 3
    rho = 0.01 + 0.99 * uniform(stream=4, count=n_el)
    prob = clamped_cube((cells,) * 3, False, 210000.0 * rho ** 3, name=f"simp_tet4_{cells}^3")
    return prob, rho


def batched_tet4(count: int = 256, lo: int = 6, hi: int = 24, load_cases: int = 8):
    """Batched Tet4: `count` unit cubes of side m ~ U{lo..hi} cells (seeded), E_e ~ U[50000,
    250000], nu = 0.3, z = 0 clamped, `load_cases` traction loads on z = 1 per mesh (direction
    uniform on the sphere, magnitude U[1, 20]). Returns (list of Problem, list of (3N, L) RHS)."""
    sides = lo + np.floor(uniform(stream=3, count=count) * (hi - lo + 1)).astype(np.int64)
    problems, rhs = [], []
    for b, m in enumerate(sides):
        m = int(m)
        n_el = 6 * m ** 3
        young = 50000.0 + 200000.0 * uniform(stream=1000 + b, count=n_el)
        prob = clamped_cube((m, m, m), False, young, pressure=0.0, name=f"batch{b}_{m}^3")
        prob.p_elem = np.zeros(0, np.int64)
        prob.p_face = np.zeros(0, np.int32)
        prob.p_value = np.zeros(0)
        u = uniform(stream=5000 + b, count=3 * load_cases).reshape(load_cases, 3)
        cos_t = 2.0 * u[:, 0] - 1.0
        phi = 2.0 * np.pi * u[:, 1]
        sin_t = np.sqrt(np.maximum(0.0, 1.0 - cos_t * cos_t))
        direction = np.stack([sin_t * np.cos(phi), sin_t * np.sin(phi), cos_t], axis=1)
        traction = direction * (1.0 + 19.0 * u[:, 2])[:, None]
        rhs.append(traction_loads(prob, 2, 1.0, traction))
        problems.append(prob)
    return problems, rhs


def large_strain_block(cells=(64, 16, 16), size=(4.0, 1.0, 1.0), tip: float = -0.4,
                       lam: float = 120000.0, mu_range=(60000.0, 100000.0)):
    """Large-strain neo-Hookean Tet4 block (size mm, cells x 6 tets): mu_e uniform in mu_range
    (seeded), lambda fixed, converted per element to E = mu (3 lambda + 2 mu) / (lambda + mu) and
    nu = lambda / (2 (lambda + mu)) (Material takes E and nu; lame() gives mu and lambda back).
    The x = 0 face is clamped; every node of the x = size_x face has its z displacement imposed
    to `tip` (reached at the end of the ramp). Returns (Problem, mu, tip z-DOFs)."""
    nodes, tets = box_grid(cells, size)
    n_el = tets.shape[0]
    mu = mu_range[0] + (mu_range[1] - mu_range[0]) * uniform(stream=6, count=n_el)
    young = mu * (3.0 * lam + 2.0 * mu) / (lam + mu)
    poisson = lam / (2.0 * (lam + mu))
    n = nodes.shape[0]
    fixed = np.zeros(3 * n, np.uint8)
    imposed = np.zeros(3 * n)
    root = np.nonzero(np.abs(nodes[:, 0]) < 1e-12)[0]
    for c in range(3):
        fixed[3 * root + c] = 1
    end = np.nonzero(np.abs(nodes[:, 0] - size[0]) < 1e-12)[0]
    fixed[3 * end + 2] = 1
    imposed[3 * end + 2] = tip
    prob = Problem(coords=nodes, conn=tets, young=young, poisson=poisson, fixed=fixed,
                   imposed=imposed, loads=np.zeros(3 * n),
                   name=f"neo_hookean_tet4_{cells[0]}x{cells[1]}x{cells[2]}")
    return prob, mu, 3 * end + 2


def traction_loads(prob: Problem, axis: int, value: float, traction: np.ndarray) -> np.ndarray:
    """Nodal loads of constant tractions t (L, 3) on the mesh faces lying on x[axis] = value:
    f_a = t * integral of N_a over the face (linear faces: area / 3 per vertex). Returns (3N, L)."""
    if prob.npe != 4:
        raise ValueError("traction_loads handles Tet4 faces")
    e, f = faces_on(prob.coords, prob.conn, axis, value)
    tri = prob.conn[e][np.arange(e.size)[:, None], TET_FACES[f]]  # (F, 3) node ids
    p = prob.coords[tri]
    area = 0.5 * np.linalg.norm(np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), axis=1)
    share = np.zeros(prob.n_nodes)
    np.add.at(share, tri.ravel(), np.repeat(area / 3.0, 3))
    out = np.zeros((3 * prob.n_nodes, traction.shape[0]))
    for c in range(3):
        out[c::3, :] = share[:, None] * traction[None, :, c]
    return out


# --- transient heat conduction -------------------------------------------------------------------

@dataclass
class ThermalProblem:
    """A transient thermal Tet4/Tet10 problem (Model with Analysis::Thermal and a transient Step,
    model.rs:621-706) in the layout of the C ABI's MailleThermalProblem."""
    coords: np.ndarray                   # (N, 3) float64
    conn: np.ndarray                     # (E, npe) int64
    conductivity: np.ndarray             # (E,) k
    rho_c: np.ndarray                    # (E,) density x specific heat
    fixed: np.ndarray                    # (N,) uint8 imposed temperature
    imposed: np.ndarray                  # (N,) float64
    loads: np.ndarray                    # (N,) float64 nodal heat loads
    initial: np.ndarray                  # (N,) float64 temperature at t = 0
    time_period: float = 1.0
    increments: int = 1
    theta: float = 1.0
    s_elem: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    s_value: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float64))
    c_elem: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    c_face: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    c_film: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float64))
    c_sink: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float64))
    name: str = ""

    @property
    def time_step(self) -> float:
        """Step::time_step (model.rs:171-173)."""
        return self.time_period / self.increments

    @property
    def npe(self) -> int:
        return int(self.conn.shape[1])

    @property
    def n_nodes(self) -> int:
        return int(self.coords.shape[0])

    @property
    def n_elems(self) -> int:
        return int(self.conn.shape[0])

    @property
    def free_nodes(self) -> int:
        return int(self.fixed.size - np.count_nonzero(self.fixed))


def thermal_cube(cells: int = 40, quadratic: bool = True, increments: int = 10,
                 time_period: float = 0.1, theta: float = 1.0) -> ThermalProblem:
    """Unit cube heated from below and cooled on top: cells^3 x 6 tets (Tet10 when `quadratic`),
    per-element conductivity lognormal (median 1, sigma_log 0.5, seeded), rho_c = 1, T = 100
    imposed on z = 0, convection h = 10 to T_inf = 20 on every face of z = 1, a uniform source
    of 50 in every element, T = 20 at t = 0; `increments` backward-Euler steps (theta = 1) over
    `time_period`. 40^3 Tet10: 531 441 nodes, 384 000 tets, 524 800 free nodes."""
    nodes, tets = box_grid((cells,) * 3, (1.0, 1.0, 1.0))
    conn = tets
    if quadratic:
        nodes, conn = to_quadratic_tet(nodes, tets)
    n, ne = nodes.shape[0], conn.shape[0]
    fixed = (np.abs(nodes[:, 2]) < 1e-12).astype(np.uint8)
    imposed = np.where(fixed != 0, 100.0, 0.0)
    ce, cf = faces_on(nodes, conn, 2, 1.0)
    k = np.exp(0.5 * normal(stream=7, count=ne))
    return ThermalProblem(coords=nodes, conn=conn, conductivity=k, rho_c=np.ones(ne), fixed=fixed,
                          imposed=imposed, loads=np.zeros(n), initial=np.full(n, 20.0),
                          time_period=time_period, increments=increments, theta=theta,
                          s_elem=np.arange(ne, dtype=np.int64), s_value=np.full(ne, 50.0),
                          c_elem=ce, c_face=cf, c_film=np.full(ce.shape[0], 10.0),
                          c_sink=np.full(ce.shape[0], 20.0),
                          name=f"{'tet10' if quadratic else 'tet4'}_{cells}^3_transient")
