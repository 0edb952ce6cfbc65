"""The entry point that allocates no device memory (maille_gpu_bsr3_spmv_dot_noalloc).

It serves callers that cannot allocate device memory where they need the product (stream
capture, plugins whose host owns every allocation, real-time loops): they pass a 3x3-block CSR
matrix and vectors that already live on the device. Here the test owns those buffers (torch
allocates them, the library does not), fills them with the assembled stiffness of a small mesh,
and checks y = K x and x . y against the existing entry point maille_gpu_multiply on two calls
in a row. A second case, about 20 000 block rows of a random block-banded matrix built here in
numpy (with some rows longer than a warp), reaches the capped grid (1024 blocks, several rows
per warp) and is checked against numpy's own product, independently of the library. The file
is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

import maille_b200 as mb
from maille_b200 import _lib, meshgen as mg

pytestmark = pytest.mark.gpu


def _handle_for(p):
    m = mb.Model.from_arrays(p.coords, p.conn, p.young, p.poisson, p.fixed, p.imposed, p.loads,
                             (p.p_elem, p.p_face, p.p_value))
    m.with_solver(mb.SolverKind.ITERATIVE)
    return mb.SolverHandle(m)


def _multiply(h, x):
    y = np.zeros_like(x)
    s = h._L.maille_gpu_multiply(h._h, _lib.ptr(x, _lib._d), _lib.ptr(y, _lib._d))
    assert s == 0, _lib.last_error()
    return y


def _block_csr(h, n_nodes):
    """K (free DOFs, 0 at fixed DOFs) probed column by column through maille_gpu_multiply, as a
    3x3-block CSR over all nodes."""
    n = 3 * n_nodes
    k = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        k[:, j] = _multiply(h, e)
    blocks = k.reshape(n_nodes, 3, n_nodes, 3).transpose(0, 2, 1, 3)
    nz = np.abs(blocks).sum(axis=(2, 3)) > 0
    row_ptr = np.zeros(n_nodes + 1, np.int64)
    row_ptr[1:] = np.cumsum(nz.sum(axis=1))
    rows, cols = np.nonzero(nz)
    vals = blocks[rows, cols].reshape(-1, 9)
    return row_ptr, cols.astype(np.int32), np.ascontiguousarray(vals)


def test_no_alloc_spmv_dot_matches_the_allocating_entry_point(gpu):
    import torch
    p = mg.plain_tet4(3)
    p.fixed[3 * 5] = 1  # one partially fixed node, so K has identity-free zero rows too
    h = _handle_for(p)
    try:
        row_ptr, col, vals = _block_csr(h, p.n_nodes)
        dev = torch.device("cuda", 0)
        t_row = torch.from_numpy(row_ptr).to(dev)
        t_col = torch.from_numpy(col).to(dev)
        t_val = torch.from_numpy(vals.ravel()).to(dev)
        t_y = torch.empty(3 * p.n_nodes, dtype=torch.float64, device=dev)
        t_xy = torch.empty(1, dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        rng = np.random.default_rng(7)
        for call in range(2):
            x = rng.standard_normal(3 * p.n_nodes)
            t_x = torch.from_numpy(x).to(dev)
            torch.cuda.synchronize()
            s = h._L.maille_gpu_bsr3_spmv_dot_noalloc(
                0, p.n_nodes, t_row.data_ptr(), t_col.data_ptr(), t_val.data_ptr(),
                t_x.data_ptr(), t_y.data_ptr(), t_xy.data_ptr(), stream)
            assert s == 0, _lib.last_error()
            torch.cuda.synchronize()
            y_ref = _multiply(h, x)
            y = t_y.cpu().numpy()
            assert np.linalg.norm(y - y_ref) <= 1e-12 * np.linalg.norm(y_ref), call
            xy_ref = float(x @ y_ref)
            assert abs(float(t_xy.cpu()[0]) - xy_ref) <= 1e-12 * abs(x) @ np.abs(y_ref), call
        # sizes beyond the stated maximum are refused with a message, before any device work
        s = h._L.maille_gpu_bsr3_spmv_dot_noalloc(
            0, _lib.MAILLE_NOALLOC_MAX_BLOCK_ROWS + 1, t_row.data_ptr(), t_col.data_ptr(),
            t_val.data_ptr(), t_y.data_ptr(), t_y.data_ptr(), t_xy.data_ptr(), stream)
        assert s == _lib.MAILLE_INVALID_INPUT and "MAILLE_NOALLOC_MAX_BLOCK_ROWS" in _lib.last_error()
    finally:
        h.close()


def _banded_bsr(nb, rng):
    """A random 3x3-block CSR matrix: each block row holds its diagonal, up to 6 random
    neighbours within 40 block columns, and every 997th row 70 blocks (longer than a warp)."""
    rows = []
    for i in range(nb):
        width = 70 if i % 997 == 0 else int(rng.integers(0, 7))
        lo, hi = max(0, i - 40), min(nb, i + 41)
        nbrs = rng.choice(np.arange(lo, hi), size=min(width, hi - lo), replace=False)
        rows.append(np.unique(np.concatenate([[i], nbrs])))
    row_ptr = np.zeros(nb + 1, np.int64)
    row_ptr[1:] = np.cumsum([len(r) for r in rows])
    col = np.concatenate(rows).astype(np.int32)
    vals = rng.standard_normal((col.size, 9))
    return row_ptr, col, vals


def _numpy_product(row_ptr, col, vals, x):
    nb = row_ptr.size - 1
    row_of = np.repeat(np.arange(nb), np.diff(row_ptr))
    contrib = np.einsum("kab,kb->ka", vals.reshape(-1, 3, 3), x.reshape(-1, 3)[col])
    y = np.zeros((nb, 3))
    np.add.at(y, row_of, contrib)
    return y.ravel()


def test_no_alloc_spmv_dot_on_a_large_matrix_matches_numpy(gpu):
    import torch
    rng = np.random.default_rng(11)
    nb = 20000  # > 8192 block rows: the grid is capped at 1024 blocks, warps take several rows
    row_ptr, col, vals = _banded_bsr(nb, rng)
    L = _lib.load()
    dev = torch.device("cuda", 0)
    t_row = torch.from_numpy(row_ptr).to(dev)
    t_col = torch.from_numpy(col).to(dev)
    t_val = torch.from_numpy(np.ascontiguousarray(vals.ravel())).to(dev)
    t_y = torch.empty(3 * nb, dtype=torch.float64, device=dev)
    t_xy = torch.empty(1, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        x = rng.standard_normal(3 * nb)
        t_x = torch.from_numpy(x).to(dev)
        torch.cuda.synchronize()
        s = L.maille_gpu_bsr3_spmv_dot_noalloc(0, nb, t_row.data_ptr(), t_col.data_ptr(), t_val.data_ptr(),
                                               t_x.data_ptr(), t_y.data_ptr(), t_xy.data_ptr(), stream)
        assert s == 0, _lib.last_error()
        torch.cuda.synchronize()
        y_ref = _numpy_product(row_ptr, col, vals, x)
        y = t_y.cpu().numpy()
        assert np.linalg.norm(y - y_ref) <= 1e-12 * np.linalg.norm(y_ref), call
        assert abs(float(t_xy.cpu()[0]) - float(x @ y_ref)) <= 1e-12 * (np.abs(x) @ np.abs(y_ref)), call
    # an in-place product (x and y the same buffer) is refused before any device work
    s = L.maille_gpu_bsr3_spmv_dot_noalloc(0, nb, t_row.data_ptr(), t_col.data_ptr(), t_val.data_ptr(),
                                           t_y.data_ptr(), t_y.data_ptr(), t_xy.data_ptr(), stream)
    assert s == _lib.MAILLE_INVALID_INPUT and "overlap" in _lib.last_error()
