"""The library's device memory pool (memory.cu): handles reuse the memory their predecessors
freed, and maille_gpu_trim_memory hands the unused part back without disturbing later solves."""
import numpy as np
import pytest
import torch

import maille_b200 as mb
from maille_b200 import _lib
from maille_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def solve_once(p):
    m = mb.Model.from_arrays(p.coords, p.conn, p.young, p.poisson, p.fixed, p.imposed, p.loads,
                             (p.p_elem, p.p_face, p.p_value))
    m.with_solver(mb.SolverKind.ITERATIVE).with_tolerance(1e-12)
    return m.solve()


def test_repeated_handles_reuse_the_pool_and_trim_returns_it(gpu):
    L = _lib.load()
    p = mg.mixed_tet10(6)
    first = solve_once(p).displacements
    free_after_first = torch.cuda.mem_get_info(0)[0]
    for _ in range(3):  # create / solve / destroy again: same result, no growth of reserved memory
        again = solve_once(p).displacements
        assert np.array_equal(again, first)
        assert torch.cuda.mem_get_info(0)[0] >= free_after_first - (64 << 20)
    assert L.maille_gpu_trim_memory(0) == _lib.MAILLE_OK, _lib.last_error()
    assert torch.cuda.mem_get_info(0)[0] >= free_after_first  # the pool's reserve went back
    assert np.array_equal(solve_once(p).displacements, first)  # and the pool refills on demand
