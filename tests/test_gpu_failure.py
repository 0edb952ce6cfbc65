"""Failure detection on the GPU without a fault: the IC(0) sweeps' bounded wait gives up and reports.

A sweep lane waits for the records of the rows it depends on; a record that never reaches the
awaited epoch (a flag that nothing sets) must end the wait after its round limit with a status the
host reads, leaving the context usable. maille_gpu_wait_selftest runs that wait on one stale record
with a short limit (4096 rounds).
"""
import ctypes

import numpy as np
import pytest

import maille_b200 as mb
from maille_b200 import _lib
from maille_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def selftest(L, stale):
    t = ctypes.c_int32(-1)
    assert L.maille_gpu_wait_selftest(0, stale, ctypes.byref(t)) == _lib.MAILLE_OK, _lib.last_error()
    return t.value


def test_a_wait_on_a_record_nothing_writes_times_out_and_the_context_stays_usable(gpu):
    L = _lib.load()
    assert selftest(L, 1) == 1   # the stale record: the wait ran out and said so
    assert selftest(L, 0) == 0   # every record current: no timeout
    # the device is still usable afterwards: a small solve runs and converges
    p = mg.plain_tet4(4)
    m = mb.Model.from_arrays(p.coords, p.conn, p.young, p.poisson, p.fixed, p.imposed, p.loads,
                             (p.p_elem, p.p_face, p.p_value))
    m.with_solver(mb.SolverKind.ITERATIVE)
    f = m.solve()
    assert np.all(np.isfinite(f.displacements)) and f.info["iterations"] > 0
