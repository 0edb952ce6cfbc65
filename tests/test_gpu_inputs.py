"""The create path reads the caller's buffers as they are: absent loads or imposed values, and
imposed values at free DOFs (which the model ignores), must give the same solve as explicit zeros.
The connectivity is narrowed and the node incidence built on the device, so these solves also
exercise the reactions and stresses that depend on them."""
import ctypes

import numpy as np
import pytest

from maille_b200 import meshgen as mg
from maille_b200._lib import MAILLE_FP64, ElasticResult, ptr, _d
from maille_b200.model import problem_struct, face_pressure_loads

pytestmark = pytest.mark.gpu


def one_shot(L, p, imposed, f):
    prob, keep = problem_struct(p.coords, p.conn.astype(np.int64), p.young, p.poisson, p.fixed, imposed, f,
                                1e-12, 10000, MAILLE_FP64, 0, 0)
    if imposed is None:
        prob.imposed = None
    out = dict(u=np.zeros(3 * p.n_nodes), r=np.zeros(3 * p.n_nodes), g=np.zeros(p.n_elems * 9),
               vm=np.zeros(p.n_elems))
    res = ElasticResult(u=ptr(out["u"], _d), reactions=ptr(out["r"], _d), gauss_stress=ptr(out["g"], _d),
                        von_mises=ptr(out["vm"], _d))
    s = L.maille_gpu_elastic_solve(ctypes.byref(prob), ctypes.byref(res))
    assert s == 0, L.maille_gpu_last_error().decode()
    return out


def cube():
    p = mg.plain_tet4(6)
    return p, face_pressure_loads(p.coords, p.conn, list(zip(p.p_elem, p.p_face, p.p_value)))


def test_absent_imposed_values_equal_zeros(gpu):
    p, f = cube()
    a = one_shot(gpu, p, None, f)
    b = one_shot(gpu, p, np.zeros(3 * p.n_nodes), f)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert np.abs(a["u"]).max() > 0


def test_absent_loads_equal_zeros_under_imposed_displacements(gpu):
    p, _ = cube()
    imposed = np.zeros(3 * p.n_nodes)
    top = np.nonzero(p.coords[:, 2] == p.coords[:, 2].max())[0]
    fixed = p.fixed.copy().reshape(-1, 3)
    fixed[top, 2] = 1
    p.fixed = fixed.ravel()
    imposed[3 * top + 2] = -1e-3
    a = one_shot(gpu, p, imposed, None)
    b = one_shot(gpu, p, imposed, np.zeros(3 * p.n_nodes))
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert np.abs(a["u"][3 * top + 2] + 1e-3).max() == 0.0
    # the imposed shortening is held by reactions that balance
    assert abs(a["r"][2::3].sum()) < 1e-9 * np.abs(a["r"]).max()


def test_imposed_values_at_free_dofs_are_ignored(gpu):
    p, f = cube()
    junk = np.where(p.fixed.astype(bool), 0.0, np.nan)
    a = one_shot(gpu, p, junk, f)
    b = one_shot(gpu, p, np.zeros(3 * p.n_nodes), f)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
