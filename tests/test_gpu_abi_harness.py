"""The C harness (tests/abi_harness.c) on a GPU: a Tet4 cube solved through the C ABI from C,
the elastic reactions balancing the applied load and the thermal step heating the cube from
its imposed face."""
import subprocess

import pytest

from test_abi import _build_harness

pytestmark = pytest.mark.gpu


def test_c_harness_solves_through_the_abi(gpu, tmp_path):
    exe = _build_harness(tmp_path)
    out = subprocess.run([str(exe), "6"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "elastic status 0" in out.stdout and "thermal status 0" in out.stdout
