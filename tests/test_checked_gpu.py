"""The range-checked build (libsgnb_checked.so, -DSGNB_CHECKED): every global access of the
fused FP64 and mixed-precision kernels is checked against its buffer and an out-of-range index is counted and
skipped instead of performed. tests/checked_run.py drives every kernel family on ragged
meshes in its own process (SGNB_LIBRARY=checked selects the library); the count must be
zero. The normal build answers SGNB_ERR_UNSUPPORTED to the count query."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import pytest

import sgnb
from conftest import ROOT

pytestmark = pytest.mark.gpu

CHECKED = os.path.join(ROOT, "sgn-hyperbolic-gpu_b200", "sgnb", "libsgnb_checked.so")


def test_no_out_of_range_access():
    if not os.path.exists(CHECKED):
        pytest.fail("libsgnb_checked.so not built (make -C sgn-hyperbolic-gpu_b200/csrc checked)")
    env = dict(os.environ, SGNB_LIBRARY="checked")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "checked_run.py")],
                       capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert r.stdout.strip().splitlines()[-1] == "oob 0", r.stdout[-2000:]


def test_normal_build_has_no_checks():
    n = C.c_longlong(-1)
    assert sgnb.lib().sgnb_checked_oob(0, C.byref(n), 0) == 2 and n.value == 0
