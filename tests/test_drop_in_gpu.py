"""The reference's own host solver driving libsgnb through include/sgnb.hpp (C++).

tests/cpp/drop_in.cpp is compiled against the reference sources where they are present
(oracle/_ref/drop_in); it swaps sgn::SGN2DCuda for sgnb::SGN2DB200 and checks rhs parity
bit for bit, lake at rest and an adaptive run against sgn::SGN2D / sgn::integrateAdaptive.
"""
from __future__ import annotations

import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "oracle", "_ref", "drop_in")


def test_reference_caller_drop_in():
    if not os.path.exists(BIN):
        pytest.skip("oracle/_ref/drop_in not built (reference sources absent at build time)")
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL PASSED" in r.stdout
