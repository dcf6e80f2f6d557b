"""Shared pytest set-up: import paths, the `gpu` marker, golden fixtures."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "sgn-hyperbolic-gpu_b200"), os.path.join(ROOT, "oracle"),
          os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libsgnb.so")


@pytest.fixture(scope="session")
def golden():
    return np.load(os.path.join(ROOT, "tests", "golden", "golden.npz"))


@pytest.fixture(scope="session")
def need_reference():
    import oracle as O

    if not O.reference_available():
        pytest.skip("oracle/_ref/libsgnref.so not built (reference sources absent)")
    return True


def bits_equal(a, b) -> bool:
    """Bit-for-bit equality of two float64 arrays (signed zeros and NaN payloads too)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def rel_per_field(a, b, n_fields=5):
    """max_v max|a_v - b_v| / max|b_v|: relative error per field, normalised by the field's
    largest magnitude (fields with max 0 use absolute error)."""
    a = a.reshape(n_fields, -1)
    b = b.reshape(n_fields, -1)
    out = []
    for v in range(n_fields):
        s = np.abs(b[v]).max()
        out.append(np.abs(a[v] - b[v]).max() / (s if s > 0 else 1.0))
    return max(out)
