"""Shared pytest configuration: the `gpu` marker and repository paths."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a library)")


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def rel_max(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = float(np.abs(b).max())
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


# history columns (nova_gpu.h NOVA_HIST_COLS) and the tolerance each is
# checked to against the oracle: relative, except the divergence maxima
# (round-off level after the projection: absolute)
HIST_RTOL = {2: 1e-11, 3: 1e-11, 6: 1e-11, 7: 1e-11, 8: 1e-10, 9: 1e-11, 10: 1e-10, 11: 1e-10, 12: 1e-10,
             13: 1e-10, 14: 1e-11, 15: 1e-11}


def check_history(h_gpu, h_ref, divtol=1e-11, cols=None):
    """Overlay a GPU history on the oracle's, step by step and column by column:
    step exact, time to 1e-13, every diagnostic to HIST_RTOL (max|div| to divtol)."""
    h_gpu = np.asarray(h_gpu)
    h_ref = np.asarray(h_ref)
    assert h_gpu.shape == h_ref.shape, (h_gpu.shape, h_ref.shape)
    assert np.array_equal(h_gpu[:, 0], h_ref[:, 0])
    np.testing.assert_allclose(h_gpu[:, 1], h_ref[:, 1], rtol=1e-13)
    for c, rt in HIST_RTOL.items():
        if cols is not None and c not in cols:
            continue
        np.testing.assert_allclose(h_gpu[:, c], h_ref[:, c], rtol=rt, atol=1e-300, err_msg="history column %d" % c)
    for c in (4, 5):
        if cols is None or c in cols:
            assert np.abs(h_gpu[:, c] - h_ref[:, c]).max() < divtol, ("history column", c)


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O
