"""The fixed point of the GPU's implicit solve iteration (tests/fdm_model.py)
against the reference's own fdMatrix::solve on the golden case
(tests/golden/im_*.npz): the two iterations differ, their converged
solutions must not.  CPU only."""
import numpy as np
import pytest

from conftest import load_golden, rel_l2
from fdm_model import line_jacobi_model


def residual(al, ap, b, x):
    """fdMatrix::residual: RMS of b - A x over the (N0+1)(N1+1)(N2+1) nodes
    the reference loops over, its duplicate periodic nodes counted again."""
    r = b - ap * x
    for l, (ax, sh) in {0: (1, 1), 1: (1, -1), 2: (0, 1), 3: (0, -1), 4: (2, 1), 5: (2, -1)}.items():
        r -= al[l] * np.roll(x, -sh, axis=ax)
    w = np.ones(x.shape)
    w[0, :, :] *= 2
    w[:, 0, :] *= 2
    w[:, :, 0] *= 2
    return float(np.sqrt(np.sum(w * r * r) / np.prod([n + 1 for n in x.shape])))


@pytest.mark.parametrize("case", ["im_7x6x8.npz", "im_9x5x6_m4.npz"])
def test_line_model_converges_to_the_reference_solution(case):
    g = load_golden(case)
    al, ap, b = g["al"], g["ap"] - float(g["c"]), g["src"] + g["f"][0]
    tol, max_its = float(g["tol"]), int(g["max_its"])
    x, its = g["x"][0].copy(), 0
    while its < max_its and residual(al, ap, b, x) > tol:
        x = line_jacobi_model(al, ap, b, x, 1)
        its += 1
    assert 0 < its < max_its
    assert rel_l2(x, g["x_solved"][0]) < 1e-12
