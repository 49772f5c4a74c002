"""A numpy model of the GPU's implicit solve iteration (nova_fdm_solve): per
iteration, line sweeps along j, i, k, each solving every line's periodic
tridiagonal system at once with the neighbours off the line taken at the
sweep's start.  Test infrastructure: the GPU tests compare the library's
iterates with it, the CPU tests its fixed point with the reference's solve."""
import numpy as np


def line_jacobi_model(al, ap, b, x, its):
    """The GPU's iteration in numpy: per iteration, sweeps along j, i, k, each
    solving every line's periodic tridiagonal system at once (dense solves)
    with the neighbours off the line from the sweep's start."""
    lo_hi = {0: (3, 2), 1: (1, 0), 2: (5, 4)}
    nbr = {0: (1, 1), 1: (1, -1), 2: (0, 1), 3: (0, -1), 4: (2, 1), 5: (2, -1)}  # l -> (axis, shift)
    for _ in range(its):
        for ax in (1, 0, 2):
            lo, hi = lo_hi[ax]
            d = b.copy()
            for l, (a2, sh) in nbr.items():
                if a2 != ax:
                    d -= al[l] * np.roll(x, -sh, axis=a2)
            A, B, Cc, D = (np.moveaxis(v, ax, -1) for v in (al[lo], ap, al[hi], d))
            n = A.shape[-1]
            T = np.zeros(A.shape[:-1] + (n, n))
            idx = np.arange(n)
            T[..., idx, idx] = B
            np.add.at(T, (Ellipsis, idx, (idx - 1) % n), A)
            np.add.at(T, (Ellipsis, idx, (idx + 1) % n), Cc)
            x = np.moveaxis(np.linalg.solve(T, D[..., None])[..., 0], -1, ax)
    return x
