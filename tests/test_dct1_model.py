"""CPU model of the DCT-I that the wall Poisson kernel (k_pois_dct) computes
from one N-point complex FFT, checked against the definition
    X_m = x_0 + (-1)^m x_N + 2 sum_{n=1}^{N-1} x_n cos(pi n m / N),
and the solve p = X(s X(rhs)) / (2N) against the periodic solve of the even
extension (the mirror image of the Neumann-0 pressure ghosts).  The kernel's
own GPU results are compared with the even-extension solve in
test_gpu_walls.py; this pins the formulas it is built on."""
import numpy as np
import pytest


def dct1_direct(x):
    N = x.shape[0] - 1
    n = np.arange(N + 1)
    C = np.cos(np.pi * np.outer(n, n) / N)
    C[:, 1:N] *= 2.0
    return C @ x


def dct1_fft(f):
    """The kernel's steps: pre-twiddle, W = DFT_N(w), even outputs from W_k +
    W_{N-k}, X_1 from the cosine sum, odd outputs as a prefix sum of
    i (W_k - W_{N-k})."""
    N = f.shape[0] - 1
    n = np.arange(1, N)
    w = np.empty((N,) + f.shape[1:], dtype=complex)
    w[0] = 0.5 * (f[0] + f[N])
    sn = np.sin(np.pi * n / N).reshape((-1,) + (1,) * (f.ndim - 1))
    w[1:] = 0.5 * (f[1:N] + f[N - 1:0:-1]) - sn * (f[1:N] - f[N - 1:0:-1])
    W = np.fft.fft(w, axis=0)
    X = np.empty((N + 1,) + f.shape[1:], dtype=complex)
    k = np.arange(N // 2 + 1)
    X[2 * k] = W[k % N] + W[(N - k) % N]
    cn = np.cos(np.pi * n / N).reshape(sn.shape)
    run = (f[0] - f[N]) + 2.0 * (cn * f[1:N]).sum(axis=0)
    X[1] = run
    for kk in range(1, N // 2):
        run = run + 1j * (W[kk] - W[N - kk])
        X[2 * kk + 1] = run
    return X


@pytest.mark.parametrize("N", [8, 16, 64, 256])
def test_dct1_from_one_fft_equals_the_definition(N):
    rng = np.random.default_rng(N)
    f = rng.standard_normal((N + 1, 5)) + 1j * rng.standard_normal((N + 1, 5))
    ref = dct1_direct(f)
    got = dct1_fft(f)
    assert np.abs(got - ref).max() < 1e-12 * np.abs(ref).max()


def test_dct1_solve_equals_the_even_extension_solve():
    """rhs on the N + 1 wall-bounded nodes: the DCT-I solve with the modified
    wavenumbers of period 2N and the periodic solve of the even extension to
    2N nodes give the same field."""
    N, L = 64, 2.0 * np.pi
    dy = L / N
    rng = np.random.default_rng(3)
    rhs = rng.standard_normal(N + 1)
    rhs -= (rhs[0] + rhs[N] + 2 * rhs[1:N].sum()) / (2 * N)  # zero mean of the extension
    # k'^2 = -(the symbol of the sixth-order second derivative, weights
    # b_l = c_l / (l+1)^2 with c = (3/2, -3/5, 1/10)) on the 2N-point ring of
    # period 2L; any symbol even in the mode index gives the identity
    m = np.arange(2 * N)
    th = np.pi * m / N
    k2 = -2.0 * (1.5 * (np.cos(th) - 1) - 0.15 * (np.cos(2 * th) - 1) + (np.cos(3 * th) - 1) / 90) / dy**2
    # periodic solve of the even extension
    ext = np.concatenate([rhs, rhs[N - 1:0:-1]])
    spec = np.fft.fft(ext)
    scale = np.where(k2 < 1e-16, 0.0, -1.0 / np.where(k2 < 1e-16, 1.0, k2))
    p_ext = np.fft.ifft(spec * scale).real[: N + 1]
    # DCT-I solve: X(rhs), scale by -1/k'^2 of the same symbol (modes 0..N), X again, / 2N
    X = dct1_fft(rhs.astype(complex).reshape(-1, 1))[:, 0]
    p_dct = (dct1_fft((X * scale[: N + 1]).reshape(-1, 1))[:, 0] / (2 * N)).real
    assert np.abs(p_dct - p_ext).max() < 1e-11 * np.abs(p_ext).max()
