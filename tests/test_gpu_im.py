"""The implicit operators of src/im on the GPU (nova_im_laplacian, nova_fdm_*)
against the reference's own runs (tests/golden/im_*.npz, 6th and 4th order, made
by tests/golden/make_golden.py from im::laplacian and fdMatrix::solve) and, on a
larger mesh, against an exact spectral solve of the same periodic 7-point
system.  The reference relaxes the lines of a sweep one after another, the GPU
all at once: the iterations differ, the converged solutions agree."""
import numpy as np
import pytest

from conftest import load_golden, rel_l2
from fdm_model import line_jacobi_model

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nova():
    from novaclone_b200 import nova
    return nova


def build(nova, N, L, mu, x0, m=6):
    M = nova.Mesh(N, L=L, m=m)
    x = nova.Field(M, 1).upload_soa(x0)
    return M, x, nova.im.laplacian(mu, x)


CASES = ["im_7x6x8.npz", "im_9x5x6_m4.npz"]


def order(g):
    return int(g["m"]) if "m" in g else 6


@pytest.mark.parametrize("case", CASES)
def test_coefficients_and_source_vs_reference(nova, case):
    g = load_golden(case)
    N = tuple(int(v) for v in g["N"])
    M, x, A = build(nova, N, tuple(g["L"]), float(g["mu"]), g["x"], order(g))
    al, ap, b = A.download()
    assert np.array_equal(al, g["al"]) and np.array_equal(ap, g["ap"])
    # b = -ex::laplacian(mu, x) + A x: the 6th-order Laplacian is the GPU's own (parity 1e-12)
    assert rel_l2(b, g["src"]) < 1e-13


@pytest.mark.parametrize("case", CASES)
def test_solve_vs_reference(nova, case):
    g = load_golden(case)
    N = tuple(int(v) for v in g["N"])
    M, x, A = build(nova, N, tuple(g["L"]), float(g["mu"]), g["x"], order(g))
    A.add_diagonal(-float(g["c"]))
    f = nova.Field(M, 1).upload_soa(g["f"])
    its, res = A.eq(f).solve(float(g["tol"]), int(g["max_its"]))
    assert res <= float(g["tol"]) and 0 < its < int(g["max_its"])
    assert rel_l2(x.download_soa(), g["x_solved"]) < 1e-12
    assert A.residual() <= float(g["tol"])


def spectral_solve(b, cx, cy, cz, apv):
    """the periodic 7-point system ap x + sum al x_nbr = b by FFT (constant coefficients)"""
    N = b.shape
    w = [2 * np.cos(2 * np.pi * np.arange(n) / n) for n in N]
    sym = apv + cx * w[0][:, None, None] + cy * w[1][None, :, None] + cz * w[2][None, None, :]
    return np.real(np.fft.ifftn(np.fft.fftn(b) / sym))


def test_solve_vs_exact_spectral_solution(nova):
    N, L, mu, c = (32, 24, 40), (2.0, 1.5, 3.0), 0.02, 5.0
    rng = np.random.default_rng(31)
    x0, f = rng.standard_normal((1,) + N), rng.standard_normal((1,) + N)
    M, x, A = build(nova, N, L, mu, x0)
    al, ap, b = A.download()
    A.add_diagonal(-c)
    fg = nova.Field(M, 1).upload_soa(f)
    its, res = A.eq(fg).solve(1e-13, 500)
    assert res <= 1e-13
    d = [L[a] / N[a] for a in range(3)]
    ref = spectral_solve(b + f[0], mu / d[0] ** 2, mu / d[1] ** 2, mu / d[2] ** 2, float(ap.flat[0]) - c)
    assert rel_l2(x.download_soa()[0], ref) < 1e-11


def test_matrix_algebra(nova):
    N, L = (8, 10, 12), (1.0, 2.0, 3.0)
    rng = np.random.default_rng(5)
    x0, f = rng.standard_normal((1,) + N), rng.standard_normal((1,) + N)
    M, x, A = build(nova, N, L, 0.3, x0)
    B = nova.im.laplacian(0.7, x)       # same mesh: matrices of two meshes do not combine
    with pytest.raises(nova.NovaError) as e:
        A.add(build(nova, N, L, 0.7, x0)[2], 1.0)
    assert e.value.status == nova.E_INVALID

    def state(Q):
        al, ap, b = Q.download()
        return np.concatenate([al, ap[None], b[None]])
    a0, b0 = state(A), state(B)
    A.add(B, -1.0)                      # operator-
    np.testing.assert_allclose(state(A), a0 - b0, rtol=0, atol=1e-13)
    A.scale(-1.0)                       # unary operator-
    np.testing.assert_allclose(state(A), b0 - a0, rtol=0, atol=1e-13)
    A.mul(B)                            # operator*=
    np.testing.assert_allclose(state(A), (b0 - a0) * b0, rtol=1e-14, atol=1e-13)
    s1 = state(B)
    B.eq(nova.Field(M, 1).upload_soa(f))  # operator==: source += f
    np.testing.assert_allclose(state(B)[7], s1[7] + f[0], rtol=1e-15, atol=1e-14)
    B.add_diagonal(-2.0).relax(0.8)     # ap -= 2, then relax(0.8) with x = x0
    s2 = state(B)
    ap_r = (s1[6] - 2.0) / 0.8
    np.testing.assert_allclose(s2[6], ap_r, rtol=1e-15)
    np.testing.assert_allclose(s2[7], s1[7] + f[0] + (1 - 0.8) / 0.8 * ((s1[6] - 2.0) * x0[0]), rtol=1e-13,
                               atol=1e-13)
    B.set_reference(1, 2, 3, 0.5)
    s3 = state(B)
    assert s3[6][1, 2, 3] == s2[6][1, 2, 3] * 1e15 and s3[7][1, 2, 3] == s2[7][1, 2, 3] + 1e15 * 0.5


def test_refusals(nova):
    W = nova.Mesh((8, 8, 8), walls=(0, 1, 0))
    with pytest.raises(nova.NovaError) as e:
        nova.im.laplacian(1.0, nova.Field(W, 1))
    assert e.value.status == nova.E_UNSUPPORTED
    M = nova.Mesh((8, 8, 8))
    with pytest.raises(nova.NovaError) as e:
        nova.im.laplacian(1.0, nova.Field(M, 3))
    assert e.value.status == nova.E_INVALID
    A = nova.im.laplacian(1.0, nova.Field(M, 1))
    with pytest.raises(nova.NovaError) as e:
        A.set_reference(8, 0, 0, 1.0)
    assert e.value.status == nova.E_INVALID
    with pytest.raises(nova.NovaError) as e:
        A.relax(0.0)
    assert e.value.status == nova.E_INVALID
    with pytest.raises(nova.NovaError) as e:
        A.solve(0.0, -1)
    assert e.value.status == nova.E_INVALID


def test_solve_without_iterations_reports_the_residual(nova):
    N = (8, 10, 12)
    x0 = np.random.default_rng(9).standard_normal((1,) + N)
    M, x, A = build(nova, N, (1.0, 2.0, 3.0), 0.4, x0)
    A.add_diagonal(-2.0)
    assert A.solve(0.0, 0) == (0, A.residual())
    assert np.array_equal(x.download_soa(), x0)


@pytest.mark.parametrize("its", [1, 2, 3])
def test_iterations_match_line_model(nova, its):
    """Exact iteration parity with the model above on a mesh with partial line
    groups and chunks (odd counts end in the solve's second buffer); then the
    matrix changes, so its line factors must be rebuilt, and two more iterations."""
    N, L = (9, 40, 35), (1.0, 2.0, 3.0)
    rng = np.random.default_rng(40 + its)
    x0, f = rng.standard_normal((1,) + N), rng.standard_normal((1,) + N)
    M, x, A = build(nova, N, L, 0.05, x0)
    A.add_diagonal(-3.0).eq(nova.Field(M, 1).upload_soa(f))
    al, ap, b = A.download()
    done, _ = A.solve(0.0, its)
    assert done == its
    assert rel_l2(x.download_soa()[0], line_jacobi_model(al, ap, b, x0[0], its)) < 1e-13
    A.add_diagonal(-1.0)
    al, ap, b = A.download()
    xa = x.download_soa()[0]
    A.solve(0.0, 2)
    assert rel_l2(x.download_soa()[0], line_jacobi_model(al, ap, b, xa, 2)) < 1e-13


def test_cpp_adapter_im_driver(tmp_path):
    """The reference-style C++ program (tests/cpp/im_driver.cpp) through
    include/nova/nova.hpp: (im::laplacian(mu, x) - c) == f, solve, on the golden
    case, against the reference's own solution."""
    import os
    import subprocess
    from oracle import oracle as O
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(root, "novaclone_b200")
    exe = tmp_path / "im_driver"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(root, "include"),
                    os.path.join(root, "tests", "cpp", "im_driver.cpp"), "-L" + libdir, "-lnova_b200",
                    "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    g = load_golden("im_7x6x8.npz")
    OM = O.Mesh(tuple(int(v) for v in g["N"]), L=tuple(g["L"]))
    case = tmp_path / "case"
    O.write_case(str(case), OM)
    OM.to_ghosted(g["x"]).tofile(str(tmp_path / "x.bin"))
    OM.to_ghosted(g["f"]).tofile(str(tmp_path / "f.bin"))
    out = tmp_path / "out.bin"
    res = subprocess.run([str(exe), str(case), repr(float(g["mu"])), repr(float(g["c"])), str(tmp_path / "x.bin"),
                          str(tmp_path / "f.bin"), repr(float(g["tol"])), str(int(g["max_its"])), str(out)],
                         capture_output=True, text=True, check=True)
    assert float(res.stdout.split()[-1]) <= float(g["tol"])
    x = OM.unique(np.fromfile(str(out)).reshape(OM.n + (1,)))
    assert rel_l2(x, g["x_solved"]) < 1e-12
