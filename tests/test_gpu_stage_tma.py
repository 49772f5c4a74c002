"""The TMA-pipelined Navier-Stokes stage kernel against the register-queue
march (NOVA_STAGE_IMPL=tma / march, read when a mesh context is created).
Both run the same point arithmetic, so whole runs must agree bit for bit; the
march itself is pinned to the oracle by test_gpu_advance.py, and meshes of
32^3 and up (N2 % 32 == 0, N1 at least twice the tile height 16 (FP64) or 8
(FP32) and, with periodic y, a multiple of it; walls in y for FP32 only) take
the TMA path by default, so those oracle tests cover it directly too."""
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nova():
    from novaclone_b200 import nova
    return nova


def mesh_with(nova, impl, N, **kw):
    old = os.environ.get("NOVA_STAGE_IMPL")
    os.environ["NOVA_STAGE_IMPL"] = impl
    try:
        return nova.Mesh(N, **kw)
    finally:
        if old is None:
            del os.environ["NOVA_STAGE_IMPL"]
        else:
            os.environ["NOVA_STAGE_IMPL"] = old


# FP64 tiles are 32 x 16, FP32-split tiles 32 x 8.  (33, 32, 32): i chunks of
# 16, 16 and 1 plane; (10, 48, 64): two k tiles, three j tiles (both wrap
# cases and an interior tile); (40, 32, 96): three k tiles.
SIZES = [(33, 32, 32), (10, 48, 64), (40, 32, 96)]
SIZES32 = [(33, 16, 32), (10, 24, 64)]


def run(nova, impl, N, U0, prec, rk_mode, steps=3, **mesh_kw):
    GM = mesh_with(nova, impl, N, **mesh_kw)
    U = nova.Field(GM, 3, prec).upload_soa(U0)
    p = nova.Field(GM, 1)
    nova.advance(GM, nova.run_desc(model="ns", rk_mode=rk_mode, precision=prec, dt=2e-3, nu=0.01), U, p,
                 nsteps=steps)
    return U.download_soa(), p.download_soa()


@pytest.mark.parametrize("N", SIZES)
@pytest.mark.parametrize("rk_mode", ["classical", "literal"])
def test_tma_equals_march_fp64(nova, N, rk_mode):
    U0 = 0.3 * np.random.default_rng(5).standard_normal((3,) + N)
    a = run(nova, "tma", N, U0, nova.F64, rk_mode)
    b = run(nova, "march", N, U0, nova.F64, rk_mode)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("N", SIZES32)
@pytest.mark.parametrize("rk_mode", ["classical", "literal"])
def test_tma_equals_march_fp32_split(nova, N, rk_mode):
    U0 = 0.3 * np.random.default_rng(6).standard_normal((3,) + N)
    a = run(nova, "tma", N, U0, nova.F32SPLIT, rk_mode)
    b = run(nova, "march", N, U0, nova.F32SPLIT, rk_mode)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_tma_equals_march_stretched_z(nova):
    N, kw = (12, 32, 64), dict(L=(2 * np.pi, 2 * np.pi, 1.0), hyperbolic_z=(0.01, 0.01))
    U0 = 0.3 * np.random.default_rng(7).standard_normal((3,) + N)
    a = run(nova, "tma", N, U0, nova.F64, "classical", **kw)
    b = run(nova, "march", N, U0, nova.F64, "classical", **kw)
    assert np.array_equal(a[0], b[0])


def test_tma_taylor_green_vs_oracle(nova, oracle):
    N = (16, 32, 32)
    OM = oracle.Mesh(N)
    U0 = oracle.ic_taylor_green(OM)
    got, _ = run(nova, "tma", N, U0, nova.F64, "classical", steps=4)
    r = oracle.run(OM, OM.to_ghosted(U0), model="ns", rk_mode="classical", nsteps=4, dt=2e-3, nu=0.01)
    ref = OM.unique(r[0])
    for c in range(2):
        assert rel_l2(got[c], ref[c]) < 1e-11


def test_adjoint_through_tma_equals_march(nova):
    """The forward passes agree bit for bit; J comes from the TMA or the tiled
    diagnostics reduction (different summation order), and the reverse stages
    of the TMA adjoint apply the first stage's 1/6 to xi instead of to g, so J
    and the gradients agree to rounding."""
    N = (16, 32, 32)
    U0 = 0.2 * np.random.default_rng(9).standard_normal((3,) + N)
    out = []
    for impl in ("tma", "march"):
        GM = mesh_with(nova, impl, N)
        J, grad = nova.adjoint_grad(GM, nova.run_desc(model="ns", dt=2e-3, nu=0.01), nova.Field(GM, 3).upload_soa(U0),
                                    nsteps=4, checkpoint_every=2)
        out.append((J, grad.download_soa()))
    assert out[0][0] == pytest.approx(out[1][0], rel=1e-14)
    assert rel_l2(out[0][1], out[1][1]) < 1e-13


def test_forcing_tma_on_a_mesh_it_does_not_fit_is_refused(nova):
    GM = mesh_with(nova, "tma", (16, 12, 8))
    U = nova.Field(GM, 3).upload_soa(np.zeros((3, 16, 12, 8)))
    p = nova.Field(GM, 1)
    with pytest.raises(nova.NovaError) as e:
        nova.advance(GM, nova.run_desc(model="ns", dt=1e-3), U, p, nsteps=1)
    assert e.value.status == nova.E_UNSUPPORTED


@pytest.mark.parametrize("rk_mode", ["classical", "literal"])
def test_history_rows_from_the_stage_kernel(nova, rk_mode):
    """FP64 TMA runs take each step's history row inside the next step's first
    stage kernel (the energy, |U|, U_x, the divergence and both curls from the
    stencil values the stage holds), the march runs from the diagnostics kernel:
    same state, same terms up to the order of the sums."""
    N = (40, 32, 64)
    U0 = 0.3 * np.random.default_rng(11).standard_normal((3,) + N)
    hist = {}
    for impl in ("tma", "march"):
        GM = mesh_with(nova, impl, N)
        U = nova.Field(GM, 3).upload_soa(U0)
        rd = nova.run_desc(model="ns", rk_mode=rk_mode, dt=2e-3, nu=0.01, diag_every=2)
        hist[impl] = nova.advance(GM, rd, U, nova.Field(GM, 1), nsteps=7)
    a, b = hist["tma"], hist["march"]
    assert np.array_equal(a[:, :2], b[:, :2])  # step, time; zero rows where no diagnostics were due
    for c in (3, 5, 7, 8, 15):  # the B columns
        assert np.array_equal(a[:, c], b[:, c]) and not np.any(a[:, c])
    assert np.all(a[[1, 3, 5, 6], 2] > 0) and np.all(a[[1, 3, 5, 6], 14] > 0)
    # energy, omega, epsilon, Umax, CFL, enstrophy: the same terms summed in another order
    for c in (2, 6, 9, 10, 11, 12, 13, 14):
        np.testing.assert_allclose(a[:, c], b[:, c], rtol=1e-12, atol=1e-300, err_msg="column %d" % c)
    np.testing.assert_allclose(a[:, 4], b[:, 4], rtol=1e-12, atol=1e-14)


# MHD TMA tiles: FP64 32 x 8, FP32 32 x 16.  (33, 16, 32): i chunks with a
# one-plane tail and both j wrap cases; (10, 32, 64): two k tiles.
MHD_SIZES = [((33, 16, 32), 0), ((10, 32, 64), 0), ((12, 32, 32), 1), ((9, 48, 64), 1)]


@pytest.mark.parametrize("N,prec", MHD_SIZES)
@pytest.mark.parametrize("rk_mode", ["classical", "literal"])
def test_mhd_tma_equals_march(nova, N, prec, rk_mode):
    """The MHD U and B stage kernels on the TMA pipeline (two halo'd fields per
    slot) against the register-queue march: the same point arithmetic
    (mhd_u_rhs, mhd_b_rhs), so whole MHD runs agree to rounding."""
    rng = np.random.default_rng(8)
    U0 = 0.3 * rng.standard_normal((3,) + N)
    B0 = 0.3 * rng.standard_normal((3,) + N)
    out = {}
    for impl in ("tma", "march"):
        GM = mesh_with(nova, impl, N)
        U, B = nova.Field(GM, 3, prec).upload_soa(U0), nova.Field(GM, 3, prec).upload_soa(B0)
        rd = nova.run_desc(model="mhd", rk_mode=rk_mode, precision=prec, dt=2e-3, nu=0.01, eta=0.02)
        nova.advance(GM, rd, U, nova.Field(GM, 1), B, nova.Field(GM, 1), nsteps=3)
        out[impl] = np.concatenate([U.download_soa(), B.download_soa()])
    assert rel_l2(out["tma"], out["march"]) < (1e-14 if prec == 0 else 1e-7)


# walls in y: N1 = N[1] + 1 stored rows, the last tile ragged.  (12, 40, 32)
# stores 41 rows: FP32 tiles of 5 x 8 rows and one of 1.  Non-zero wall values
# exercise both ghost formulas on every component.
WALL_N, WALL_L = (12, 40, 32), (2 * np.pi, 2 * np.pi, np.pi)


def wall_run(nova, impl, prec, rk_mode, poisson, steps=3):
    GM = mesh_with(nova, impl, WALL_N, L=WALL_L, walls=(0, 1, 0))
    y = np.arange(WALL_N[1] + 1) * WALL_L[1] / WALL_N[1]
    U0 = np.zeros((3, WALL_N[0], WALL_N[1] + 1, WALL_N[2]))
    U0[0] = np.tanh(3.0 * (y - np.pi))[None, :, None]
    U0 = U0 + 1e-2 * np.random.default_rng(9).standard_normal(U0.shape)
    types, vals = [0] * 18, [0.0] * 18
    for c in range(3):  # u, w Neumann, v Dirichlet on both walls, non-zero values
        types[6 * c] = types[6 * c + 1] = 2 if c == 1 else 1
        vals[6 * c], vals[6 * c + 1] = 0.1 * (c + 1), -0.05 * (c + 1)
    U = nova.Field(GM, 3, prec).set_bc(types, vals).upload_soa(U0)
    p = nova.Field(GM, 1).set_bc([1, 1] + [0] * 16)
    nova.advance(GM, nova.run_desc(model="ns", rk_mode=rk_mode, precision=prec, dt=2e-3, nu=0.01, poisson=poisson),
                 U, p, nsteps=steps)
    return U.download_soa(), p.download_soa()


@pytest.mark.parametrize("rk_mode,poisson", [("classical", "fft"), ("literal", "fft"), ("shear", "dct")])
def test_tma_equals_march_with_walls(nova, rk_mode, poisson):
    """The FP32-split TMA stage and projection on a wall mesh (one row box
    per plane from j0 - 3, zero filled outside the stored rows, ghosts of the
    mirror rows formed by the warps next to a wall, ragged last tiles) give
    the march's bits; the shear-layer loop runs its stage 5 on it."""
    a = wall_run(nova, "tma", nova.F32SPLIT, rk_mode, poisson)
    b = wall_run(nova, "march", nova.F32SPLIT, rk_mode, poisson)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert np.abs(a[0]).max() > 0.5


@pytest.mark.parametrize("rk_mode,poisson", [("classical", "fft"), ("shear", "dct")])
def test_fp64_walls_projection_on_tma(nova, rk_mode, poisson):
    """FP64 on a wall mesh: the stages run the march by default, the projection
    (divergence with U*'s wall ghosts, correction with p's) the TMA pipeline;
    the run gives the all-march bits.  Forcing the TMA stage in FP64 on a
    wall mesh is refused."""
    a = wall_run(nova, "auto", nova.F64, rk_mode, poisson)
    b = wall_run(nova, "march", nova.F64, rk_mode, poisson)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    with pytest.raises(nova.NovaError) as e:
        wall_run(nova, "tma", nova.F64, "shear", "dct", steps=1)
    assert e.value.status == nova.E_UNSUPPORTED
