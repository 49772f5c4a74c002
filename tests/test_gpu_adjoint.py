"""GPU checks of the hand-written discrete adjoint (nova_adjoint_grad).

The gradient of J = mean(1/2 |U(T)|^2) (MHD: also + mean(1/2 |B(T)|^2)) with
respect to U(0) (and B(0)) is compared with central finite differences of the
forward solver (nova_advance) along seeded random directions of unit RMS
amplitude, eps = 1e-6, fourth order (central_fd): agreement <= 1e-6
relative.  The result must not depend on the checkpoint interval, and the
adjoint's own forward pass must reproduce the forward solver's J."""
import numpy as np
import pytest

from conftest import rel_l2


def central_fd(f, eps):
    """d/ds f(s) at s = 0 by the fourth-order central difference
    (8 (f(e) - f(-e)) - (f(2e) - f(-2e))) / 12e: the two-point form's
    truncation e^2 f^(3)(0) / 6 cancels (f may return arrays)."""
    return (8 * (f(eps) - f(-eps)) - (f(2 * eps) - f(-2 * eps))) / (12 * eps)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nova():
    from novaclone_b200 import nova
    return nova


def smooth_direction(rng, N, kmax=3):
    """random low-wavenumber vector field, unit RMS amplitude"""
    x = [np.arange(n) * 2 * np.pi / n for n in N]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    v = np.zeros((3,) + tuple(N))
    for c in range(3):
        for _ in range(6):
            k = rng.integers(-kmax, kmax + 1, size=3)
            ph = rng.uniform(0, 2 * np.pi)
            v[c] += rng.standard_normal() * np.cos(k[0] * X + k[1] * Y + k[2] * Z + ph)
    return v / np.sqrt(np.mean(v ** 2))


def forward_J(nova, N, U0, dt, nu, nsteps):
    GM = nova.Mesh(N)
    U = nova.Field(GM, 3).upload_soa(U0)
    p = nova.Field(GM, 1)
    nova.advance(GM, nova.run_desc(model="ns", rk_mode="classical", dt=dt, nu=nu, diag_every=0), U, p,
                 nsteps=nsteps, history=False)
    u = U.download_soa()
    return 0.5 * float(np.sum(u * u)) / float(np.prod(N))


def base_state(oracle, N, seed=0):
    OM = oracle.Mesh(N)
    rng = np.random.default_rng(seed)
    U0 = oracle.ic_taylor_green(OM) + 0.05 * smooth_direction(rng, N)
    return U0, oracle.cfl_dt(OM, [U0])


@pytest.mark.parametrize("N", [(24, 24, 24), (16, 16, 32)])
def test_adjoint_gradient_matches_central_differences(nova, oracle, N):
    """(16, 16, 32) runs the TMA-fed adjoint stage, (24, 24, 24) the tiled one."""
    nsteps, nu = 12, 1e-2
    U0, dt = base_state(oracle, N)
    GM = nova.Mesh(N)
    U = nova.Field(GM, 3).upload_soa(U0)
    J, grad = nova.adjoint_grad(GM, nova.run_desc(model="ns", rk_mode="classical", dt=dt, nu=nu), U, nsteps,
                                checkpoint_every=5)
    g = grad.download_soa()
    assert J == pytest.approx(forward_J(nova, N, U0, dt, nu, nsteps), rel=1e-13)
    rng = np.random.default_rng(123)
    eps = 1e-6
    for _ in range(4):
        v = smooth_direction(rng, N)
        fd = central_fd(lambda e: forward_J(nova, N, U0 + e * v, dt, nu, nsteps), eps)
        ad = float(np.sum(g * v))
        assert abs(fd - ad) <= 1e-6 * abs(ad), (fd, ad)


def test_adjoint_independent_of_checkpoint_interval(nova, oracle):
    N = (16, 12, 20)
    U0, dt = base_state(oracle, N, seed=1)
    GM = nova.Mesh(N)
    U = nova.Field(GM, 3).upload_soa(U0)
    rd = nova.run_desc(model="ns", rk_mode="classical", dt=dt, nu=5e-3)
    grads = [nova.adjoint_grad(GM, rd, U, 7, checkpoint_every=k)[1].download_soa() for k in (1, 3, 7, 50)]
    for gk in grads[1:]:
        assert rel_l2(gk, grads[0]) < 1e-14
    assert np.array_equal(U.download_soa(), U0)  # the initial field is left untouched


def test_adjoint_zero_steps_is_identity_gradient(nova, oracle):
    """One step with nu = 0 on a divergence-free field: the adjoint still lands in the
    solenoidal space it came from, and <grad, U0> equals 2J to first order."""
    N = (16, 16, 16)
    OM = oracle.Mesh(N)
    U0 = oracle.ic_taylor_green(OM)
    GM = nova.Mesh(N)
    U = nova.Field(GM, 3).upload_soa(U0)
    J, grad = nova.adjoint_grad(GM, nova.run_desc(model="ns", rk_mode="classical", dt=1e-4, nu=0.0), U, 1,
                                checkpoint_every=1)
    g = grad.download_soa() * np.prod(N)
    assert rel_l2(g, U0) < 1e-3


def test_adjoint_unsupported_modes(nova):
    GM = nova.Mesh((8, 8, 8))
    U, B = nova.Field(GM, 3), nova.Field(GM, 3)
    with pytest.raises(nova.NovaError) as e:  # MHD needs B0 and gradB
        nova.adjoint_grad(GM, nova.run_desc(model="mhd", dt=0.01), U, 2)
    assert e.value.status == nova.E_INVALID
    with pytest.raises(nova.NovaError) as e:
        nova.adjoint_grad(GM, nova.run_desc(rk_mode="literal", dt=0.01), U, 2)
    assert e.value.status == nova.E_UNSUPPORTED
    with pytest.raises(nova.NovaError) as e:
        nova.adjoint_grad(GM, nova.run_desc(model="mhd", rk_mode="literal", dt=0.01), U, 2, B0=B)
    assert e.value.status == nova.E_UNSUPPORTED
    with pytest.raises(nova.NovaError) as e:  # Em has no meaning without B
        nova.adjoint_grad(GM, nova.run_desc(dt=0.01), U, 2, total_energy=True)
    assert e.value.status == nova.E_UNSUPPORTED
    SM = nova.Mesh((8, 8, 16), hyperbolic_z=(0.02, 0.02))
    with pytest.raises(nova.NovaError) as e:  # the transposes assume a uniform mesh
        nova.adjoint_grad(SM, nova.run_desc(dt=0.01), nova.Field(SM, 3), 2)
    assert e.value.status == nova.E_UNSUPPORTED


def ek_after(nova, N, U0, dt, nu, nsteps):
    return forward_J(nova, N, U0, dt, nu, nsteps) if nsteps > 0 else 0.5 * float(np.sum(U0 * U0)) / float(np.prod(N))


def test_dissipation_window_objective(nova, oracle):
    """J = sum of the dissipation eps_n dt over steps n0+1..N = Ek(n0) - Ek(N)."""
    N = (16, 16, 16)
    nsteps, n0, nu = 9, 4, 1e-2
    U0, dt = base_state(oracle, N, seed=2)
    GM = nova.Mesh(N)
    U = nova.Field(GM, 3).upload_soa(U0)
    rd = nova.run_desc(model="ns", rk_mode="classical", dt=dt, nu=nu)

    def Jf(u):
        return ek_after(nova, N, u, dt, nu, n0) - ek_after(nova, N, u, dt, nu, nsteps)

    J, grad = nova.adjoint_grad(GM, rd, U, nsteps, checkpoint_every=3, window_start=n0)
    g = grad.download_soa()
    assert J == pytest.approx(Jf(U0), rel=1e-12)
    rng = np.random.default_rng(7)
    eps = 1e-5  # J is a difference of two energies: see test_mhd_dissipation_window_objective
    for _ in range(3):
        v = smooth_direction(rng, N)
        fd = central_fd(lambda e: Jf(U0 + e * v), eps)
        ad = float(np.sum(g * v))
        assert abs(fd - ad) <= 1e-6 * abs(ad), (fd, ad)
    # window from step 0: dJ/dU0 = U0/N^3 - dEk(N)/dU0
    _, g0 = nova.adjoint_grad(GM, rd, U, nsteps, checkpoint_every=4, window_start=0)
    _, gk = nova.adjoint_grad(GM, rd, U, nsteps, checkpoint_every=4)
    assert rel_l2(g0.download_soa(), U0 / np.prod(N) - gk.download_soa()) < 1e-13


# ------------------------------------------------------------------ MHD ----
def energies(u, b, N):
    n = float(np.prod(N))
    return 0.5 * float(np.sum(u * u)) / n, 0.5 * float(np.sum(b * b)) / n


def mhd_forward(nova, N, U0, B0, dt, nu, eta, nsteps):
    """(Ek, Em) after nsteps of the MHD loop body (U loop, then B loop)."""
    if nsteps == 0:
        return energies(U0, B0, N)
    GM = nova.Mesh(N)
    U, B = nova.Field(GM, 3).upload_soa(U0), nova.Field(GM, 3).upload_soa(B0)
    nova.advance(GM, nova.run_desc(model="mhd", rk_mode="classical", dt=dt, nu=nu, eta=eta, diag_every=0), U,
                 nova.Field(GM, 1), B, nova.Field(GM, 1), nsteps=nsteps, history=False)
    return energies(U.download_soa(), B.download_soa(), N)


def mhd_base(oracle, N, seed):
    OM = oracle.Mesh(N)
    rng = np.random.default_rng(seed)
    U0, B0 = oracle.ic_orszag_tang(OM)
    U0 = U0 + 0.05 * smooth_direction(rng, N)
    B0 = B0 + 0.05 * smooth_direction(rng, N)
    return U0, B0, oracle.cfl_dt(OM, [U0, B0])


@pytest.mark.parametrize("total,N", [(True, (16, 16, 16)), (False, (16, 16, 16)), (True, (16, 16, 32))])
def test_mhd_adjoint_matches_central_differences(nova, oracle, total, N):
    """Orszag-Tang + perturbations, 6 steps: directions in U alone, B alone and both;
    (16, 16, 32) runs the TMA-fed adjoint kernels, (16, 16, 16) the tiled ones."""
    nsteps, nu, eta = 6, 1e-2, 2e-2
    U0, B0, dt = mhd_base(oracle, N, seed=4)
    GM = nova.Mesh(N)
    U, B = nova.Field(GM, 3).upload_soa(U0), nova.Field(GM, 3).upload_soa(B0)
    rd = nova.run_desc(model="mhd", rk_mode="classical", dt=dt, nu=nu, eta=eta)
    J, gU, gB = nova.adjoint_grad(GM, rd, U, nsteps, checkpoint_every=4, B0=B, total_energy=total)
    gu, gb = gU.download_soa(), gB.download_soa()

    def Jf(u, b):
        ek, em = mhd_forward(nova, N, u, b, dt, nu, eta, nsteps)
        return ek + em if total else ek

    assert J == pytest.approx(Jf(U0, B0), rel=1e-13)
    assert np.abs(gb).max() > 1e-3 * np.abs(gu).max()  # the coupling really carries gradient into B
    rng = np.random.default_rng(99)
    eps = 1e-6
    for wu, wb in ((1.0, 0.0), (0.0, 1.0), (1.0, 1.0)):
        v, w = wu * smooth_direction(rng, N), wb * smooth_direction(rng, N)
        fd = central_fd(lambda e: Jf(U0 + e * v, B0 + e * w), eps)
        ad = float(np.sum(gu * v) + np.sum(gb * w))
        assert abs(fd - ad) <= 1e-6 * abs(ad), (wu, wb, fd, ad)
    assert np.array_equal(U.download_soa(), U0) and np.array_equal(B.download_soa(), B0)


def test_mhd_adjoint_independent_of_checkpoint_interval(nova, oracle):
    N = (12, 16, 20)
    U0, B0, dt = mhd_base(oracle, N, seed=5)
    GM = nova.Mesh(N)
    U, B = nova.Field(GM, 3).upload_soa(U0), nova.Field(GM, 3).upload_soa(B0)
    rd = nova.run_desc(model="mhd", rk_mode="classical", dt=dt, nu=5e-3, eta=5e-3)
    runs = [nova.adjoint_grad(GM, rd, U, 7, checkpoint_every=k, B0=B, total_energy=True) for k in (1, 3, 7, 50)]
    for r in runs[1:]:
        assert r[0] == runs[0][0]
        assert rel_l2(r[1].download_soa(), runs[0][1].download_soa()) < 1e-14
        assert rel_l2(r[2].download_soa(), runs[0][2].download_soa()) < 1e-14


def test_mhd_dissipation_window_objective(nova, oracle):
    """J = E(n0) - E(N), E = Ek + Em: the total-energy dissipation over the window."""
    N = (16, 16, 16)
    nsteps, n0, nu, eta = 7, 3, 1e-2, 1e-2
    U0, B0, dt = mhd_base(oracle, N, seed=6)
    GM = nova.Mesh(N)
    U, B = nova.Field(GM, 3).upload_soa(U0), nova.Field(GM, 3).upload_soa(B0)
    rd = nova.run_desc(model="mhd", rk_mode="classical", dt=dt, nu=nu, eta=eta)

    def Jf(u, b):
        return sum(mhd_forward(nova, N, u, b, dt, nu, eta, n0)) - sum(mhd_forward(nova, N, u, b, dt, nu, eta, nsteps))

    J, gU, gB = nova.adjoint_grad(GM, rd, U, nsteps, checkpoint_every=2, window_start=n0, B0=B)
    assert J == pytest.approx(Jf(U0, B0), rel=1e-12)
    gu, gb = gU.download_soa(), gB.download_soa()
    rng = np.random.default_rng(11)
    # J is a difference of two O(1) energies (slopes here ~3e-4), so each
    # evaluation carries a rounding of ~1e-15: at eps = 1e-6 that is ~1e-6 of
    # the slope.  eps = 1e-5 brings it to ~1e-7; the fourth-order stencil
    # keeps the truncation (eps^4) negligible.
    eps = 1e-5
    for _ in range(2):
        v, w = smooth_direction(rng, N), smooth_direction(rng, N)
        fd = central_fd(lambda e: Jf(U0 + e * v, B0 + e * w), eps)
        ad = float(np.sum(gu * v) + np.sum(gb * w))
        assert abs(fd - ad) <= 1e-6 * abs(ad), (fd, ad)


# ------------------------------------------------------------ FP32-split ----
SPLIT_TOL = 1e-5  # the split path's error bound against FP64


def split_forward_J(nova, N, U0, dt, nu, nsteps):
    GM = nova.Mesh(N)
    U = nova.Field(GM, 3, nova.F32SPLIT).upload_soa(U0)
    nova.advance(GM, nova.run_desc(model="ns", rk_mode="classical", precision=nova.F32SPLIT, dt=dt, nu=nu,
                                   diag_every=0), U, nova.Field(GM, 1), nsteps=nsteps, history=False)
    u = U.download_soa()
    return 0.5 * float(np.sum(u * u)) / float(np.prod(N))


@pytest.mark.parametrize("N", [(24, 24, 24), (16, 16, 32)])
def test_split_adjoint_matches_fp64_adjoint(nova, oracle, N):
    """(16, 16, 32) runs the TMA split stage kernels, (24, 24, 24) the tiled ones."""
    nsteps, nu = 10, 1e-2
    U0, dt = base_state(oracle, N, seed=8)
    GM = nova.Mesh(N)
    U64 = nova.Field(GM, 3).upload_soa(U0)
    U32 = nova.Field(GM, 3, nova.F32SPLIT).upload_soa(U0)
    kw = dict(model="ns", rk_mode="classical", dt=dt, nu=nu)
    J64, g64 = nova.adjoint_grad(GM, nova.run_desc(**kw), U64, nsteps, checkpoint_every=4)
    J32, g32 = nova.adjoint_grad(GM, nova.run_desc(precision=nova.F32SPLIT, **kw), U32, nsteps, checkpoint_every=4)
    assert J32 == pytest.approx(split_forward_J(nova, N, U0, dt, nu, nsteps), rel=1e-13)
    assert J32 == pytest.approx(J64, rel=1e-6)
    e = rel_l2(g32.download_soa(), g64.download_soa())
    assert e < SPLIT_TOL, e
    assert e > 1e-12  # it really ran in FP32


def test_split_adjoint_checkpoint_interval_and_window(nova, oracle):
    N = (16, 16, 32)
    nsteps, n0, nu = 9, 4, 1e-2
    U0, dt = base_state(oracle, N, seed=9)
    GM = nova.Mesh(N)
    U32 = nova.Field(GM, 3, nova.F32SPLIT).upload_soa(U0)
    rd32 = nova.run_desc(model="ns", rk_mode="classical", precision=nova.F32SPLIT, dt=dt, nu=nu)
    grads = [nova.adjoint_grad(GM, rd32, U32, nsteps, checkpoint_every=k)[1].download_soa() for k in (1, 4, 50)]
    for gk in grads[1:]:  # the recomputed segments repeat the forward pass bit for bit
        assert rel_l2(gk, grads[0]) < 1e-14
    U64 = nova.Field(GM, 3).upload_soa(U0)
    rd64 = nova.run_desc(model="ns", rk_mode="classical", dt=dt, nu=nu)
    J32, w32 = nova.adjoint_grad(GM, rd32, U32, nsteps, checkpoint_every=3, window_start=n0)
    J64, w64 = nova.adjoint_grad(GM, rd64, U64, nsteps, checkpoint_every=3, window_start=n0)
    assert J32 == pytest.approx(J64, rel=1e-5)
    assert rel_l2(w32.download_soa(), w64.download_soa()) < SPLIT_TOL


@pytest.mark.parametrize("N,model", [((16, 16, 32), "ns"), ((12, 24, 64), "ns"), ((16, 16, 32), "mhd")])
def test_tma_adjoint_equals_tiled(nova, oracle, N, model):
    """The TMA-fed adjoint stage (meshes with N2 % 32 == 0, N1 % 8 == 0, N1 >= 16)
    against the tiled one (NOVA_STAGE_IMPL=march): the same arithmetic up to the
    place of the 1/6 of the first reverse stage."""
    import os
    rng = np.random.default_rng(21)
    U0 = 0.5 * smooth_direction(rng, N)
    B0 = 0.5 * smooth_direction(rng, N)
    OM = oracle.Mesh(N)
    dt = oracle.cfl_dt(OM, [U0, B0])
    grads = {}
    for impl in ("auto", "march"):  # auto: the TMA adjoint wherever the mesh fits it
        old = os.environ.get("NOVA_STAGE_IMPL")
        if impl == "auto":
            os.environ.pop("NOVA_STAGE_IMPL", None)
        else:
            os.environ["NOVA_STAGE_IMPL"] = impl
        try:
            GM = nova.Mesh(N)
        finally:
            if old is None:
                os.environ.pop("NOVA_STAGE_IMPL", None)
            else:
                os.environ["NOVA_STAGE_IMPL"] = old
        U = nova.Field(GM, 3).upload_soa(U0)
        rd = nova.run_desc(model=model, rk_mode="classical", dt=dt, nu=1e-2, eta=1e-2)
        if model == "mhd":
            B = nova.Field(GM, 3).upload_soa(B0)
            r = nova.adjoint_grad(GM, rd, U, 5, checkpoint_every=2, B0=B, total_energy=True)
            grads[impl] = [r[1].download_soa(), r[2].download_soa()]
        else:
            r = nova.adjoint_grad(GM, rd, U, 5, checkpoint_every=2)
            grads[impl] = [r[1].download_soa()]
    for a, b in zip(grads["auto"], grads["march"]):
        assert rel_l2(a, b) < 1e-13, rel_l2(a, b)


def split_mhd_energies(nova, N, U0, B0, dt, nu, eta, nsteps):
    GM = nova.Mesh(N)
    U, B = nova.Field(GM, 3, nova.F32SPLIT).upload_soa(U0), nova.Field(GM, 3, nova.F32SPLIT).upload_soa(B0)
    nova.advance(GM, nova.run_desc(model="mhd", rk_mode="classical", precision=nova.F32SPLIT, dt=dt, nu=nu, eta=eta,
                                   diag_every=0), U, nova.Field(GM, 1), B, nova.Field(GM, 1), nsteps=nsteps,
                 history=False)
    return energies(U.download_soa(), B.download_soa(), N)


@pytest.mark.parametrize("N", [(16, 16, 16), (16, 16, 32)])
def test_split_mhd_adjoint_matches_fp64(nova, oracle, N):
    nsteps, nu, eta = 6, 1e-2, 2e-2
    U0, B0, dt = mhd_base(oracle, N, seed=12)
    GM = nova.Mesh(N)
    kw = dict(model="mhd", rk_mode="classical", dt=dt, nu=nu, eta=eta)
    U64, B64 = nova.Field(GM, 3).upload_soa(U0), nova.Field(GM, 3).upload_soa(B0)
    U32, B32 = (nova.Field(GM, 3, nova.F32SPLIT).upload_soa(U0), nova.Field(GM, 3, nova.F32SPLIT).upload_soa(B0))
    J64, gu64, gb64 = nova.adjoint_grad(GM, nova.run_desc(**kw), U64, nsteps, checkpoint_every=4, B0=B64,
                                        total_energy=True)
    J32, gu32, gb32 = nova.adjoint_grad(GM, nova.run_desc(precision=nova.F32SPLIT, **kw), U32, nsteps,
                                        checkpoint_every=4, B0=B32, total_energy=True)
    assert J32 == pytest.approx(sum(split_mhd_energies(nova, N, U0, B0, dt, nu, eta, nsteps)), rel=1e-13)
    assert J32 == pytest.approx(J64, rel=1e-6)
    for a, b in ((gu32, gu64), (gb32, gb64)):
        e = rel_l2(a.download_soa(), b.download_soa())
        assert 1e-12 < e < SPLIT_TOL, e


def test_split_mhd_adjoint_checkpoints_and_window(nova, oracle):
    N = (16, 16, 32)
    nsteps, n0 = 7, 3
    U0, B0, dt = mhd_base(oracle, N, seed=13)
    GM = nova.Mesh(N)
    kw = dict(model="mhd", rk_mode="classical", dt=dt, nu=1e-2, eta=1e-2)
    U32, B32 = (nova.Field(GM, 3, nova.F32SPLIT).upload_soa(U0), nova.Field(GM, 3, nova.F32SPLIT).upload_soa(B0))
    rd32 = nova.run_desc(precision=nova.F32SPLIT, **kw)
    runs = [nova.adjoint_grad(GM, rd32, U32, nsteps, checkpoint_every=k, B0=B32) for k in (1, 3, 50)]
    for r in runs[1:]:
        assert r[0] == runs[0][0]
        assert rel_l2(r[1].download_soa(), runs[0][1].download_soa()) < 1e-14
        assert rel_l2(r[2].download_soa(), runs[0][2].download_soa()) < 1e-14
    U64, B64 = nova.Field(GM, 3).upload_soa(U0), nova.Field(GM, 3).upload_soa(B0)
    J32, u32, b32 = nova.adjoint_grad(GM, rd32, U32, nsteps, checkpoint_every=2, window_start=n0, B0=B32)
    J64, u64, b64 = nova.adjoint_grad(GM, nova.run_desc(**kw), U64, nsteps, checkpoint_every=2, window_start=n0,
                                      B0=B64)
    assert J32 == pytest.approx(J64, rel=1e-5)
    assert rel_l2(u32.download_soa(), u64.download_soa()) < SPLIT_TOL
    assert rel_l2(b32.download_soa(), b64.download_soa()) < SPLIT_TOL


@pytest.mark.parametrize("N", [(24, 24, 24), (16, 16, 32)])
def test_dot_product_identity(nova, oracle, N):
    """<D Phi v, w> = <v, D Phi^T w> for the N-step map Phi of nova_advance
    (classical RK4 + projection, FP64).  The adjoint side is nova_adjoint_grad
    with the linear objective J = <w, U(N)>/N^3 (its gradient is D Phi^T w / N^3);
    the tangent side is the central difference of the forward states,
    (Phi(U0 + e v) - Phi(U0 - e v)) / (2 e), e = 1e-6.  w and v are seeded white
    noise (every mode, no symmetry of the base state annihilates them)."""
    nsteps, nu, eps = 8, 1e-2, 1e-6
    U0, dt = base_state(oracle, N)
    rng = np.random.default_rng(77)
    v = rng.standard_normal((3,) + N)
    w = rng.standard_normal((3,) + N)
    n3 = float(np.prod(N))
    GM = nova.Mesh(N)
    rd = nova.run_desc(model="ns", rk_mode="classical", dt=dt, nu=nu, diag_every=0)

    def phi(U_init):
        U = nova.Field(GM, 3).upload_soa(U_init)
        nova.advance(GM, rd, U, nova.Field(GM, 1), nsteps=nsteps, history=False)
        return U.download_soa()

    J, g = nova.adjoint_grad(GM, rd, nova.Field(GM, 3).upload_soa(U0), nsteps, checkpoint_every=3,
                             weight=nova.Field(GM, 3).upload_soa(w))
    UN = phi(U0)
    assert J == pytest.approx(float(np.sum(w * UN)) / n3, rel=1e-12)
    tangent = central_fd(lambda e: phi(U0 + e * v), eps)
    lhs = float(np.sum(tangent * w)) / n3
    rhs = float(np.sum(v * g.download_soa()))
    err = abs(lhs - rhs) / abs(rhs)
    print("dot-product test %s: <J v, w> = %.15e, <v, J^T w> = %.15e, rel. err %.2e" % (N, lhs, rhs, err))
    assert err < 1e-7


def test_linear_objective_is_refused_where_not_built(nova):
    GM = nova.Mesh((16, 16, 16))
    U, w = nova.Field(GM, 3, nova.F32SPLIT), nova.Field(GM, 3)
    rd = nova.run_desc(model="ns", rk_mode="classical", precision=nova.F32SPLIT, dt=1e-3, nu=1e-2)
    with pytest.raises(nova.NovaError) as e:
        nova.adjoint_grad(GM, rd, U, 2, checkpoint_every=1, weight=w)
    assert e.value.status == nova.E_UNSUPPORTED
