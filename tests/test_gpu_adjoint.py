"""GPU checks of the hand-written discrete adjoint (nova_adjoint_grad).

The gradient of J = mean(1/2 |U(T)|^2) with respect to U(0) is compared with
central finite differences of the forward solver (nova_advance) along seeded
random directions of unit RMS amplitude, eps = 1e-6: agreement <= 1e-6
relative.  The result must not depend on the checkpoint interval, and the
adjoint's own forward pass must reproduce the forward solver's J."""
import numpy as np
import pytest

from conftest import rel_l2

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


def test_adjoint_gradient_matches_central_differences(nova, oracle):
    N = (24, 24, 24)
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
        fd = (forward_J(nova, N, U0 + eps * v, dt, nu, nsteps) - forward_J(nova, N, U0 - eps * v, dt, nu, nsteps)) / (2 * eps)
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
    U = nova.Field(GM, 3)
    with pytest.raises(nova.NovaError) as e:
        nova.adjoint_grad(GM, nova.run_desc(model="mhd", dt=0.01), U, 2)
    assert e.value.status == nova.E_UNSUPPORTED
    with pytest.raises(nova.NovaError) as e:
        nova.adjoint_grad(GM, nova.run_desc(rk_mode="literal", dt=0.01), U, 2)
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
    eps = 1e-6
    for _ in range(3):
        v = smooth_direction(rng, N)
        fd = (Jf(U0 + eps * v) - Jf(U0 - eps * v)) / (2 * eps)
        ad = float(np.sum(g * v))
        assert abs(fd - ad) <= 1e-6 * abs(ad), (fd, ad)
    # window from step 0: dJ/dU0 = U0/N^3 - dEk(N)/dU0
    _, g0 = nova.adjoint_grad(GM, rd, U, nsteps, checkpoint_every=4, window_start=0)
    _, gk = nova.adjoint_grad(GM, rd, U, nsteps, checkpoint_every=4)
    assert rel_l2(g0.download_soa(), U0 / np.prod(N) - gk.download_soa()) < 1e-13
