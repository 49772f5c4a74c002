"""GPU parity of the weakly-compressible path (nova_advance_wc,
nova_wc_hydrostatic) against the reference's own output (golden fixtures of
app/TG and app/shearLayerWC) and the oracle.  FP64: relative L2 <= 1e-11 per
field (vector fields over all components)."""
import numpy as np
import pytest

from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-11


@pytest.fixture(scope="module")
def nova():
    from novaclone_b200 import nova
    return nova


def fields(nova, M, U, rho, p, T=None):
    f = [nova.Field(M, 3).upload_soa(U), nova.Field(M, 1).upload_soa(rho), nova.Field(M, 1).upload_soa(p)]
    f.append(None if T is None else nova.Field(M, 1).upload_soa(T))
    return f


def check(got, ref, names):
    for name, a, b in zip(names, got, ref):
        assert rel_l2(a, b) < TOL, (name, rel_l2(a, b))


def test_compressible_taylor_green_vs_reference_golden(nova):
    g = load_golden("wc_tg_12.npz")
    M = nova.Mesh(tuple(int(v) for v in g["N"]), L=tuple(g["L"]))
    U, rho, p, _ = fields(nova, M, g["U0"], g["rho0"], g["p0"])
    wd = nova.wc_desc("tg", dt=float(g["dt"]), mu=float(g["mu"]), eos_k=50.0)
    hist = nova.advance_wc(M, wd, U, rho, p, nsteps=int(g["nsteps"]))
    check([U.download_soa(), rho.download_soa(), p.download_soa()], [g["U"], g["rho"], g["p"]], "U rho p".split())
    np.testing.assert_allclose(hist[:, 2], g["hist"][:, 2], rtol=1e-12)
    assert np.abs(hist[:, 4] - g["hist"][:, 4]).max() < 1e-10 * np.abs(g["hist"][:, 4]).max()


def shear_desc(nova, oracle, g):
    prm = {k: float(g[k]) for k in ("mu", "ka", "c", "rho0", "gz")}
    return prm, nova.wc_desc("shear", dt=float(g["dt"]), mu=prm["mu"], ka=prm["ka"],
                             eos_k=oracle.wc_eos_k(prm["c"], prm["rho0"]), g=(0.0, 0.0, prm["gz"]))


def test_weakly_compressible_shear_vs_reference_golden(nova, oracle):
    g = load_golden("wc_shear_12x8x16.npz")
    M = nova.Mesh(tuple(int(v) for v in g["N"]), L=tuple(g["L"]))
    prm, wd = shear_desc(nova, oracle, g)
    T = nova.Field(M, 1).upload_soa(g["T0"])
    p, rho = nova.Field(M, 1), nova.Field(M, 1)
    nova.wc_hydrostatic(M, wd, prm["rho0"], T, p, rho)
    # the column sum is the reference's; rho = pow(p/K, 1/2) may differ by an ulp
    assert np.array_equal(p.download_soa(), g["p_init"])
    assert np.abs(rho.download_soa() - g["rho_init"]).max() <= 4e-16 * np.abs(g["rho_init"]).max()

    U, rho, p, T = fields(nova, M, g["U0"], g["rho_init"], g["p_init"], g["T0"])
    hist = nova.advance_wc(M, wd, U, rho, p, T, nsteps=int(g["nsteps"]))
    check([U.download_soa(), rho.download_soa(), p.download_soa(), T.download_soa()],
          [g["U"], g["rho"], g["p"], g["T"]], "U rho p T".split())
    # the density and the temperature really moved
    assert rel_l2(g["rho"], g["rho_init"]) > 1e3 * TOL and rel_l2(g["T"], g["T0"]) > 1e3 * TOL
    np.testing.assert_allclose(hist[:, 2], g["hist"][:, 2], rtol=1e-12)


def test_weakly_compressible_shear_stretched_z_vs_oracle(nova, oracle):
    prm = oracle.wc_shear_params(0.1)
    h0 = prm["h0"]
    N, L, hz = (12, 8, 32), (14.0 * h0, 1.7 * h0, 15.0 * h0), (0.02, 0.02)
    OM = oracle.Mesh(N, L=L, hyperbolic_z=hz)
    M = nova.Mesh(N, L=L, hyperbolic_z=hz)
    U0, T0 = oracle.ic_wc_shear(OM, prm, seed=3)
    pg, rg = oracle.wc_hydrostatic(OM, OM.to_ghosted(T0), c=prm["c"], rho0=prm["rho0"], gz=prm["gz"])
    dt = 0.2 * min(OM.d) / (prm["u0"] / 0.1 + prm["u0"] / 2.0)
    kw = {k: prm[k] for k in ("mu", "ka", "c", "rho0", "gz")}
    r = oracle.wc_run(OM, OM.to_ghosted(U0), rg, pg, OM.to_ghosted(T0), order="shear", nsteps=3, dt=dt, **kw)
    U, rho, p, T = fields(nova, M, U0, OM.unique(rg), OM.unique(pg), T0)
    wd = nova.wc_desc("shear", dt=dt, mu=prm["mu"], ka=prm["ka"], eos_k=oracle.wc_eos_k(prm["c"], prm["rho0"]),
                      g=(0.0, 0.0, prm["gz"]))
    nova.advance_wc(M, wd, U, rho, p, T, nsteps=3)
    check([U.download_soa(), rho.download_soa(), p.download_soa(), T.download_soa()],
          [OM.unique(a) for a in r[:4]], "U rho p T".split())


def test_weakly_compressible_argument_errors(nova):
    M = nova.Mesh((8, 8, 8))
    U, rho, p = nova.Field(M, 3), nova.Field(M, 1), nova.Field(M, 1)
    with pytest.raises(nova.NovaError) as e:  # the shear case needs T
        nova.advance_wc(M, nova.wc_desc("shear", dt=1e-3, eos_k=1.0), U, rho, p, None, nsteps=1)
    assert e.value.status == nova.E_INVALID
    W = nova.Mesh((8, 8, 8), walls=(0, 1, 0))
    with pytest.raises(nova.NovaError) as e:
        nova.advance_wc(W, nova.wc_desc("tg", dt=1e-3), nova.Field(W, 3), nova.Field(W, 1), nova.Field(W, 1),
                        nsteps=1)
    assert e.value.status == nova.E_UNSUPPORTED
