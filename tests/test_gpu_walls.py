"""GPU parity with walls in y (config: temporal shear layer), against the
oracle running the reference's Neumann/Dirichlet ghost fills
(src/BC/neumannBC.hxx, src/BC/dirichletBC.hxx), its wall-node overwrites and
the periodic FFT solve the reference's wall case uses (app/shearLayer/UEqn.H
calls poisson::solve).  FP64: relative L2 <= 1e-11 per field."""
import numpy as np
import pytest

from conftest import rel_l2, rel_max

pytestmark = pytest.mark.gpu

N = (16, 12, 8)
L = (2 * np.pi, 2 * np.pi, np.pi)
# u, w Neumann / v Dirichlet on the y walls (north = high y, south = low y)
UBC = {"north": [(1, 0.0), (2, 0.0), (1, 0.0)], "south": [(1, 0.0), (2, 0.0), (1, 0.0)]}
PBC = {"north": (1, 0.0), "south": (1, 0.0)}
# non-zero values exercise every ghost formula
UBC_VALS = {"north": [(1, 0.3), (2, 0.1), (1, -0.2)], "south": [(1, -0.4), (2, 0.25), (2, 0.05)]}


@pytest.fixture(scope="module")
def nova():
    from novaclone_b200 import nova
    return nova


def stored(OM, g):
    """ghosted oracle field -> the stored nodes of a mesh with y walls: (nc, N0, N1+1, N2)"""
    h = OM.h
    u = g[h:h + OM.N[0], h:h + OM.N[1] + 1, h:h + OM.N[2]]
    return np.ascontiguousarray(np.moveaxis(u, -1, 0))


def gpu_mesh(nova):
    return nova.Mesh(N, L=L, walls=(0, 1, 0))


def set_bc(nova, f, spec, nc):
    from oracle import oracle as O
    t, v = O.bc_arrays(nc, spec)
    f.set_bc(list(t) + [0] * (18 - len(t)), list(v) + [0.0] * (18 - len(v)))
    return f


def initial_field(oracle, OM, seed=0):
    rng = np.random.default_rng(seed)
    x = OM.origin[0] + np.arange(N[0]) * OM.d[0]
    y = OM.origin[1] + np.arange(N[1] + 1) * OM.d[1]
    z = OM.origin[2] + np.arange(N[2]) * OM.d[2]
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    U = np.stack([np.tanh(2.0 * (Y - np.pi)), 0.1 * np.sin(X) * np.sin(Y), 0.05 * np.cos(Z) * np.sin(Y)])
    return U + 1e-3 * rng.standard_normal(U.shape)


def ghosted_from_stored(oracle, OM, U, spec):
    """stored nodes -> ghosted array with the reference's BCs applied"""
    g = OM.zeros(U.shape[0])
    h = OM.h
    g[h:h + N[0], h:h + N[1] + 1, h:h + N[2]] = np.moveaxis(U, 0, -1)
    return oracle.bc_apply(OM, g, spec)


@pytest.mark.parametrize("spec", [UBC, UBC_VALS])
def test_operators_with_walls(nova, oracle, spec):
    OM = oracle.Mesh(N, L=L)
    GM = gpu_mesh(nova)
    Ug = ghosted_from_stored(oracle, OM, initial_field(oracle, OM), spec)
    sg = ghosted_from_stored(oracle, OM, initial_field(oracle, OM, 1)[:1], {"north": (1, 0.1), "south": (2, -0.3)})
    dU = set_bc(nova, nova.Field(GM, 3), spec, 3).upload(Ug)
    ds = set_bc(nova, nova.Field(GM, 1), {"north": (1, 0.1), "south": (2, -0.3)}, 1).upload(sg)
    cases = {"grad_s": (nova.ex.grad(ds), oracle.grad_s(OM, sg)), "div_v": (nova.ex.div(dU), oracle.div_v(OM, Ug)),
             "div_vv": (nova.ex.div(dU, dU), oracle.div_vf(OM, Ug, Ug)),
             "lap_v": (nova.ex.laplacian(0.02, dU), oracle.lap(OM, 0.02, Ug)),
             "curl": (nova.ex.curl(dU), oracle.curl(OM, Ug))}
    for name, (g, o) in cases.items():
        assert rel_max(g.download_soa(), stored(OM, o)) < 1e-12, name
    # downloads synthesise the wall ghosts with the field's own BC formulas
    assert np.array_equal(dU.download(), Ug)


@pytest.mark.parametrize("rk_mode", ["classical", "literal"])
@pytest.mark.parametrize("spec", [UBC, UBC_VALS])
def test_shear_layer_advance_with_walls(nova, oracle, rk_mode, spec):
    OM = oracle.Mesh(N, L=L)
    GM = gpu_mesh(nova)
    U0 = initial_field(oracle, OM)
    Ug = ghosted_from_stored(oracle, OM, U0, spec)
    kw = dict(model="ns", rk_mode=rk_mode, nsteps=6, dt=0.01, nu=1e-2)
    r = oracle.run(OM, Ug, bcU=spec, bcp=PBC, **kw)
    U = set_bc(nova, nova.Field(GM, 3), spec, 3).upload(Ug)
    p = set_bc(nova, nova.Field(GM, 1), PBC, 1)
    kw.pop("nsteps")
    hist = nova.advance(GM, nova.run_desc(**kw), U, p, nsteps=6)
    got = U.download_soa()
    ref = stored(OM, r[0])
    for c in range(3):
        assert rel_l2(got[c], ref[c]) < 1e-11, (c, rel_l2(got[c], ref[c]))
    assert rel_l2(p.download_soa(), stored(OM, r[2])) < 1e-11
    np.testing.assert_allclose(hist[:, 2], r[4][:, 2], rtol=1e-11)
    assert np.abs(hist[:, 4] - r[4][:, 4]).max() < 1e-10 * max(1.0, np.abs(r[4][:, 4]).max())


@pytest.mark.parametrize("rk_mode", ["shear", "classical"])
def test_shear_layer_golden_with_walls(nova, oracle, rk_mode):
    """The wall-bounded shear layer against the reference's own run
    (tests/golden/shear_walls_12x10x8.npz: app/shearLayer/UEqn.H, the RK4
    weights as stage coefficients with a projection per stage) and, in the
    classical mode, against the oracle."""
    from conftest import check_history, load_golden
    g = load_golden("shear_walls_12x10x8.npz")
    N_ = tuple(int(v) for v in g["N"])
    OM = oracle.Mesh(N_, L=tuple(g["L"]))
    GM = nova.Mesh(N_, L=tuple(g["L"]), walls=(0, 1, 0))
    kw = dict(model="ns", rk_mode=rk_mode, dt=float(g["dt"]), nu=float(g["nu"]))
    U = set_bc(nova, nova.Field(GM, 3), UBC, 3).upload_soa(g["U0"])
    p = set_bc(nova, nova.Field(GM, 1), PBC, 1)
    hist = nova.advance(GM, nova.run_desc(**kw), U, p, nsteps=int(g["nsteps"]))
    if rk_mode == "shear":
        ref_U, ref_p, ref_h = g["U"], g["p"], g["hist"]
    else:
        r = oracle.run(OM, oracle.ghosted_from_stored(OM, g["U0"], UBC), bcU=UBC, bcp=PBC, nsteps=int(g["nsteps"]),
                       **kw)
        ref_U, ref_p, ref_h = oracle.stored_of(OM, r[0]), oracle.stored_of(OM, r[2]), r[4]
    got = U.download_soa()
    for c in range(3):
        assert rel_l2(got[c], ref_U[c]) < 1e-11, (c, rel_l2(got[c], ref_U[c]))
    assert rel_l2(p.download_soa(), ref_p) < 1e-11
    check_history(hist, ref_h, divtol=1e-10 * max(1.0, np.abs(ref_h[:, 4]).max()))


def test_shear_layer_loop_with_walls_vs_oracle(nova, oracle):
    """The shear-layer loop on a 32 x 24 x 16 wall mesh over 12 steps, FP64 against
    the oracle (the periodic solve of the app), and FP32-split against FP64."""
    from conftest import check_history
    N_ = (32, 24, 16)
    Lw = (2 * np.pi, 2 * np.pi, np.pi)
    OM = oracle.Mesh(N_, L=Lw)
    GM = nova.Mesh(N_, L=Lw, walls=(0, 1, 0))
    U0 = oracle.ic_temporal_shear(OM, seed=0, noise=1e-2, delta=4.0)
    kw = dict(model="ns", rk_mode="shear", dt=0.01, nu=1 / 2000)
    r = oracle.run(OM, oracle.ghosted_from_stored(OM, U0, UBC), bcU=UBC, bcp=PBC, nsteps=12, **kw)
    out = {}
    for prec in (nova.F64, nova.F32SPLIT):
        U = set_bc(nova, nova.Field(GM, 3, prec), UBC, 3).upload_soa(U0)
        p = set_bc(nova, nova.Field(GM, 1), PBC, 1)
        h = nova.advance(GM, nova.run_desc(precision=prec, **kw), U, p, nsteps=12)
        out[prec] = (U.download_soa(), p.download_soa(), h)
    got, gp, gh = out[nova.F64]
    ref = oracle.stored_of(OM, r[0])
    for c in range(3):
        assert rel_l2(got[c], ref[c]) < 1e-11, (c, rel_l2(got[c], ref[c]))
    assert rel_l2(gp, oracle.stored_of(OM, r[2])) < 1e-11
    check_history(gh, r[4], divtol=1e-10 * max(1.0, np.abs(r[4][:, 4]).max()))
    assert 0 < rel_l2(out[nova.F32SPLIT][0], got) < 1e-5


def test_walls_fp32_split_error_is_bounded(nova, oracle):
    OM = oracle.Mesh(N, L=L)
    GM = gpu_mesh(nova)
    Ug = ghosted_from_stored(oracle, OM, initial_field(oracle, OM), UBC)
    out = []
    for prec in (nova.F64, nova.F32SPLIT):
        U = set_bc(nova, nova.Field(GM, 3, prec), UBC, 3).upload(Ug)
        p = set_bc(nova, nova.Field(GM, 1), PBC, 1)
        nova.advance(GM, nova.run_desc(model="ns", rk_mode="classical", precision=prec, dt=0.01, nu=1e-2), U, p,
                     nsteps=6)
        out.append(U.download_soa())
    for c in range(3):
        assert rel_l2(out[1][c], out[0][c]) < 1e-5


def test_wall_bc_validation(nova):
    GM = gpu_mesh(nova)
    f = nova.Field(GM, 3)
    with pytest.raises(nova.NovaError) as e:
        f.set_bc([0] * 18)  # periodic faces on the wall axis
    assert e.value.status == nova.E_INVALID
    with pytest.raises(nova.NovaError) as e:
        nova.Mesh(N, L=L, walls=(1, 0, 0))
    assert e.value.status == nova.E_UNSUPPORTED


def test_dct_wall_poisson_makes_interior_rows_divergence_free(nova, oracle):
    """NOVA_POISSON_DCT solves div grad p = div U*/dt on the even extension of
    the N1+1 wall-bounded rows, i.e. with the Neumann-0 mirror the pressure's
    ghosts use, so with no-penetration U* the corrected field is discretely
    divergence-free on every row between the walls.  The reference's periodic
    solve (the FFT mode) leaves an O(dt) divergence there."""
    OM = oracle.Mesh(N, L=L)
    GM = gpu_mesh(nova)
    Ug = ghosted_from_stored(oracle, OM, initial_field(oracle, OM), UBC)
    divs = {}
    for mode in ("dct", "fft"):
        U = set_bc(nova, nova.Field(GM, 3), UBC, 3).upload(Ug)
        p = set_bc(nova, nova.Field(GM, 1), PBC, 1)
        nova.advance(GM, nova.run_desc(model="ns", rk_mode="classical", dt=0.01, nu=1e-2, poisson=mode), U, p,
                     nsteps=3)
        d = nova.ex.div(U).download_soa()[0]
        divs[mode] = np.abs(d[:, 1:N[1], :]).max()
        assert np.all(np.isfinite(U.download_soa()))
    scale = 1.0 / OM.d[1]  # |D U| is O(|U|/dy) at most
    assert divs["dct"] < 1e-12 * scale, divs
    assert divs["fft"] > 1e4 * divs["dct"], divs


def test_dct_wall_poisson_needs_neumann_zero_pressure(nova, oracle):
    OM = oracle.Mesh(N, L=L)
    GM = gpu_mesh(nova)
    Ug = ghosted_from_stored(oracle, OM, initial_field(oracle, OM), UBC)
    U = set_bc(nova, nova.Field(GM, 3), UBC, 3).upload(Ug)
    p = set_bc(nova, nova.Field(GM, 1), {"north": (2, 0.0), "south": (1, 0.0)}, 1)
    with pytest.raises(nova.NovaError) as e:
        nova.advance(GM, nova.run_desc(model="ns", dt=0.01, nu=1e-2, poisson="dct"), U, p, nsteps=1)
    assert e.value.status == nova.E_INVALID


def test_dct1_wall_poisson_equals_even_extension(nova, oracle):
    """With N[1] = 256 the DCT-mode wall solve runs the (i, k) planes of the
    stored rows as batched 2-D cuFFT transforms and the y direction as DCT-I
    from one 256-point FFT per column (k_pois_dct); NOVA_DCT=extend keeps the
    periodic solve on the even extension.  The two are the same linear map:
    the shear-layer loop (a projection per stage) agrees to 1e-12 after 3
    steps, and the interior rows stay divergence-free."""
    import os
    Nb, Lb = (16, 256, 32), (2 * np.pi, 2 * np.pi, np.pi)
    OM = oracle.Mesh(Nb, L=Lb)
    y = np.arange(Nb[1] + 1) * OM.d[1]
    U0 = np.zeros((3, Nb[0], Nb[1] + 1, Nb[2]))
    U0[0] = np.tanh(28.0 * (y - np.pi))[None, :, None]
    U0 = U0 + 1e-3 * np.random.default_rng(3).standard_normal(U0.shape)
    U0[1][:, [0, -1], :] = 0.0
    out, divs = {}, {}
    for impl in ("dct1", "extend"):
        old = os.environ.get("NOVA_DCT")
        if impl == "extend":
            os.environ["NOVA_DCT"] = "extend"
        else:
            os.environ.pop("NOVA_DCT", None)
        try:
            GM = nova.Mesh(Nb, L=Lb, walls=(0, 1, 0))
        finally:
            if old is None:
                os.environ.pop("NOVA_DCT", None)
            else:
                os.environ["NOVA_DCT"] = old
        U = set_bc(nova, nova.Field(GM, 3), UBC, 3).upload_soa(U0)
        p = set_bc(nova, nova.Field(GM, 1), PBC, 1)
        dt = 0.3 * OM.d[0] / np.abs(U0).sum(axis=0).max()
        nova.advance(GM, nova.run_desc(model="ns", rk_mode="shear", dt=dt, nu=1.0 / 2000, poisson="dct"), U, p,
                     nsteps=3)
        out[impl] = U.download_soa()
        divs[impl] = np.abs(nova.ex.div(U).download_soa()[0][:, 1:Nb[1], :]).max()
    assert rel_max(out["dct1"], out["extend"]) < 1e-12
    assert divs["dct1"] < 1e-12 / OM.d[1], divs
