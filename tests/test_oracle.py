"""CPU tests of the oracle: pinned against the reference's golden vectors
(tests/golden, produced by the reference compiled in place), against numpy's
FFT, and against the analytic identities of the central stencils."""
import numpy as np
import pytest

from conftest import load_golden, rel_max


def test_fft_matches_numpy():
    import ctypes as C
    from oracle import oracle as O
    lib = C.CDLL(O.LIB_PATH)
    rng = np.random.default_rng(3)
    for n in [(8, 6, 5), (12, 9, 16), (24, 18, 12), (1, 4, 3), (7, 11, 13)]:
        a = rng.standard_normal(n[::-1]) + 1j * rng.standard_normal(n[::-1])
        buf = np.ascontiguousarray(np.stack([a.real, a.imag], -1))
        for sign, ref in ((-1, np.fft.fftn(a)), (+1, np.fft.ifftn(a) * a.size)):
            b = buf.copy()
            lib.orc_fft3d(np.array(n, np.int32).ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p), sign)
            got = b[..., 0] + 1j * b[..., 1]
            assert np.abs(got - ref).max() / np.abs(ref).max() < 5e-15


@pytest.mark.parametrize("name", ["ops_10x8x6.npz", "ops_16x12x8_m4.npz", "ops_hypz_12x10x16.npz"])
def test_operators_bitwise_vs_reference_golden(oracle, name):
    """Every operator against the reference's own output, bit for bit: 6th and
    4th order, and a 'hypz:' stretched z (Mesh.cpp:373-407), whose metrics the
    operators carry"""
    g = load_golden(name)
    hz = tuple(float(v) for v in g["hypz"]) if "hypz" in g else None
    M = oracle.Mesh(tuple(g["N"]), L=tuple(g["L"]), m=int(g["m"]), hyperbolic_z=hz)
    U = M.to_ghosted(g["U"])
    s = M.to_ghosted(g["s"])
    nu = float(g["nu"])
    mine = {"grad_s": oracle.grad_s(M, s), "div_v": oracle.div_v(M, U), "div_vv": oracle.div_vf(M, U, U),
            "div_vs": oracle.div_vf(M, U, s), "lap_v": oracle.lap(M, nu, U), "lap_s": oracle.lap(M, nu, s),
            "curl": oracle.curl(M, U), "poisson": oracle.poisson_solve(M, s)}
    for k, v in mine.items():
        assert np.array_equal(M.interior(v), g["out_" + k]), k


@pytest.mark.parametrize("name", ["tg_12_classical.npz", "tg_12_literal.npz", "ot_12_classical.npz",
                                  "ot_12_literal.npz", "tg_12_shear.npz", "ot_12_shear.npz"])
def test_time_loop_bitwise_vs_reference_golden(oracle, name):
    """The loop bodies (app/TG_Piosson/RKLoop.H, app/OT_Poisson/UEqn.H + BEqn.H,
    app/shearLayer/UEqn.H) and every history column (app/OT_Poisson/OT.cpp:132-176,
    tools::CFL, tools::maximum of the divergences, the central-curl enstrophies)
    against the reference's own run, bit for bit"""
    g = load_golden(name)
    M = oracle.Mesh(tuple(g["N"]), L=tuple(g["L"]))
    model = str(g["model"])
    B0 = M.to_ghosted(g["B0"]) if model == "mhd" else None
    U, B, p, pB, hist = oracle.run(M, M.to_ghosted(g["U0"]), B0, model=model, rk_mode=str(g["rk_mode"]),
                                   nsteps=int(g["nsteps"]), dt=float(g["dt"]), nu=float(g["nu"]),
                                   eta=float(g["eta"]))
    assert np.array_equal(M.unique(U), g["U"])
    assert np.array_equal(M.unique(p), g["p"])
    assert hist.shape == (int(g["nsteps"]), oracle.HIST_COLS)
    assert np.array_equal(hist, g["hist"])
    if model == "mhd":
        assert np.array_equal(M.unique(B), g["B"])
        assert np.array_equal(M.unique(pB), g["pB"])
        assert np.all(hist[:, 7] > 0) and np.all(hist[:, 15] > 0)  # J terms present
    assert np.all(hist[:, 6] > 0) and np.all(hist[:, 14] > 0) and np.all(hist[:, 11] > 0)


def test_shear_layer_loop_with_walls_bitwise_vs_reference_golden(oracle):
    """app/shearLayer/UEqn.H with Neumann/Dirichlet y walls and the periodic solve
    the app calls (Q8), against the reference's own run"""
    g = load_golden("shear_walls_12x10x8.npz")
    M = oracle.Mesh(tuple(int(v) for v in g["N"]), L=tuple(g["L"]))
    bc = {"north": [(1, 0.0), (2, 0.0), (1, 0.0)], "south": [(1, 0.0), (2, 0.0), (1, 0.0)]}
    pbc = {"north": (1, 0.0), "south": (1, 0.0)}
    Ug = oracle.ghosted_from_stored(M, g["U0"], bc)
    U, B, p, pB, hist = oracle.run(M, Ug, model="ns", rk_mode="shear", nsteps=int(g["nsteps"]), dt=float(g["dt"]),
                                   nu=float(g["nu"]), bcU=bc, bcp=pbc)
    assert np.array_equal(oracle.stored_of(M, U), g["U"])
    assert np.array_equal(oracle.stored_of(M, p), g["p"])
    assert np.array_equal(hist, g["hist"])


def test_history_columns_of_the_taylor_green_field(oracle):
    """Known values of a history row at t = 0 for u = sin x cos y cos z,
    v = -cos x sin y cos z: Ek = 1/8, Umax = 1 and the central curl's enstrophy
    from the modified wavenumber k' of the 6th-order first derivative (all three
    curl components are products of one sine or cosine per axis, each
    differentiated once)"""
    N = 16
    M = oracle.Mesh((N, N, N))
    Ug = M.to_ghosted(oracle.ic_taylor_green(M))
    row = oracle.diag_row(M, Ug, dt=0.1, nu=0.01, t=0.5)
    h = 2 * np.pi / N
    kp = sum(c / (l + 1) * np.sin((l + 1) * h) / h for l, c in enumerate((1.5, -0.6, 0.1)))
    # w = (-cos x sin y sin z D_z', -sin x cos y sin z D_z', 2 sin x sin y cos z D') k' up to signs:
    # 1/2 <|w|^2> = 1/2 k'^2 (1/8 + 1/8 + 4/8) = 3 k'^2 / 8
    assert abs(row[2] - 0.125) < 1e-14
    assert abs(row[10] - 1.0) < 1e-12
    assert abs(row[14] - 3 * kp * kp / 8) < 1e-12
    assert row[4] < 1e-13
    assert abs(row[11] - 0.1 / h) < 1e-12 and abs(row[12] - row[11]) < 1e-15


def test_live_reference_matches_restatement_with_walls(oracle):
    """Neumann/Dirichlet walls and the periodic solve of the wall case (Q8) vs the reference build."""
    if not oracle.ref_available():
        pytest.skip("reference not compiled here (make -C oracle ref)")
    M = oracle.Mesh((12, 10, 8))
    rng = np.random.default_rng(1)
    U0 = M.to_ghosted(oracle.ic_taylor_green(M) + 0.1 * rng.standard_normal((3,) + M.N))
    wallU = {"north": [(1, 0.0), (2, 0.3), (1, 0.1)], "south": [(1, 0.2), (2, 0.0), (1, 0.0)],
             "top": [(2, 0.1), (1, 0.0), (2, 0.0)], "bottom": [(1, 0.0), (1, 0.5), (2, 0.0)]}
    wallp = {"north": (1, 0.0), "south": (1, 0.0)}
    for mode in ("literal", "classical"):
        r = oracle.ref_run(M, U0, model="ns", rk_mode=mode, nsteps=3, dt=0.01, nu=1e-2,
                           bc={"U": wallU, "p": wallp})
        o = oracle.run(M, U0, model="ns", rk_mode=mode, nsteps=3, dt=0.01, nu=1e-2, bcU=wallU, bcp=wallp)
        assert np.array_equal(r[0], o[0]) and np.array_equal(r[2], o[2]) and np.array_equal(r[4], o[4])


def test_first_derivative_modified_wavenumber(oracle):
    """D_x sin(kx) = k'(k) cos(kx), k' = sum_l c_l/(l+1) sin((l+1)k dx)/dx (exact for central stencils)."""
    N = (32, 8, 8)
    M = oracle.Mesh(N)
    x = M.coords()[0]
    dx = M.d[0]
    for kk in (1, 3, 7, 15):
        f = np.broadcast_to(np.sin(kk * x)[:, None, None], N)[None]
        g = M.unique(oracle.grad_s(M, M.to_ghosted(f)))[0]
        c = [1.5, -0.6, 0.1]
        kp = sum(c[l] / (l + 1) * np.sin((l + 1) * kk * dx) / dx for l in range(3))
        assert rel_max(g, kp * np.cos(kk * x)[:, None, None] * np.ones(N)) < 1e-12


def test_laplacian_symbol(oracle):
    N = (8, 32, 8)
    M = oracle.Mesh(N)
    y = M.coords()[1]
    dy = M.d[1]
    kk = 5
    f = np.broadcast_to(np.sin(kk * y)[None, :, None], N)[None]
    lap = M.unique(oracle.lap(M, 1.0, M.to_ghosted(f)))[0]
    c = [1.5, -0.6, 0.1]
    sym = -sum(2 * c[l] * (1 - np.cos((l + 1) * kk * dy)) / ((l + 1) * dy) ** 2 for l in range(3))
    assert rel_max(lap, sym * np.sin(kk * y)[None, :, None] * np.ones(N)) < 1e-11


def test_projection_makes_discrete_divergence_vanish(oracle):
    M = oracle.Mesh((16, 12, 10))
    rng = np.random.default_rng(5)
    U = M.to_ghosted(rng.standard_normal((3,) + M.N))
    d0 = oracle.maximum(M, oracle.div_v(M, U))
    p = oracle.poisson_solve(M, oracle.div_v(M, U))
    p = oracle.bc_apply(M, p)
    U2 = oracle.bc_apply(M, U - oracle.grad_s(M, p))
    d1 = oracle.maximum(M, oracle.div_v(M, U2))
    assert d0 > 1.0 and d1 < 1e-12


def test_taylor_green_initial_field_is_discretely_solenoidal(oracle):
    M = oracle.Mesh((24, 24, 24))
    U = M.to_ghosted(oracle.ic_taylor_green(M))
    assert oracle.maximum(M, oracle.div_v(M, U)) < 1e-13


def test_metrics_of_uniform_mesh(oracle):
    """Mesh::dzdxi_ is 1 and d2zdxi2_ is 0 up to round-off on a uniform mesh."""
    M = oracle.Mesh((8, 8, 256))
    h = M.h
    assert np.abs(M.dzdxi[h:-h] - 1).max() < 1e-12
    assert np.abs(M.d2zdxi2[h:-h]).max() < 1e-9


def test_compressible_taylor_green_bitwise_vs_reference_golden(oracle):
    """app/TG (rhoEqn.H, pEqn.H, UEqn.H) restated with the pinned operators."""
    g = load_golden("wc_tg_12.npz")
    M = oracle.Mesh(tuple(int(v) for v in g["N"]), L=tuple(g["L"]))
    U, rho, p, T, hist = oracle.wc_run(M, M.to_ghosted(g["U0"]), M.to_ghosted(g["rho0"]), M.to_ghosted(g["p0"]),
                                       order="tg", nsteps=int(g["nsteps"]), dt=float(g["dt"]), mu=float(g["mu"]))
    for name, a in (("U", U), ("rho", rho), ("p", p)):
        assert np.array_equal(M.unique(a), g[name]), name
    assert np.array_equal(hist[:, :6], g["hist"])


def test_weakly_compressible_shear_bitwise_vs_reference_golden(oracle):
    """app/shearLayerWC: hydrostatic initialisation (shearLayer.cpp:114-155), then
    UEqn.H (buoyancy), rhoEqn.H, pEqn.H (EOS), TEqn.H."""
    g = load_golden("wc_shear_12x8x16.npz")
    M = oracle.Mesh(tuple(int(v) for v in g["N"]), L=tuple(g["L"]))
    prm = {k: float(g[k]) for k in ("mu", "ka", "c", "rho0", "gz")}
    Tg = M.to_ghosted(g["T0"])
    p, rho = oracle.wc_hydrostatic(M, Tg, c=prm["c"], rho0=prm["rho0"], gz=prm["gz"])
    assert np.array_equal(M.unique(p), g["p_init"]) and np.array_equal(M.unique(rho), g["rho_init"])
    U, rho, p, T, hist = oracle.wc_run(M, M.to_ghosted(g["U0"]), rho, p, Tg, order="shear",
                                       nsteps=int(g["nsteps"]), dt=float(g["dt"]), **prm)
    for name, a in (("U", U), ("rho", rho), ("p", p), ("T", T)):
        assert np.array_equal(M.unique(a), g[name]), name
    assert np.array_equal(hist[:, :6], g["hist"])
    assert np.abs(g["rho"] - g["rho_init"]).max() > 0  # the density really evolves


def test_tensor_operators_and_field_nu_laplacian_bitwise_vs_reference_golden(oracle):
    """ex::div(tensor), div(symmTensor), div(scalar, tensor), laplacian(Field nu, .)."""
    g = load_golden("ops2_7x6x5.npz")
    M = oracle.Mesh(tuple(int(v) for v in g["N"]), L=tuple(g["L"]))
    G = {k: M.to_ghosted(g[k]) for k in ("T", "S", "s", "nu", "U")}
    mine = {"div_t": oracle.div_t(M, G["T"]), "div_st": oracle.div_t(M, G["S"]),
            "div_sT": oracle.div_sT(M, G["s"], G["T"]), "lap_f_v": oracle.lap_f(M, G["nu"], G["U"]),
            "lap_f_s": oracle.lap_f(M, G["nu"], G["s"])}
    for k, v in mine.items():
        assert np.array_equal(M.interior(v), g["out_" + k]), k


@pytest.mark.parametrize("case", ["im_7x6x8.npz", "im_9x5x6_m4.npz"])
def test_im_laplacian_and_line_relaxation_match_the_reference(oracle, case):
    """im::laplacian (coefficients, deferred-correction source) and fdMatrix::solve
    restated against the reference's own runs (tests/golden/im_*.npz, 6th and 4th
    order): bit for bit, the solve's iterations included."""
    g = load_golden(case)
    N = tuple(int(v) for v in g["N"])
    M = oracle.Mesh(N, L=tuple(g["L"]), m=int(g["m"]) if "m" in g else 6)
    xg = M.to_ghosted(g["x"])
    al, ap, src = oracle.im_laplacian(M, float(g["mu"]), xg)
    h = M.h
    inner = (slice(h, h + N[0]), slice(h, h + N[1]), slice(h, h + N[2]))
    assert np.array_equal(np.stack([a[inner] for a in al]), g["al"])
    assert np.array_equal(ap[inner], g["ap"]) and np.array_equal(src[inner], g["src"])
    ap2, src2 = ap - float(g["c"]), src + M.to_ghosted(g["f"])[..., 0]
    x, its, _ = oracle.fdm_solve(M, al, ap2, src2, xg, float(g["tol"]), int(g["max_its"]))
    assert np.array_equal(x[inner][None], g["x_solved"])
    assert oracle.fdm_residual(M, al, ap2, src2, x) == float(g["res"])
