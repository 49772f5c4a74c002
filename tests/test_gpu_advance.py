"""GPU parity of the fused time advance (nova_advance) against the oracle and
the reference's golden vectors: FP64 relative L2 error per field <= 1e-11
after N steps (the FP64 parity bar), the diagnostics history overlaid,
and the FP32-split path's error against FP64 stated and bounded."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, check_history, load_golden, rel_l2

pytestmark = pytest.mark.gpu

TOL64 = 1e-11


@pytest.fixture(scope="module")
def nova():
    from novaclone_b200 import nova
    return nova


def gpu_run(nova, OM, U0, B0=None, precision=0, **kw):
    GM = nova.Mesh(OM.N, L=OM.L)
    U = nova.Field(GM, 3, precision).upload_soa(U0)
    p = nova.Field(GM, 1)
    B = pB = None
    if B0 is not None:
        B = nova.Field(GM, 3, precision).upload_soa(B0)
        pB = nova.Field(GM, 1)
    nsteps = kw.pop("nsteps")
    rd = nova.run_desc(precision=precision, **kw)
    hist = nova.advance(GM, rd, U, p, B, pB, nsteps=nsteps)
    out = {"U": U.download_soa(), "p": p.download_soa(), "hist": hist}
    if B is not None:
        out["B"] = B.download_soa()
        out["pB"] = pB.download_soa()
    return out


def oracle_run(oracle, OM, U0, B0=None, **kw):
    r = oracle.run(OM, OM.to_ghosted(U0), None if B0 is None else OM.to_ghosted(B0), **kw)
    out = {"U": OM.unique(r[0]), "p": OM.unique(r[2]), "hist": r[4]}
    if B0 is not None:
        out["B"] = OM.unique(r[1])
        out["pB"] = OM.unique(r[3])
    return out


def check_hist(h_gpu, h_ref, divtol=1e-11):
    check_history(h_gpu, h_ref, divtol=divtol)


@pytest.mark.parametrize("rk_mode,N", [("classical", (32, 32, 32)), ("literal", (32, 32, 32)),
                                        ("classical", (64, 16, 32))])
def test_taylor_green_fp64_vs_oracle(nova, oracle, rk_mode, N):
    """(64, 16, 32): TMA stage kernels and the i-direction solve fused with the scale."""
    OM = oracle.Mesh(N)
    U0 = oracle.ic_taylor_green(OM)
    dt = oracle.cfl_dt(OM, [U0])
    kw = dict(model="ns", rk_mode=rk_mode, nsteps=20, dt=dt, nu=1 / 1600)
    g = gpu_run(nova, OM, U0, **kw)
    o = oracle_run(oracle, OM, U0, **kw)
    for c in range(3):  # w = 0 initially; -dp/dz makes it grow
        assert rel_l2(g["U"][c], o["U"][c]) < TOL64, (c, rel_l2(g["U"][c], o["U"][c]))
    assert rel_l2(g["p"], o["p"]) < TOL64
    check_hist(g["hist"], o["hist"])


@pytest.mark.parametrize("rk_mode", ["classical", "literal"])
def test_orszag_tang_fp64_vs_oracle(nova, oracle, rk_mode):
    OM = oracle.Mesh((24, 24, 24))
    U0, B0 = oracle.ic_orszag_tang(OM)
    dt = oracle.cfl_dt(OM, [U0, B0])
    kw = dict(model="mhd", rk_mode=rk_mode, nsteps=10, dt=dt, nu=1e-3, eta=1e-3)
    g = gpu_run(nova, OM, U0, B0, **kw)
    o = oracle_run(oracle, OM, U0, B0, **kw)
    for f in ("U", "B"):
        for c in range(3):
            if np.abs(o[f][c]).max() > 1e-8:
                assert rel_l2(g[f][c], o[f][c]) < TOL64, (f, c)
    assert rel_l2(g["p"], o["p"]) < TOL64
    check_hist(g["hist"], o["hist"])


@pytest.mark.parametrize("name", ["tg_12_classical.npz", "tg_12_literal.npz", "ot_12_classical.npz",
                                  "ot_12_literal.npz", "tg_12_shear.npz", "ot_12_shear.npz"])
def test_advance_vs_reference_golden(nova, oracle, name):
    g = load_golden(name)
    OM = oracle.Mesh(tuple(int(v) for v in g["N"]), L=tuple(g["L"]))
    model = str(g["model"])
    kw = dict(model=model, rk_mode=str(g["rk_mode"]), nsteps=int(g["nsteps"]), dt=float(g["dt"]),
              nu=float(g["nu"]), eta=float(g["eta"]))
    r = gpu_run(nova, OM, g["U0"], g["B0"] if model == "mhd" else None, **kw)
    fields = ("U", "p", "B", "pB") if model == "mhd" else ("U", "p")
    for f in fields:
        for c in range(g[f].shape[0]):
            if np.abs(g[f][c]).max() > 1e-8:
                assert rel_l2(r[f][c], g[f][c]) < TOL64, (f, c)
    check_hist(r["hist"], g["hist"])


@pytest.mark.parametrize("N", [(20, 12, 36), (40, 9, 16), (7, 33, 10)])
def test_non_tile_multiple_sizes(nova, oracle, N):
    OM = oracle.Mesh(N, L=(2 * np.pi, 3.0, 5.0))
    rng = np.random.default_rng(9)
    U0 = oracle.ic_taylor_green(OM) + 0.05 * rng.standard_normal((3,) + N)
    kw = dict(model="ns", rk_mode="classical", nsteps=4, dt=0.01, nu=0.01)
    g = gpu_run(nova, OM, U0, **kw)
    o = oracle_run(oracle, OM, U0, **kw)
    for c in range(3):
        assert rel_l2(g["U"][c], o["U"][c]) < TOL64


def test_fp32_split_error_is_bounded(nova, oracle):
    """FP32-split vs FP64 (both on the GPU) and vs the oracle: relative L2 <= 1e-5."""
    OM = oracle.Mesh((32, 32, 32))
    U0 = oracle.ic_taylor_green(OM)
    dt = oracle.cfl_dt(OM, [U0])
    kw = dict(model="ns", rk_mode="classical", nsteps=20, dt=dt, nu=1 / 1600)
    g64 = gpu_run(nova, OM, U0, precision=0, **kw)
    g32 = gpu_run(nova, OM, U0, precision=1, **kw)
    o = oracle_run(oracle, OM, U0, **kw)
    for c in range(2):
        e64 = rel_l2(g32["U"][c], g64["U"][c])
        eor = rel_l2(g32["U"][c], o["U"][c])
        assert e64 < 1e-5 and eor < 1e-5, (e64, eor)
        assert e64 > 1e-12  # it really ran in FP32
    assert g32["hist"][-1, 4] < 1e-10  # the FP64 projection still removes the divergence


def test_mhd_jet_vs_oracle_and_split_error(nova, oracle):
    """The MHD jet configuration on a small mesh (x, y in [-4, 4], z in [0, 16],
    the reference app's scheme: literal U loop, refreshed B loop): FP64 against
    the oracle, FP32-split against FP64."""
    OM = oracle.Mesh((24, 24, 48), L=(8.0, 8.0, 16.0), origin=(-4.0, -4.0, 0.0))
    U0, B0 = oracle.ic_mhd_jet(OM)
    dt = oracle.cfl_dt(OM, [U0, B0])
    kw = dict(model="mhd", rk_mode="literal", nsteps=10, dt=dt, nu=1 / 1500, eta=1 / 1500)
    g = gpu_run(nova, OM, U0, B0, **kw)
    o = oracle_run(oracle, OM, U0, B0, **kw)
    for f in ("U", "B"):
        assert rel_l2(g[f], o[f]) < TOL64, (f, rel_l2(g[f], o[f]))
    assert rel_l2(g["p"], o["p"]) < TOL64
    check_hist(g["hist"], o["hist"])
    s = gpu_run(nova, OM, U0, B0, precision=nova.F32SPLIT, **kw)
    for f in ("U", "B"):
        assert rel_l2(s[f], g[f]) < 1e-5


def test_fp32_split_mhd_error_is_bounded(nova, oracle):
    OM = oracle.Mesh((24, 24, 24))
    U0, B0 = oracle.ic_orszag_tang(OM)
    dt = oracle.cfl_dt(OM, [U0, B0])
    kw = dict(model="mhd", rk_mode="classical", nsteps=10, dt=dt, nu=1e-3, eta=1e-3)
    g64 = gpu_run(nova, OM, U0, B0, precision=0, **kw)
    g32 = gpu_run(nova, OM, U0, B0, precision=1, **kw)
    for f in ("U", "B"):
        for c in range(2):
            assert rel_l2(g32[f][c], g64[f][c]) < 1e-5


def test_nonfinite_state_is_reported(nova, oracle):
    OM = oracle.Mesh((8, 8, 8))
    U0 = oracle.ic_taylor_green(OM)
    U0[0, 1, 2, 3] = np.nan
    with pytest.raises(nova.NovaError) as e:
        gpu_run(nova, OM, U0, model="ns", rk_mode="classical", nsteps=2, dt=0.01, nu=0.01)
    assert e.value.status == nova.E_NONFINITE


def test_advance_argument_errors(nova):
    GM = nova.Mesh((8, 8, 8))
    U = nova.Field(GM, 3, nova.F32SPLIT)
    p = nova.Field(GM, 1)
    with pytest.raises(nova.NovaError) as e:
        nova.advance(GM, nova.run_desc(precision=nova.F64, dt=0.01), U, p, nsteps=1)  # precision mismatch
    assert e.value.status == nova.E_INVALID
    GM4 = nova.Mesh((8, 8, 8), m=4)
    U4 = nova.Field(GM4, 3)
    p4 = nova.Field(GM4, 1)
    with pytest.raises(nova.NovaError) as e:
        nova.advance(GM4, nova.run_desc(dt=0.01), U4, p4, nsteps=1)
    assert e.value.status == nova.E_UNSUPPORTED


def test_cpp_adapter_driver(nova, oracle, tmp_path):
    """The reference-style C++ host program (tests/cpp/tg_driver.cpp) through include/nova/nova.hpp."""
    exe = tmp_path / "tg_driver"
    libdir = os.path.join(ROOT, "novaclone_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "tg_driver.cpp"), "-L" + libdir, "-lnova_b200",
                    "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    OM = oracle.Mesh((16, 16, 16))
    case = tmp_path / "case"
    oracle.write_case(str(case), OM)
    out = tmp_path / "U.bin"
    res = subprocess.run([str(exe), str(case), "5", "0.05", str(1 / 1600), "classical", str(out)],
                         capture_output=True, text=True, check=True)
    Ug = np.fromfile(out).reshape(OM.n + (3,))
    o = oracle_run(oracle, OM, oracle.ic_taylor_green(OM), model="ns", rk_mode="classical", nsteps=5, dt=0.05,
                   nu=1 / 1600)
    for c in range(2):
        assert rel_l2(OM.unique(Ug)[c], o["U"][c]) < TOL64
    maxdiv = float(res.stdout.split()[-1])
    assert maxdiv < 1e-12
