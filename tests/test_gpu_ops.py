"""GPU parity of the ex:: drop-in operators and the Poisson solve, through the
C ABI, against the oracle (same seeded inputs) and the reference's golden
vectors.  FP64: relative max error <= 1e-12 (operators are O(1/dx^2) sums of
O(1) inputs, so this bounds a few ulps of the largest term)."""
import numpy as np
import pytest

from conftest import load_golden, rel_max

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def nova():
    from novaclone_b200 import nova
    return nova


SIZES = [((10, 8, 6), (2 * np.pi, 2.0, 3.0), 6), ((33, 17, 40), (2 * np.pi,) * 3, 6), ((16, 12, 8), (1.0, 2.0, 3.0), 4),
         ((8, 8, 8), (2 * np.pi,) * 3, 2), ((12, 10, 20), (2 * np.pi,) * 3, 8), ((3, 5, 7), (1.0, 1.0, 1.0), 6)]


@pytest.mark.parametrize("N,L,m", SIZES)
def test_operators_vs_oracle(nova, oracle, N, L, m):
    rng = np.random.default_rng(11)
    OM = oracle.Mesh(N, L=L, m=m)
    GM = nova.Mesh(N, L=L, m=m)
    U = rng.standard_normal((3,) + N)
    s = rng.standard_normal((1,) + N)
    Ug, sg = OM.to_ghosted(U), OM.to_ghosted(s)
    dU = nova.Field(GM, 3).upload(Ug)
    ds = nova.Field(GM, 1).upload(sg)
    nu = 0.013
    cases = {
        "grad_s": (nova.ex.grad(ds), oracle.grad_s(OM, sg)),
        "grad_v": (nova.ex.grad(dU), oracle.grad_v(OM, Ug)),
        "div_v": (nova.ex.div(dU), oracle.div_v(OM, Ug)),
        "div_vv": (nova.ex.div(dU, dU), oracle.div_vf(OM, Ug, Ug)),
        "div_vs": (nova.ex.div(dU, ds), oracle.div_vf(OM, Ug, sg)),
        "curl": (nova.ex.curl(dU), oracle.curl(OM, Ug)),
        "lap_v": (nova.ex.laplacian(nu, dU), oracle.lap(OM, nu, Ug)),
        "lap_s": (nova.ex.laplacian(nu, ds), oracle.lap(OM, nu, sg)),
    }
    for name, (g, o) in cases.items():
        got = OM.interior(g.download())
        ref = OM.interior(o)
        assert rel_max(got, ref) < TOL, (name, rel_max(got, ref))


@pytest.mark.parametrize("name", ["ops_10x8x6.npz", "ops_16x12x8_m4.npz"])
def test_operators_vs_reference_golden(nova, oracle, name):
    g = load_golden(name)
    N, L, m = tuple(int(v) for v in g["N"]), tuple(g["L"]), int(g["m"])
    OM = oracle.Mesh(N, L=L, m=m)
    GM = nova.Mesh(N, L=L, m=m)
    dU = nova.Field(GM, 3).upload(OM.to_ghosted(g["U"]))
    ds = nova.Field(GM, 1).upload(OM.to_ghosted(g["s"]))
    nu = float(g["nu"])
    p = nova.Field(GM, 1)
    pe = nova.poisson(p)
    pe.rhs(ds)
    pe.solve()
    got = {"grad_s": nova.ex.grad(ds), "div_v": nova.ex.div(dU), "div_vv": nova.ex.div(dU, dU),
           "div_vs": nova.ex.div(dU, ds), "lap_v": nova.ex.laplacian(nu, dU), "lap_s": nova.ex.laplacian(nu, ds),
           "curl": nova.ex.curl(dU)}
    for k, f in got.items():
        assert rel_max(OM.interior(f.download()), g["out_" + k]) < TOL, k
    # poisson::solve writes only the N^3 unique nodes (the duplicate node stays as it was)
    ref_p = g["out_poisson"][:, :N[0], :N[1], :N[2]]
    assert rel_max(p.download_soa(), ref_p) < TOL


# N0 = 64 and 256 run the i-direction FFT fused with the scale (k_pois_i);
# N2 = 10 and 18 leave a ragged last group of kz columns; (256, 16, 32) and
# (256, 24, 16) run the TMA-fed k_pois_tma (8-column tiles, the last kz of 8
# j per remainder tile: 2 and 3 of them)
@pytest.mark.parametrize("N", [(16, 16, 16), (24, 12, 18), (9, 6, 15), (64, 12, 18), (256, 8, 10), (64, 32, 64),
                               (64, 256, 256), (256, 16, 32), (256, 24, 16)])
def test_poisson_vs_oracle(nova, oracle, N):
    rng = np.random.default_rng(2)
    OM = oracle.Mesh(N)
    GM = nova.Mesh(N)
    s = rng.standard_normal((1,) + N)
    ds = nova.Field(GM, 1).upload(OM.to_ghosted(s))
    p = nova.Field(GM, 1)
    pe = nova.poisson(p)
    pe.rhs(ds)
    pe.solve()
    ref = OM.unique(oracle.poisson_solve(OM, OM.to_ghosted(s)))
    assert rel_max(p.download_soa(), ref) < TOL


def test_maximum_and_layout_round_trip(nova, oracle):
    N = (12, 10, 14)
    rng = np.random.default_rng(4)
    OM = oracle.Mesh(N)
    GM = nova.Mesh(N)
    U = rng.standard_normal((3,) + N)
    f = nova.Field(GM, 3).upload(OM.to_ghosted(U))
    assert np.array_equal(f.download(), OM.to_ghosted(U))       # ghosts = periodic images
    assert np.array_equal(f.download_soa(), U)
    d = nova.ex.div(f)
    assert nova.tools.maximum(d) == pytest.approx(oracle.maximum(OM, oracle.div_v(OM, OM.to_ghosted(U))), rel=1e-12)


def test_split_field_holds_48_bits(nova):
    N = (8, 8, 8)
    GM = nova.Mesh(N)
    x = np.random.default_rng(5).standard_normal((3,) + N) * 3.0
    f = nova.Field(GM, 3, nova.F32SPLIT).upload_soa(x)
    assert np.abs(f.download_soa() - x).max() <= 4e-14 * np.abs(x).max()


def test_operator_argument_errors(nova):
    GM = nova.Mesh((8, 8, 8))
    a = nova.Field(GM, 3)
    s = nova.Field(GM, 1)
    with pytest.raises(nova.NovaError) as e:
        GM.check(GM.lib.nova_grad_s(GM.h, a.h, s.h))  # wrong component counts
    assert e.value.status == nova.E_INVALID
    # a host buffer whose ghosted shape does not match the mesh is refused by the C ABI
    bad = np.zeros((5, 5, 5, 3))
    n = np.array([5, 5, 5], np.int32)
    st = GM.lib.nova_field_upload(GM.h, a.h, bad.ctypes.data_as(nova.C.POINTER(nova.C.c_double)),
                                  n.ctypes.data_as(nova.C.POINTER(nova.C.c_int)))
    assert st == nova.E_INVALID


def test_stretched_z_metrics_and_operators(nova, oracle):
    """Mesh 'hypz:' stretching (src/Mesh/Mesh.cpp:373-407): metrics equal the
    oracle's, and every operator carries the dz/dxi terms as the reference does."""
    N, hz = (12, 10, 16), (0.03, 0.03)
    OM = oracle.Mesh(N, L=(2 * np.pi, 2 * np.pi, 1.0), hyperbolic_z=hz)
    GM = nova.Mesh(N, L=(2 * np.pi, 2 * np.pi, 1.0), hyperbolic_z=hz)
    a, b = GM.metrics()
    h = OM.h
    assert np.array_equal(a[h:-h], OM.dzdxi[h:-h]) and np.array_equal(b[h:-h], OM.d2zdxi2[h:-h])
    assert np.abs(OM.dzdxi[h:-h] - 1).max() > 0.1  # really stretched
    rng = np.random.default_rng(8)
    U = rng.standard_normal((3,) + N)
    s = rng.standard_normal((1,) + N)
    Ug, sg = OM.to_ghosted(U), OM.to_ghosted(s)
    dU = nova.Field(GM, 3).upload(Ug)
    ds = nova.Field(GM, 1).upload(sg)
    # unique nodes only: the stretched metric is not periodic, so the reference's duplicate
    # node N (which a periodic device field does not store) sees other d2z/dxi2 values
    for got, ref in ((nova.ex.grad(ds), oracle.grad_s(OM, sg)), (nova.ex.div(dU), oracle.div_v(OM, Ug)),
                     (nova.ex.div(dU, dU), oracle.div_vf(OM, Ug, Ug)),
                     (nova.ex.laplacian(0.1, dU), oracle.lap(OM, 0.1, Ug))):
        assert rel_max(got.download_soa(), OM.unique(ref)) < TOL


def test_stretched_z_advance(nova, oracle):
    N, hz = (12, 10, 16), (0.03, 0.03)
    L = (2 * np.pi, 2 * np.pi, 1.0)
    OM = oracle.Mesh(N, L=L, hyperbolic_z=hz)
    GM = nova.Mesh(N, L=L, hyperbolic_z=hz)
    rng = np.random.default_rng(2)
    U0 = 0.3 * rng.standard_normal((3,) + N)
    U = nova.Field(GM, 3).upload_soa(U0)
    p = nova.Field(GM, 1)
    nova.advance(GM, nova.run_desc(model="ns", rk_mode="classical", dt=2e-3, nu=0.01), U, p, nsteps=3)
    r = oracle.run(OM, OM.to_ghosted(U0), model="ns", rk_mode="classical", nsteps=3, dt=2e-3, nu=0.01)
    ref = OM.unique(r[0])
    for c in range(3):
        assert np.linalg.norm(U.download_soa()[c] - ref[c]) / np.linalg.norm(ref[c]) < 1e-11


def test_tensor_divergences_and_field_nu_laplacian_vs_reference_golden(nova, oracle):
    """nova_div_t (tensor, symmTensor), nova_div_st, nova_laplacian_f against the
    reference's own operators (src/ex/div/div.hxx:173-285, laplacian.hxx:64-127)."""
    g = load_golden("ops2_7x6x5.npz")
    N, L = tuple(int(v) for v in g["N"]), tuple(g["L"])
    OM = oracle.Mesh(N, L=L)
    GM = nova.Mesh(N, L=L)
    F = {k: nova.Field(GM, g[k].shape[0]).upload_soa(g[k]) for k in ("T", "S", "s", "nu", "U")}
    got = {"div_t": nova.ex.div(F["T"]), "div_st": nova.ex.div(F["S"]), "div_sT": nova.ex.div(F["s"], F["T"]),
           "lap_f_v": nova.ex.laplacian(F["nu"], F["U"]), "lap_f_s": nova.ex.laplacian(F["nu"], F["s"])}
    for k, f in got.items():
        assert rel_max(OM.interior(f.download()), g["out_" + k]) < TOL, k


def test_field_nu_laplacian_stretched_z_and_walls_vs_oracle(nova, oracle):
    rng = np.random.default_rng(14)
    N, L, hz = (10, 8, 16), (2 * np.pi, 2.0, 1.0), (0.03, 0.03)
    OM = oracle.Mesh(N, L=L, hyperbolic_z=hz)
    GM = nova.Mesh(N, L=L, hyperbolic_z=hz)
    nu = 0.5 + rng.random((1,) + N)
    U = rng.standard_normal((3,) + N)
    ref = oracle.lap_f(OM, OM.to_ghosted(nu), OM.to_ghosted(U))
    got = nova.ex.laplacian(nova.Field(GM, 1).upload_soa(nu), nova.Field(GM, 3).upload_soa(U))
    assert rel_max(got.download_soa(), OM.unique(ref)) < TOL

    # y walls: nu Neumann, U with Dirichlet v and Neumann u, w (the ghosts of src/BC)
    N = (12, 10, 8)
    OM = oracle.Mesh(N, L=(2 * np.pi, 2.0, 1.5))
    GM = nova.Mesh(N, L=(2 * np.pi, 2.0, 1.5), walls=(0, 1, 0))
    spec_u = {"north": [(1, 0.0), (2, 0.3), (1, 0.0)], "south": [(1, 0.1), (2, 0.0), (1, 0.0)]}
    spec_n = {"north": (1, 0.0), "south": (1, 0.0)}
    h = OM.h

    def ghosted(x, spec):
        gg = OM.zeros(x.shape[0])
        gg[h:h + N[0], h:h + N[1] + 1, h:h + N[2]] = np.moveaxis(x, 0, -1)
        return oracle.bc_apply(OM, gg, spec)

    nu = 0.5 + rng.random((1, N[0], N[1] + 1, N[2]))
    U = rng.standard_normal((3, N[0], N[1] + 1, N[2]))
    nug, Ug = ghosted(nu, spec_n), ghosted(U, spec_u)
    ref = oracle.lap_f(OM, nug, Ug)
    fn = nova.Field(GM, 1)
    t, v = oracle.bc_arrays(1, spec_n)
    fn.set_bc(list(t), list(v))
    fu = nova.Field(GM, 3)
    t, v = oracle.bc_arrays(3, spec_u)
    fu.set_bc(list(t), list(v))
    got = nova.ex.laplacian(fn.upload(nug), fu.upload(Ug))
    stored = np.ascontiguousarray(np.moveaxis(ref[h:h + N[0], h:h + N[1] + 1, h:h + N[2]], -1, 0))
    assert rel_max(got.download_soa(), stored) < TOL


def test_cpp_adapter_tensor_operators(oracle, tmp_path):
    """The reference-style C++ program (tests/cpp/ops2_driver.cpp) through
    include/nova/nova.hpp, with its tensor and symmTensor types: the operators
    against the reference's own outputs (tests/golden/ops2_7x6x5.npz), grad of
    a vector against the oracle."""
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(root, "novaclone_b200")
    exe = tmp_path / "ops2_driver"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(root, "include"),
                    os.path.join(root, "tests", "cpp", "ops2_driver.cpp"), "-L" + libdir, "-lnova_b200",
                    "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    g = load_golden("ops2_7x6x5.npz")
    OM = oracle.Mesh(tuple(int(v) for v in g["N"]), L=tuple(g["L"]))
    case = tmp_path / "case"
    oracle.write_case(str(case), OM)
    for k in ("T", "S", "s", "nu", "U"):
        OM.to_ghosted(g[k]).tofile(str(tmp_path / ("in_" + k + ".bin")))
    subprocess.run([str(exe), str(case), str(tmp_path / "in_"), str(tmp_path / "out_")], check=True)

    def read(name, nc):
        return OM.interior(np.fromfile(str(tmp_path / ("out_" + name + ".bin"))).reshape(OM.n + (nc,)))
    for k, nc in (("div_t", 3), ("div_st", 3), ("div_sT", 3), ("lap_f_v", 3), ("lap_f_s", 1)):
        assert rel_max(read(k, nc), g["out_" + k]) < TOL, k
    want = OM.interior(oracle.grad_v(OM, OM.to_ghosted(g["U"])))
    assert rel_max(read("grad_v", 9), want) < TOL


def test_fields_of_another_mesh_are_refused(nova):
    """A field made by a context of a smaller mesh, passed with a larger
    context, is refused with NOVA_E_INVALID by every entry point that reads or
    writes its nodes (its buffers hold fewer nodes than the context's mesh)."""
    import ctypes as C
    small, big = nova.Mesh((8, 8, 8)), nova.Mesh((16, 16, 16))
    s1, s3 = nova.Field(small, 1), nova.Field(small, 3)
    b1, b3 = nova.Field(big, 1), nova.Field(big, 3)
    L, h = big.lib, big.h
    v = C.c_double()
    host = np.zeros(3 * 16 ** 3)
    calls = {
        "maxabs": L.nova_field_maxabs(h, s1.h, C.byref(v)),
        "maxabs_noalloc": L.nova_field_maxabs_noalloc(h, s1.h, C.byref(v)),
        "grad_s": L.nova_grad_s(h, s1.h, b3.h),
        "grad_s out": L.nova_grad_s(h, b1.h, s3.h),
        "div_vf": L.nova_div_vf(h, b3.h, s3.h, b3.h),
        "poisson": L.nova_poisson_solve(h, s1.h, b1.h),
        "upload_soa": L.nova_field_upload_soa(h, s3.h, nova._dptr(host)),
        "download_soa": L.nova_field_download_soa(h, s3.h, nova._dptr(host)),
    }
    st = nova.State(s3.h, b1.h, None, None)
    rd = nova.run_desc(dt=1e-3)
    calls["advance"] = L.nova_advance(h, C.byref(rd), C.byref(st), 1, None)
    assert calls == {k: nova.E_INVALID for k in calls}, calls


def test_cluster_plane_transforms_match_cufft(nova):
    """The one-pass (j, k) plane transforms (clusters of eight CTAs sharing
    their rows through distributed shared memory) against cuFFT's batched 2-D
    transforms (the default) in the same spectral solve: a random
    right-hand side on 64 x 256 x 256, relative max difference <= 1e-13."""
    import os
    N = (64, 256, 256)
    s = np.random.default_rng(12).standard_normal((1,) + N)
    out = {}
    for impl in ("cluster", "cufft"):
        old = os.environ.get("NOVA_FFT")
        if impl == "cluster":
            os.environ["NOVA_FFT"] = "cluster"
        else:
            os.environ.pop("NOVA_FFT", None)
        try:
            GM = nova.Mesh(N)
        finally:
            if old is None:
                os.environ.pop("NOVA_FFT", None)
            else:
                os.environ["NOVA_FFT"] = old
        p = nova.Field(GM, 1)
        pe = nova.poisson(p)
        pe.rhs(nova.Field(GM, 1).upload_soa(s))
        pe.solve()
        out[impl] = p.download_soa()
    assert rel_max(out["cluster"], out["cufft"]) < 1e-13
    assert np.abs(out["cluster"]).max() > 1e-3


@pytest.mark.parametrize("N", [(256, 16, 32), (256, 32, 64)])
def test_pois_tma_equals_register_kernel(nova, N):
    """k_pois_tma (double-buffered bulk-copy tiles, persistent grid) against
    k_pois_i (NOVA_POIS_I=direct) in the same spectral solve: the same
    arithmetic in the same order, so identical bits."""
    import os
    s = np.random.default_rng(13).standard_normal((1,) + N)
    out = {}
    for impl in ("tma", "direct"):
        old = os.environ.get("NOVA_POIS_I")
        if impl == "direct":
            os.environ["NOVA_POIS_I"] = "direct"
        else:
            os.environ.pop("NOVA_POIS_I", None)
        try:
            GM = nova.Mesh(N)
        finally:
            if old is None:
                os.environ.pop("NOVA_POIS_I", None)
            else:
                os.environ["NOVA_POIS_I"] = old
        p = nova.Field(GM, 1)
        pe = nova.poisson(p)
        pe.rhs(nova.Field(GM, 1).upload_soa(s))
        pe.solve()
        out[impl] = p.download_soa()
    assert np.array_equal(out["tma"], out["direct"])
    assert np.abs(out["tma"]).max() > 1e-3
