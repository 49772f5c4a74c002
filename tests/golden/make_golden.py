"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs oracle/_ref/nova_ref -- the reference's own sources (src/ex, src/poisson,
src/BC, src/Field, src/im, app/TG_Piosson/RKLoop.H, app/OT_Poisson/UEqn.H +
BEqn.H, app/shearLayer/UEqn.H, the compressible app/TG and app/shearLayerWC
loop bodies, and the per-step diagnostics of app/OT_Poisson/OT.cpp with
tools::CFL)
compiled in place by `make -C oracle ref` -- on small seeded inputs and stores
inputs and outputs as .npz.  Needs the reference tree (only present where the
fixtures are generated); the tests only read the .npz files.

    make -C oracle ref && python tests/golden/make_golden.py [name ...]
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402


def ops_case(name, N, L, seed, nu, m=6, hyperbolic_z=None):
    M = O.Mesh(N, L=L, m=m, hyperbolic_z=hyperbolic_z)
    rng = np.random.default_rng(seed)
    U = rng.standard_normal((3,) + M.N)
    s = rng.standard_normal((1,) + M.N)
    out = O.ref_ops(M, M.to_ghosted(U), M.to_ghosted(s), nu)
    res = {"N": np.array(N), "L": np.array(L), "m": np.array(m), "nu": np.array(nu), "U": U, "s": s}
    if hyperbolic_z is not None:
        res["hypz"] = np.array(hyperbolic_z)
    for k, v in out.items():
        res["out_" + k] = M.interior(v)  # incl. the duplicate node, as the reference stores it
    np.savez_compressed(os.path.join(HERE, name), **res)


def run_case(name, N, model, rk_mode, nsteps, dt, nu, eta, L=None):
    L = L or (2 * np.pi,) * 3
    M = O.Mesh(N, L=L)
    if model == "ns":
        U = O.ic_taylor_green(M)
        B = None
    else:
        U, B = O.ic_orszag_tang(M)
    r = O.ref_run(M, M.to_ghosted(U), None if B is None else M.to_ghosted(B), model=model, rk_mode=rk_mode,
                  nsteps=nsteps, dt=dt, nu=nu, eta=eta)
    res = {"N": np.array(N), "L": np.array(L), "model": np.array(model), "rk_mode": np.array(rk_mode),
           "nsteps": np.array(nsteps), "dt": np.array(dt), "nu": np.array(nu), "eta": np.array(eta),
           "U0": U, "U": M.unique(r[0]), "p": M.unique(r[2]), "hist": r[4]}
    if B is not None:
        res["B0"] = B
        res["B"] = M.unique(r[1])
        res["pB"] = M.unique(r[3])
    np.savez_compressed(os.path.join(HERE, name), **res)


# the wall BCs of the temporal shear layer: u, w Neumann-0 and v Dirichlet-0 on
# the y walls, p Neumann-0
SHEAR_BC = {"U": {"north": [(1, 0.0), (2, 0.0), (1, 0.0)], "south": [(1, 0.0), (2, 0.0), (1, 0.0)]},
            "p": {"north": (1, 0.0), "south": (1, 0.0)}}


def shear_case(name, N, L, nsteps, dt, nu, seed=0):
    """app/shearLayer/UEqn.H (RK4 weights as stage coefficients, a projection per
    stage) on a mesh with y walls, the temporal shear layer's initial field"""
    M = O.Mesh(N, L=L)
    U = O.ic_temporal_shear(M, seed=seed, noise=1e-2, delta=2.0)
    Ug = O.ghosted_from_stored(M, U, SHEAR_BC["U"])
    r = O.ref_run(M, Ug, model="ns", rk_mode="shear", nsteps=nsteps, dt=dt, nu=nu, bc=SHEAR_BC)
    np.savez_compressed(os.path.join(HERE, name), N=np.array(N), L=np.array(L), nsteps=np.array(nsteps),
                        dt=np.array(dt), nu=np.array(nu), U0=U, U=O.stored_of(M, r[0]), p=O.stored_of(M, r[2]),
                        hist=r[4])


def wc_tg_case(name, N, nsteps, dt, mu):
    """compressible Taylor-Green (app/TG/TG.cpp): rhoEqn.H, pEqn.H, UEqn.H"""
    M = O.Mesh(N)
    U, rho, p = O.ic_tg_compressible(M)
    r = O.ref_wc_run(M, M.to_ghosted(U), M.to_ghosted(rho), M.to_ghosted(p), order="tg", nsteps=nsteps, dt=dt,
                     mu=mu)
    np.savez_compressed(os.path.join(HERE, name), N=np.array(N), L=np.array(M.L), nsteps=np.array(nsteps),
                        dt=np.array(dt), mu=np.array(mu), U0=U, rho0=rho, p0=p, U=M.unique(r[0]),
                        rho=M.unique(r[1]), p=M.unique(r[2]), hist=r[4])


def wc_shear_case(name, N, nsteps, cfl=0.3, mach=0.1, seed=0):
    """weakly-compressible shear layer (app/shearLayerWC): the hydrostatic
    initialisation of shearLayer.cpp:114-155, then UEqn.H, rhoEqn.H, pEqn.H, TEqn.H"""
    prm = O.wc_shear_params(mach)
    h0 = prm["h0"]
    M = O.Mesh(N, L=(14.0 * h0, 1.7 * h0, 15.0 * h0))
    U, T = O.ic_wc_shear(M, prm, seed)
    pi, rhoi = O.ref_wc_init(M, M.to_ghosted(T), c=prm["c"], rho0=prm["rho0"], gz=prm["gz"])
    dt = cfl * min(M.d) / (prm["u0"] / mach + prm["u0"] / 2.0)  # shearLayer.cpp:182
    kw = {k: prm[k] for k in ("mu", "ka", "c", "rho0", "gz")}
    r = O.ref_wc_run(M, M.to_ghosted(U), rhoi, pi, M.to_ghosted(T), order="shear", nsteps=nsteps, dt=dt, **kw)
    np.savez_compressed(os.path.join(HERE, name), N=np.array(N), L=np.array(M.L), nsteps=np.array(nsteps),
                        dt=np.array(dt), mach=np.array(mach), U0=U, T0=T, p_init=M.unique(pi),
                        rho_init=M.unique(rhoi), U=M.unique(r[0]), rho=M.unique(r[1]), p=M.unique(r[2]),
                        T=M.unique(r[3]), hist=r[4], **{k: np.array(v) for k, v in prm.items()})


def ensight_case(name, N, L, origin, seed, walls=False):
    """the reference's EnSight output of seeded U and p (Mesh::write, Field<T>::write, 2 steps)"""
    import tempfile
    M = O.Mesh(N, L=L, origin=origin)
    rng = np.random.default_rng(seed)
    bc = None
    if walls:
        n1 = N[1] + 1  # the wall nodes are stored: seed the N1+1 rows, apply the reference's BCs
        U = rng.standard_normal((3, N[0], n1, N[2]))
        p = rng.standard_normal((1, N[0], n1, N[2]))
        bc = {"U": {"north": [(1, 0.0), (2, 0.0), (1, 0.0)], "south": [(1, 0.0), (2, 0.0), (1, 0.0)]},
              "p": {"north": (1, 0.0), "south": (1, 0.0)}}
        Ug, pg = M.zeros(3), M.zeros(1)
        h = M.h
        Ug[h:h + N[0], h:h + n1, h:h + N[2]] = np.moveaxis(U, 0, -1)
        pg[h:h + N[0], h:h + n1, h:h + N[2]] = np.moveaxis(p, 0, -1)
        Ug, pg = O.bc_apply(M, Ug, bc["U"]), O.bc_apply(M, pg, bc["p"])
        U = np.ascontiguousarray(np.moveaxis(Ug[h:h + N[0], h:h + n1, h:h + N[2]], -1, 0))
        p = np.ascontiguousarray(np.moveaxis(pg[h:h + N[0], h:h + n1, h:h + N[2]], -1, 0))
    else:
        U = rng.standard_normal((3,) + M.N)
        p = rng.standard_normal((1,) + M.N)
        Ug, pg = M.to_ghosted(U), M.to_ghosted(p)
    dt = 0.125
    with tempfile.TemporaryDirectory() as td:
        case = os.path.join(td, "case")
        O.write_case(case, M, bc)
        Ug.tofile(os.path.join(td, "U.bin"))
        pg.tofile(os.path.join(td, "p.bin"))
        out = os.path.join(td, "out")
        os.makedirs(out)
        import subprocess
        subprocess.run([O.REF_BIN, "ensight", case, "2", repr(dt), os.path.join(td, "U.bin"), os.path.join(td, "p.bin"),
                        out, "-m", str(M.m)], check=True, stdout=subprocess.DEVNULL)
        geo = O.ensight_parse(os.path.join(out, "geom.p0000.geo"), "geo")
        dat = {k: O.ensight_parse(os.path.join(out, "%s.0000.00002.dat" % k), "dat") for k in ("U", "p")}
        case_text = open(os.path.join(out, "fd.p0000.case")).read()
        restart_text = open(os.path.join(out, "restart.p.0000.case")).read()
    np.savez_compressed(os.path.join(HERE, name), N=np.array(N), L=np.array(L), origin=np.array(origin),
                        walls=np.array(int(walls)), U=U, p=p, times=np.array([0.0, dt]),
                        geo_lines=np.array(geo["lines"]), geo_dims=geo["dims"], geo_coords=geo["coords"],
                        geo_size=np.array(geo["size"]), dat_lines=np.array(dat["U"]["lines"]),
                        U_values=dat["U"]["values"], p_values=dat["p"]["values"], case_text=np.array(case_text),
                        restart_text=np.array(restart_text))


def ops2_case(name, N, L, seed):
    """the reference's div(tensor), div(symmTensor), div(scalar, tensor), laplacian(Field nu, .)"""
    M = O.Mesh(N, L=L)
    rng = np.random.default_rng(seed)
    ins = {"T": rng.standard_normal((9,) + M.N), "S": rng.standard_normal((6,) + M.N),
           "s": rng.standard_normal((1,) + M.N), "nu": 0.5 + rng.random((1,) + M.N),
           "U": rng.standard_normal((3,) + M.N)}
    out = O.ref_ops2(M, *(M.to_ghosted(ins[k]) for k in ("T", "S", "s", "nu", "U")))
    np.savez_compressed(os.path.join(HERE, name), N=np.array(N), L=np.array(L), **ins,
                        **{"out_" + k: M.interior(v) for k, v in out.items()})


def im_case(name, N, L, seed, mu, c, tol, max_its, m=6):
    """the reference's im::laplacian(mu, x) (coefficients, deferred-correction
    source), ap -= c, and (M == f).solve(tol, max_its) on x, stencil order m"""
    M = O.Mesh(N, L=L, m=m)
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((1,) + M.N)
    f = rng.standard_normal((1,) + M.N)
    out = O.ref_im(M, mu, c, M.to_ghosted(x), M.to_ghosted(f), tol, max_its)
    h = M.h
    inner = (slice(h, h + N[0]), slice(h, h + N[1]), slice(h, h + N[2]))
    np.savez_compressed(os.path.join(HERE, name), N=np.array(N), L=np.array(L), m=np.array(m), mu=np.array(mu),
                        c=np.array(c),
                        tol=np.array(tol), max_its=np.array(max_its), x=x, f=f,
                        al=np.stack([a[inner] for a in out["al"]]), ap=out["ap"][inner], src=out["src"][inner],
                        x_solved=out["x"][inner][None], res=np.array(out["res"]))


CASES = {
    "ops_10x8x6.npz": lambda n: ops_case(n, (10, 8, 6), (2 * np.pi, 2.0, 3.0), 7, 0.01),
    "ops_16x12x8_m4.npz": lambda n: ops_case(n, (16, 12, 8), (2 * np.pi,) * 3, 8, 0.02, m=4),
    "ops_hypz_12x10x16.npz": lambda n: ops_case(n, (12, 10, 16), (2 * np.pi, 2 * np.pi, 1.0), 29, 0.02,
                                                hyperbolic_z=(0.03, 0.03)),
    "tg_12_classical.npz": lambda n: run_case(n, (12, 12, 12), "ns", "classical", 6, 0.05, 1 / 1600, 0.0),
    "tg_12_literal.npz": lambda n: run_case(n, (12, 12, 12), "ns", "literal", 6, 0.05, 1 / 1600, 0.0),
    "ot_12_classical.npz": lambda n: run_case(n, (12, 12, 12), "mhd", "classical", 4, 0.01, 1e-3, 1e-3),
    "ot_12_literal.npz": lambda n: run_case(n, (12, 12, 12), "mhd", "literal", 4, 0.01, 1e-3, 1e-3),
    "tg_12_shear.npz": lambda n: run_case(n, (12, 12, 12), "ns", "shear", 6, 0.05, 1 / 1600, 0.0),
    "ot_12_shear.npz": lambda n: run_case(n, (12, 12, 12), "mhd", "shear", 4, 0.01, 1e-3, 1e-3),
    "shear_walls_12x10x8.npz": lambda n: shear_case(n, (12, 10, 8), (2 * np.pi, 2 * np.pi, np.pi), 6, 0.01, 1e-2),
    "wc_tg_12.npz": lambda n: wc_tg_case(n, (12, 12, 12), 5, 0.02, 1 / 1600),
    "wc_shear_12x8x16.npz": lambda n: wc_shear_case(n, (12, 8, 16), 4),
    "ops2_7x6x5.npz": lambda n: ops2_case(n, (7, 6, 5), (2.0, 1.5, 3.0), 13),
    "ensight_7x5x6.npz": lambda n: ensight_case(n, (7, 5, 6), (2.0, 1.5, 3.0), (0.5, -1.0, 0.25), 11),
    "ensight_walls_6x8x5.npz": lambda n: ensight_case(n, (6, 8, 5), (1.0, 2.0, 1.5), (0.0, 0.0, 0.0), 12, True),
    "im_7x6x8.npz": lambda n: im_case(n, (7, 6, 8), (2.0, 1.5, 3.0), 17, 0.7, 6.0, 1e-14, 400),
    "im_9x5x6_m4.npz": lambda n: im_case(n, (9, 5, 6), (1.5, 1.0, 2.5), 23, 0.35, 4.0, 1e-14, 600, m=4),
}


def main():
    if not O.ref_available():
        raise SystemExit("build the reference first: make -C oracle ref")
    for name in sys.argv[1:] or CASES:
        CASES[name](name)
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
