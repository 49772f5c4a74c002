"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs oracle/_ref/nova_ref -- the reference's own sources (src/ex, src/poisson,
src/BC, src/Field, app/TG_Piosson/RKLoop.H, app/OT_Poisson/UEqn.H + BEqn.H,
the compressible app/TG and app/shearLayerWC loop bodies)
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


def ops_case(name, N, L, seed, nu, m=6):
    M = O.Mesh(N, L=L, m=m)
    rng = np.random.default_rng(seed)
    U = rng.standard_normal((3,) + M.N)
    s = rng.standard_normal((1,) + M.N)
    out = O.ref_ops(M, M.to_ghosted(U), M.to_ghosted(s), nu)
    res = {"N": np.array(N), "L": np.array(L), "m": np.array(m), "nu": np.array(nu), "U": U, "s": s}
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


CASES = {
    "ops_10x8x6.npz": lambda n: ops_case(n, (10, 8, 6), (2 * np.pi, 2.0, 3.0), 7, 0.01),
    "ops_16x12x8_m4.npz": lambda n: ops_case(n, (16, 12, 8), (2 * np.pi,) * 3, 8, 0.02, m=4),
    "tg_12_classical.npz": lambda n: run_case(n, (12, 12, 12), "ns", "classical", 6, 0.05, 1 / 1600, 0.0),
    "tg_12_literal.npz": lambda n: run_case(n, (12, 12, 12), "ns", "literal", 6, 0.05, 1 / 1600, 0.0),
    "ot_12_classical.npz": lambda n: run_case(n, (12, 12, 12), "mhd", "classical", 4, 0.01, 1e-3, 1e-3),
    "ot_12_literal.npz": lambda n: run_case(n, (12, 12, 12), "mhd", "literal", 4, 0.01, 1e-3, 1e-3),
    "wc_tg_12.npz": lambda n: wc_tg_case(n, (12, 12, 12), 5, 0.02, 1 / 1600),
    "wc_shear_12x8x16.npz": lambda n: wc_shear_case(n, (12, 8, 16), 4),
}


def main():
    if not O.ref_available():
        raise SystemExit("build the reference first: make -C oracle ref")
    for name in sys.argv[1:] or CASES:
        CASES[name](name)
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
