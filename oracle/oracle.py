"""TEST INFRASTRUCTURE ONLY -- Python access to the CPU oracle.

Loads ``oracle/libnova_oracle.so`` (the C restatement of the reference's
explicit time advance, see ``nova_oracle.h``) and, where it was built,
drives ``oracle/_ref/nova_ref`` (the reference's own sources compiled in place).
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module; the product path never does.

Layout helpers convert between the reference's ghosted array-of-structs
``Field<T>`` layout (``(n0, n1, n2, nc)``, z fastest, n = N + 1 + m;
src/Field/Field.h:82-85) and the unique-point component-major layout
``(nc, N0, N1, N2)`` used by the device library.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnova_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "nova_ref")

PERIODIC, NEUMANN, DIRICHLET = 0, 1, 2
# src/BC/BCenums.h:8
FACES = ("north", "south", "east", "west", "top", "bottom")
# history row columns (nova_oracle.h ORC_HIST_COLS)
HIST_COLS = 16


class RunDesc(C.Structure):
    _fields_ = [
        ("model", C.c_int), ("rk_mode", C.c_int), ("nsteps", C.c_int), ("diag_every", C.c_int),
        ("dt", C.c_double), ("nu", C.c_double), ("eta", C.c_double),
        ("bcU_type", C.c_int * 18), ("bcU_val", C.c_double * 18),
        ("bcp_type", C.c_int * 6), ("bcp_val", C.c_double * 6),
        ("bcB_type", C.c_int * 18), ("bcB_val", C.c_double * 18),
        ("bcpB_type", C.c_int * 6), ("bcpB_val", C.c_double * 6),
    ]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "libnova_oracle.so"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
        ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
        L.orc_mesh_new.restype = C.c_void_p
        L.orc_mesh_new.argtypes = [ip, dp, dp, C.c_int, C.c_int, C.c_double, C.c_double]
        L.orc_mesh_free.argtypes = [C.c_void_p]
        L.orc_mesh_dims.argtypes = [C.c_void_p, ip]
        L.orc_mesh_metrics.argtypes = [C.c_void_p, dp, dp]
        L.orc_bc_apply.argtypes = [C.c_void_p, dp, C.c_int, ip, dp]
        L.orc_grad_s.argtypes = [C.c_void_p, dp, dp]
        L.orc_grad_v.argtypes = [C.c_void_p, dp, dp]
        L.orc_curl.argtypes = [C.c_void_p, dp, dp]
        L.orc_div_v.argtypes = [C.c_void_p, dp, dp]
        L.orc_div_vf.argtypes = [C.c_void_p, dp, dp, C.c_int, dp]
        L.orc_lap.argtypes = [C.c_void_p, C.c_double, dp, C.c_int, dp]
        L.orc_div_t.argtypes = [C.c_void_p, dp, C.c_int, dp]
        L.orc_div_sT.argtypes = [C.c_void_p, dp, dp, dp]
        L.orc_lap_f.argtypes = [C.c_void_p, dp, dp, C.c_int, dp]
        L.orc_maximum.restype = C.c_double
        L.orc_maximum.argtypes = [C.c_void_p, dp]
        L.orc_poisson_solve.argtypes = [C.c_void_p, dp, dp]
        L.orc_poisson_k2.argtypes = [C.c_void_p, dp]
        L.orc_run.restype = C.c_int
        L.orc_run.argtypes = [C.c_void_p, C.POINTER(RunDesc), dp, dp, dp, dp, dp]
        L.orc_diag_row.restype = None
        L.orc_diag_row.argtypes = [C.c_void_p, C.POINTER(RunDesc), C.c_int, C.c_double, dp, C.c_void_p, dp]
        _lib = L
    return _lib


class Mesh:
    """Reference Mesh (src/Mesh/Mesh.cpp:24-179) for one rank."""

    def __init__(self, N, L=(2 * np.pi,) * 3, origin=(0.0, 0.0, 0.0), m=6, hyperbolic_z=None):
        self.N = tuple(int(v) for v in N)
        self.L = tuple(float(v) for v in L)
        self.origin = tuple(float(v) for v in origin)
        self.m = int(m)
        self.h = self.m // 2
        hz = hyperbolic_z is not None
        s1, s2 = hyperbolic_z if hz else (0.0, 0.0)
        self.hyperbolic_z = (float(s1), float(s2)) if hz else None
        self._p = lib().orc_mesh_new(np.array(self.N, np.int32), np.array(self.L), np.array(self.origin),
                                     self.m, int(hz), float(s1), float(s2))
        if not self._p:
            raise ValueError("invalid mesh")
        n = np.zeros(3, np.int32)
        lib().orc_mesh_dims(self._p, n)
        self.n = tuple(int(v) for v in n)
        self.dzdxi = np.zeros(self.n[2])
        self.d2zdxi2 = np.zeros(self.n[2])
        lib().orc_mesh_metrics(self._p, self.dzdxi, self.d2zdxi2)

    def __del__(self):
        p = getattr(self, "_p", None)
        if p and _lib is not None:
            _lib.orc_mesh_free(p)
            self._p = None

    @property
    def d(self):
        return tuple(self.L[a] / self.N[a] for a in range(3))

    def zeros(self, nc):
        return np.zeros(self.n + (nc,), np.float64)

    # --- layout helpers -------------------------------------------------
    def to_ghosted(self, u):
        """(nc, N0, N1, N2) unique points -> ghosted AoS with periodic wrap in every slot."""
        u = np.asarray(u, np.float64)
        if u.ndim == 3:
            u = u[None]
        h = self.h
        idx = [(np.arange(self.n[a]) - h) % self.N[a] for a in range(3)]
        g = u[:, idx[0]][:, :, idx[1]][:, :, :, idx[2]]
        return np.ascontiguousarray(np.moveaxis(g, 0, -1))

    def unique(self, g):
        """ghosted AoS -> (nc, N0, N1, N2) unique interior points."""
        h = self.h
        N = self.N
        u = g[h:h + N[0], h:h + N[1], h:h + N[2]]
        return np.ascontiguousarray(np.moveaxis(u, -1, 0))

    def interior(self, g):
        """ghosted AoS -> (nc, N0+1, N1+1, N2+1) incl. the duplicate node."""
        h = self.h
        N = self.N
        u = g[h:h + N[0] + 1, h:h + N[1] + 1, h:h + N[2] + 1]
        return np.ascontiguousarray(np.moveaxis(u, -1, 0))

    def coords(self):
        """unique-point coordinates x_i = origin + i*d (uniform mesh)."""
        return [self.origin[a] + np.arange(self.N[a]) * self.d[a] for a in range(3)]


def bc_arrays(nc, spec=None):
    """spec: dict face -> (type, val) or per-comp list; default all periodic."""
    t = np.zeros(6 * nc, np.int32)
    v = np.zeros(6 * nc, np.float64)
    if spec:
        for c in range(nc):
            for f, face in enumerate(FACES):
                if face in spec:
                    typ, val = spec[face][c] if isinstance(spec[face], list) else spec[face]
                    t[f + 6 * c] = typ
                    v[f + 6 * c] = val
    return t, v


def bc_apply(mesh, g, spec=None):
    nc = g.shape[-1]
    t, v = bc_arrays(nc, spec)
    g = np.ascontiguousarray(g)
    lib().orc_bc_apply(mesh._p, g, nc, t, v)
    return g


def _op(fn, mesh, out_nc, *args):
    out = mesh.zeros(out_nc)
    fn(mesh._p, *args, out)
    return out


def grad_s(mesh, s):
    return _op(lib().orc_grad_s, mesh, 3, np.ascontiguousarray(s))


def grad_v(mesh, U):
    return _op(lib().orc_grad_v, mesh, 9, np.ascontiguousarray(U))


def curl(mesh, U):
    return _op(lib().orc_curl, mesh, 3, np.ascontiguousarray(U))


def div_v(mesh, U):
    return _op(lib().orc_div_v, mesh, 1, np.ascontiguousarray(U))


def div_vf(mesh, U, f):
    nc = f.shape[-1]
    out = mesh.zeros(nc)
    lib().orc_div_vf(mesh._p, np.ascontiguousarray(U), np.ascontiguousarray(f), nc, out)
    return out


def lap(mesh, nu, f):
    nc = f.shape[-1]
    out = mesh.zeros(nc)
    lib().orc_lap(mesh._p, float(nu), np.ascontiguousarray(f), nc, out)
    return out


def div_t(mesh, T):
    """ex::div(Field<tensor>) (9 components) or ex::div(Field<symmTensor>) (6)."""
    nc = T.shape[-1]
    out = mesh.zeros(3)
    lib().orc_div_t(mesh._p, np.ascontiguousarray(T), int(nc == 6), out)
    return out


def div_sT(mesh, s, T):
    """ex::div(Field<scalar>, Field<tensor>)."""
    out = mesh.zeros(3)
    lib().orc_div_sT(mesh._p, np.ascontiguousarray(s), np.ascontiguousarray(T), out)
    return out


def lap_f(mesh, nu, f):
    """ex::laplacian(Field<scalar> nu, Field<T>)."""
    nc = f.shape[-1]
    out = mesh.zeros(nc)
    lib().orc_lap_f(mesh._p, np.ascontiguousarray(nu), np.ascontiguousarray(f), nc, out)
    return out


def maximum(mesh, s):
    return lib().orc_maximum(mesh._p, np.ascontiguousarray(s))


def poisson_solve(mesh, rhs, p=None):
    p = mesh.zeros(1) if p is None else np.ascontiguousarray(p)
    lib().orc_poisson_solve(mesh._p, np.ascontiguousarray(rhs), p)
    return p


def poisson_k2(mesh):
    k2 = np.zeros(int(np.prod(mesh.N)))
    lib().orc_poisson_k2(mesh._p, k2)
    return k2.reshape(mesh.N[2], mesh.N[1], mesh.N[0])  # [k, j, i]


def run(mesh, U, B=None, *, model="ns", rk_mode="classical", nsteps=1, dt=0.01, nu=0.0, eta=0.0,
        diag_every=1, bcU=None, bcp=None, bcB=None, bcpB=None):
    """Advance ghosted U (and B) in place by nsteps with the restated loop bodies.
    rk_mode: "literal", "classical" or "shear" (app/shearLayer/UEqn.H).
    Returns (U, B, p, pB, hist[nsteps, HIST_COLS])."""
    rd = RunDesc()
    rd.model = 1 if model == "mhd" else 0
    rd.rk_mode = {"literal": 0, "classical": 1, "shear": 2}[rk_mode]
    rd.nsteps = nsteps
    rd.diag_every = diag_every
    rd.dt, rd.nu, rd.eta = dt, nu, eta
    for name, nc, spec in (("bcU", 3, bcU), ("bcp", 1, bcp), ("bcB", 3, bcB), ("bcpB", 1, bcpB)):
        t, v = bc_arrays(nc, spec)
        getattr(rd, name + "_type")[:] = list(t)
        getattr(rd, name + "_val")[:] = list(v)
    U = np.ascontiguousarray(U, np.float64).copy()
    B = mesh.zeros(3) if B is None else np.ascontiguousarray(B, np.float64).copy()
    p = mesh.zeros(1)
    pB = mesh.zeros(1)
    hist = np.zeros((nsteps, HIST_COLS))
    lib().orc_bc_apply(mesh._p, U, 3, *bc_arrays(3, bcU))
    if rd.model == 1:
        lib().orc_bc_apply(mesh._p, B, 3, *bc_arrays(3, bcB))
    rc = lib().orc_run(mesh._p, C.byref(rd), U, B, p, pB, hist)
    if rc != 0:
        raise RuntimeError("orc_run failed")
    return U, B, p, pB, hist


def diag_row(mesh, U, B=None, *, model="ns", dt=0.01, nu=0.0, eta=0.0, step=0, t=0.0):
    """One history row (nova_oracle.h ORC_HIST_COLS) of ghosted U (and B for "mhd")."""
    rd = RunDesc()
    rd.model = 1 if model == "mhd" else 0
    rd.dt, rd.nu, rd.eta = dt, nu, eta
    U = np.ascontiguousarray(U, np.float64)
    Bc = None if B is None else np.ascontiguousarray(B, np.float64)
    row = np.zeros(HIST_COLS)
    lib().orc_diag_row(mesh._p, C.byref(rd), int(step), float(t), U, None if Bc is None else Bc.ctypes.data, row)
    return row


# ------------------------------------------------------ reference in place --

def ref_available():
    return os.path.exists(REF_BIN)


def write_case(dirname, mesh, bc=None):
    """Write the reference's `mesh` and BC files (Mesh.cpp:38-62, Field.hxx:519-547)."""
    os.makedirs(dirname, exist_ok=True)
    with open(os.path.join(dirname, "mesh"), "w") as f:
        f.write("origin: %.17g %.17g %.17g\n" % mesh.origin)
        f.write("N: %d %d %d\n" % mesh.N)
        f.write("L: %.17g %.17g %.17g\n" % mesh.L)
        if mesh.hyperbolic_z is not None:
            f.write("hypz: %.17g %.17g\n" % mesh.hyperbolic_z)
    bc = bc or {}
    for name, nc in (("U", 3), ("p", 1), ("B", 3), ("pB", 1), ("rho", 1), ("T", 1)):
        t, v = bc_arrays(nc, bc.get(name))
        with open(os.path.join(dirname, name + "BC"), "w") as f:
            for c in range(nc):
                for fi, face in enumerate(FACES):
                    typ = ("periodic", "neumann", "dirichlet")[t[fi + 6 * c]]
                    f.write("%s %s %.17g %d\n" % (face, typ, v[fi + 6 * c], c))


def ref_run(mesh, U, B=None, *, model="ns", rk_mode="classical", nsteps=1, dt=0.01, nu=0.0, eta=0.0, bc=None):
    """Run the reference's own loop bodies (oracle/_ref/nova_ref). Returns (U, B, p, pB, hist)."""
    with tempfile.TemporaryDirectory() as td:
        case = os.path.join(td, "case")
        write_case(case, mesh, bc)
        np.ascontiguousarray(U, np.float64).tofile(os.path.join(td, "U.bin"))
        bpath = "-"
        if B is not None:
            bpath = os.path.join(td, "B.bin")
            np.ascontiguousarray(B, np.float64).tofile(bpath)
        out = os.path.join(td, "out")
        subprocess.run([REF_BIN, "run", case, model, rk_mode, str(nsteps), repr(float(dt)), repr(float(nu)),
                        repr(float(eta)), os.path.join(td, "U.bin"), bpath, out, "-m", str(mesh.m)],
                       check=True, stdout=subprocess.DEVNULL)
        shp3 = mesh.n + (3,)
        shp1 = mesh.n + (1,)
        Uo = np.fromfile(out + "_U.bin").reshape(shp3)
        po = np.fromfile(out + "_p.bin").reshape(shp1)
        Bo = np.fromfile(out + "_B.bin").reshape(shp3) if model == "mhd" else None
        pBo = np.fromfile(out + "_pB.bin").reshape(shp1) if model == "mhd" else None
        hist = np.fromfile(out + "_hist.bin").reshape(nsteps, HIST_COLS)
    return Uo, Bo, po, pBo, hist


def ref_ops(mesh, U, s, nu):
    """Apply the reference's ex:: operators and poisson::solve once."""
    names = {"grad_s": 3, "div_v": 1, "div_vv": 3, "div_vs": 1, "lap_v": 3, "lap_s": 1, "curl": 3, "poisson": 1}
    with tempfile.TemporaryDirectory() as td:
        case = os.path.join(td, "case")
        write_case(case, mesh)
        np.ascontiguousarray(U, np.float64).tofile(os.path.join(td, "U.bin"))
        np.ascontiguousarray(s, np.float64).tofile(os.path.join(td, "s.bin"))
        out = os.path.join(td, "out")
        subprocess.run([REF_BIN, "ops", case, repr(float(nu)), os.path.join(td, "U.bin"),
                        os.path.join(td, "s.bin"), out, "-m", str(mesh.m)], check=True, stdout=subprocess.DEVNULL)
        return {k: np.fromfile("%s_%s.bin" % (out, k)).reshape(mesh.n + (nc,)) for k, nc in names.items()}


# ------------------------------------------------- compressible loop bodies --
# Restated with the pinned operators above and numpy point operations in the
# reference's expression order; fields are ghosted AoS arrays.

RK4W = (1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0)  # app/TG/TG.cpp:62, shearLayer.cpp:164


def wc_eos_k(c, rho0):
    """c*c/2.0/rho0 of app/shearLayerWC/pEqn.H:2."""
    return c * c / 2.0 / rho0


def _u_eqn(mesh, U, rho, p, T, dt, mu, gz, buoy, bcU):
    """app/TG/UEqn.H:1-38, app/shearLayerWC/UEqn.H:1-42 (buoyancy -(rho*T)*g)."""
    g = np.array([0.0, 0.0, gz])
    rhoUc = rho * U
    rhoUOld = rho * U
    for rk in range(4):
        e = -div_vf(mesh, rho * U, U)
        e = e - grad_s(mesh, p)
        e = e + lap(mesh, mu, U)
        if buoy:
            e = e - (rho * T) * g
        drhoU = dt * e
        rhoUc = rhoUc + RK4W[rk] * drhoU
        if rk < 3:
            U = rhoUOld / rho + (int(rk / 2) + 1) / 2.0 * (drhoU / rho)
        else:
            U = rhoUc / rho
        U = bc_apply(mesh, U, bcU)
    return U


def _rho_eqn(mesh, U, rho, dt, bcr):
    """app/TG/rhoEqn.H:1-37 (= app/shearLayerWC/rhoEqn.H)."""
    rhoOld = rho.copy()
    rhoc = rho.copy()
    for rk in range(4):
        drho = dt * (-div_v(mesh, rho * U))
        rhoc = rhoc + RK4W[rk] * drho
        rho = rhoOld + (int(rk / 2) + 1) / 2.0 * drho if rk < 3 else rhoc
        rho = bc_apply(mesh, rho, bcr)
    return rho


def _t_eqn(mesh, U, rho, T, dt, ka, bcT):
    """app/shearLayerWC/TEqn.H:1-38."""
    rhoTc = rho * T
    rhoTOld = rho * T
    for rk in range(4):
        drhoT = dt * (-div_vf(mesh, rho * U, T) + lap(mesh, ka, T))
        rhoTc = rhoTc + RK4W[rk] * drhoT
        if rk < 3:
            T = rhoTOld / rho + (int(rk / 2) + 1) / 2.0 * (drhoT / rho)
        else:
            T = rhoTc / rho
        T = bc_apply(mesh, T, bcT)
    return T


def wc_run(mesh, U, rho, p, T=None, *, order="shear", nsteps=1, dt=0.01, mu=0.0, ka=0.0, c=0.0, rho0=1.0,
           gz=0.0, bc=None):
    """The compressible time step on ghosted arrays.
    order "tg":    app/TG/TG.cpp:73-75, rhoEqn.H, pEqn.H (p = 50 rho^2), UEqn.H;
    order "shear": app/shearLayerWC/shearLayer.cpp:197-200, UEqn.H (with buoyancy),
                   rhoEqn.H, pEqn.H (p = c^2/(2 rho0) rho^2), TEqn.H.
    Returns (U, rho, p, T, hist[nsteps, HIST_COLS]) with hist rows (step, t, Ek, 0, max|div U|, 0, 0...)."""
    bc = bc or {}
    U = bc_apply(mesh, np.array(U, np.float64), bc.get("U"))
    rho = bc_apply(mesh, np.array(rho, np.float64), bc.get("rho"))
    p = bc_apply(mesh, np.array(p, np.float64), bc.get("p"))
    T = bc_apply(mesh, mesh.zeros(1) if T is None else np.array(T, np.float64), bc.get("T"))
    K = wc_eos_k(c, rho0)
    hist = np.zeros((nsteps, HIST_COLS))
    h, N = mesh.h, mesh.N
    for step in range(nsteps):
        if order == "tg":
            rho = _rho_eqn(mesh, U, rho, dt, bc.get("rho"))
            p = 50.0 * (rho * rho)
            U = _u_eqn(mesh, U, rho, p, T, dt, mu, gz, False, bc.get("U"))
        else:
            U = _u_eqn(mesh, U, rho, p, T, dt, mu, gz, True, bc.get("U"))
            rho = _rho_eqn(mesh, U, rho, dt, bc.get("rho"))
            p = (K * rho) * rho
            T = _t_eqn(mesh, U, rho, T, dt, ka, bc.get("T"))
        u = U[h:h + N[0], h:h + N[1], h:h + N[2]]
        ek = 0.0
        for v in (0.5 * (u[..., 0] * u[..., 0] + u[..., 1] * u[..., 1] + u[..., 2] * u[..., 2])).ravel():
            ek += v
        hist[step, :6] = (step + 1, (step + 1) * dt, ek / u[..., 0].size, 0.0, maximum(mesh, div_v(mesh, U)), 0.0)
    return U, rho, p, T, hist


def wc_hydrostatic(mesh, T, *, c, rho0, gz):
    """Initial p and rho of app/shearLayerWC/shearLayer.cpp:114-155 for a given T:
    pEqn.H on rho = rho0, the column integral of hydrostaticP.H:1-38 (from the
    top node down, T*dz*g_z*rho0, unique i and k, j including the duplicate
    node), rho = (p/K)^0.5.  Returns ghosted (p, rho)."""
    K = wc_eos_k(c, rho0)
    T = bc_apply(mesh, np.array(T, np.float64))
    rho = np.full(mesh.n + (1,), rho0)
    p = (K * rho) * rho
    h, n = mesh.h, mesh.n
    dz = mesh.L[2] / mesh.N[2]
    pHyd = mesh.zeros(1)
    col = T[h:n[0] - h - 1, h:n[1] - h, h:n[2] - h - 1, 0]
    terms = ((col * dz) * gz) * rho0
    pHyd[h:n[0] - h - 1, h:n[1] - h, h:n[2] - h - 1, 0] = np.cumsum(terms[..., ::-1], axis=-1)[..., ::-1]
    p = p + pHyd
    # std::pow(x, 0.5) (C pow, not numpy's sqrt shortcut for the exponent 0.5)
    q = p[h:n[0] - h, h:n[1] - h, h:n[2] - h] / K
    rho[h:n[0] - h, h:n[1] - h, h:n[2] - h] = np.array([math.pow(v, 0.5) for v in q.ravel()]).reshape(q.shape)
    return bc_apply(mesh, p), bc_apply(mesh, rho)


def ref_wc_run(mesh, U, rho, p, T=None, *, order="shear", nsteps=1, dt=0.01, mu=0.0, ka=0.0, c=0.0, rho0=1.0,
               gz=0.0, bc=None):
    """The reference's own compressible loop bodies (oracle/_ref/nova_ref wc)."""
    with tempfile.TemporaryDirectory() as td:
        case = os.path.join(td, "case")
        write_case(case, mesh, bc)
        paths = {}
        for name, a in (("U", U), ("rho", rho), ("p", p), ("T", T)):
            if a is None:
                paths[name] = "-"
                continue
            paths[name] = os.path.join(td, name + ".bin")
            np.ascontiguousarray(a, np.float64).tofile(paths[name])
        out = os.path.join(td, "out")
        subprocess.run([REF_BIN, "wc", case, order, str(nsteps)] + [repr(float(v)) for v in (dt, mu, ka, c, rho0, gz)]
                       + [paths["U"], paths["rho"], paths["p"], paths["T"], out, "-m", str(mesh.m)],
                       check=True, stdout=subprocess.DEVNULL)
        r = tuple(np.fromfile("%s_%s.bin" % (out, k)).reshape(mesh.n + (nc,))
                  for k, nc in (("U", 3), ("rho", 1), ("p", 1), ("T", 1)))
        hist = np.zeros((nsteps, HIST_COLS))
        hist[:, :6] = np.fromfile(out + "_hist.bin").reshape(nsteps, 6)
    return r + (hist,)


def ref_wc_init(mesh, T, *, c, rho0, gz):
    """The reference's weakly-compressible initialisation (oracle/_ref/nova_ref wcinit)."""
    with tempfile.TemporaryDirectory() as td:
        case = os.path.join(td, "case")
        write_case(case, mesh)
        np.ascontiguousarray(T, np.float64).tofile(os.path.join(td, "T.bin"))
        out = os.path.join(td, "out")
        subprocess.run([REF_BIN, "wcinit", case, repr(float(c)), repr(float(rho0)), repr(float(gz)),
                        os.path.join(td, "T.bin"), out, "-m", str(mesh.m)], check=True, stdout=subprocess.DEVNULL)
        return tuple(np.fromfile("%s_%s.bin" % (out, k)).reshape(mesh.n + (1,)) for k in ("p", "rho"))


def ref_ensight(mesh, U, p, *, nsteps, dt, outdir):
    """The reference's EnSight output (Mesh::write, Field<T>::write after each of
    nsteps steps) of ghosted U and p into outdir (oracle/_ref/nova_ref ensight)."""
    with tempfile.TemporaryDirectory() as td:
        case = os.path.join(td, "case")
        write_case(case, mesh)
        np.ascontiguousarray(U, np.float64).tofile(os.path.join(td, "U.bin"))
        np.ascontiguousarray(p, np.float64).tofile(os.path.join(td, "p.bin"))
        subprocess.run([REF_BIN, "ensight", case, str(nsteps), repr(float(dt)), os.path.join(td, "U.bin"),
                        os.path.join(td, "p.bin"), outdir, "-m", str(mesh.m)], check=True, stdout=subprocess.DEVNULL)


def ensight_parse(path, kind, n=None, nc=1):
    """EnSight Gold file -> dict of its content: header lines as text up to the
    first NUL, integers and float32 arrays.  kind "geo" or "dat"; n = nodes per axis."""
    b = open(path, "rb").read()
    text = lambda o: b[o:o + 80].split(b"\0")[0].decode()
    if kind == "geo":
        lines = [text(80 * i) for i in range(6)]
        o = 480
        part = int(np.frombuffer(b, np.int32, 1, o)[0])
        lines += [text(o + 4), text(o + 84)]
        o += 164
        dims = np.frombuffer(b, np.int32, 3, o)
        o += 12
        coords = np.frombuffer(b, np.float32, int(dims.sum()), o)
        return {"lines": lines, "part": part, "dims": dims.copy(), "coords": coords.copy(), "size": len(b)}
    lines = [text(0), text(80), text(164)]
    part = int(np.frombuffer(b, np.int32, 1, 160)[0])
    vals = np.frombuffer(b, np.float32, offset=244)
    return {"lines": lines, "part": part, "values": vals.copy(), "size": len(b)}


def ref_ops2(mesh, T, S, s, nu, U):
    """The reference's div(tensor), div(symmTensor), div(scalar, tensor),
    laplacian(Field nu, vector / scalar) on ghosted inputs (oracle/_ref/nova_ref ops2)."""
    names = {"div_t": 3, "div_st": 3, "div_sT": 3, "lap_f_v": 3, "lap_f_s": 1}
    with tempfile.TemporaryDirectory() as td:
        case = os.path.join(td, "case")
        write_case(case, mesh)
        paths = []
        for k, a in (("T", T), ("S", S), ("s", s), ("nu", nu), ("U", U)):
            paths.append(os.path.join(td, k + ".bin"))
            np.ascontiguousarray(a, np.float64).tofile(paths[-1])
        out = os.path.join(td, "out")
        subprocess.run([REF_BIN, "ops2", case] + paths + [out, "-m", str(mesh.m)], check=True,
                       stdout=subprocess.DEVNULL)
        return {k: np.fromfile("%s_%s.bin" % (out, k)).reshape(mesh.n + (nc,)) for k, nc in names.items()}


# ------------------------------------------------------- implicit operators --

def im_laplacian(mesh, mu, xg):
    """im::laplacian(mu, x) (src/im/laplacian/laplacian.hxx:24-58) for a ghosted
    scalar x (periodic images filled): the 7-point coefficients al[0..5] (the
    neighbours j+1, j-1, i+1, i-1, k+1, k-1) and ap on the interior nodes, and
    the source of the deferred correction (src/im/fdMatrix/fdMatrix.hxx:201-225)
    src = -ex::laplacian(mu, x) + sum_l al_l x(neighbour l) + ap x, summed in that
    order.  Ghost entries are 0, as in the reference's pooled fields."""
    n, h = mesh.n, mesh.h
    dx, dy, dz = mesh.d
    x = xg[..., 0] if xg.ndim == 4 else xg
    I, J, K = slice(h, n[0] - h), slice(h, n[1] - h), slice(h, n[2] - h)
    al = np.zeros((6,) + n)
    ap = np.zeros(n)
    src = np.zeros(n)
    for l, d in ((0, dy), (1, dy), (2, dx), (3, dx), (4, dz), (5, dz)):
        al[l][I, J, K] = mu / (d * d)
    ap[I, J, K] = -2.0 * mu / (dx * dx) - 2.0 * mu / (dy * dy) - 2.0 * mu / (dz * dz)
    hoa = lap(mesh, mu, x[..., None])[..., 0]

    def sh(di, dj, dk):
        return x[h + di:n[0] - h + di, h + dj:n[1] - h + dj, h + dk:n[2] - h + dk]
    c = [a[I, J, K] for a in al]
    src[I, J, K] = (((((((-hoa[I, J, K] + c[0] * sh(0, 1, 0)) + c[1] * sh(0, -1, 0)) + c[2] * sh(1, 0, 0)) +
                        c[3] * sh(-1, 0, 0)) + c[4] * sh(0, 0, 1)) + c[5] * sh(0, 0, -1)) + ap[I, J, K] * sh(0, 0, 0))
    return al, ap, src


def fdm_residual(mesh, al, ap, src, xg):
    """fdMatrix::residual (fdMatrix.hxx:249-290) for a scalar: the RMS of
    src - sum_l al_l x(neighbour l) - ap x over the interior nodes, the duplicate
    periodic nodes included."""
    n, h = mesh.n, mesh.h
    x = xg[..., 0] if xg.ndim == 4 else xg
    I, J, K = slice(h, n[0] - h), slice(h, n[1] - h), slice(h, n[2] - h)

    def sh(di, dj, dk):
        return x[h + di:n[0] - h + di, h + dj:n[1] - h + dj, h + dk:n[2] - h + dk]
    r = ((((((src[I, J, K] - al[0][I, J, K] * sh(0, 1, 0)) - al[1][I, J, K] * sh(0, -1, 0)) -
            al[2][I, J, K] * sh(1, 0, 0)) - al[3][I, J, K] * sh(-1, 0, 0)) - al[4][I, J, K] * sh(0, 0, 1)) -
         al[5][I, J, K] * sh(0, 0, -1)) - ap[I, J, K] * sh(0, 0, 0)
    cnt = r.size
    return float(np.sqrt(float(np.sum(r * r)) / cnt))


def _tdma(a, b, c, d):
    """tools::tdma (src/Tools/Tools.cpp:43-62), Python floats."""
    m = len(a)
    cp, dp, x = [0.0] * m, [0.0] * m, [0.0] * m
    cp[0] = c[0] / b[0]
    dp[0] = d[0] / b[0]
    for i in range(1, m):
        cp[i] = c[i] / (b[i] - a[i] * cp[i - 1])
        dp[i] = (d[i] - a[i] * dp[i - 1]) / (b[i] - a[i] * cp[i - 1])
    x[m - 1] = dp[m - 1]
    for i in range(m - 2, -1, -1):
        x[i] = dp[i] - cp[i] * x[i + 1]
    return x


def fdm_solve(mesh, al, ap, src, xg, tol, max_its):
    """fdMatrix::solve(tol, maxIts) (fdMatrix.hxx:59-198) for a scalar on a
    periodic mesh, in the reference's order: per iteration the residual check,
    then line sweeps along j (lines in i-then-k order), along i, along k, each
    line a tridiagonal solve over the whole ghosted line with the ghost rows and
    the last (duplicate) node held at their current values, Gauss-Seidel across
    lines; then the periodic ghost refresh.  Small meshes only (Python loops).
    Returns (x ghosted, iterations, residual)."""
    n, h = mesh.n, mesh.h
    x = (xg[..., 0] if xg.ndim == 4 else xg).copy()
    its, res = 0, fdm_residual(mesh, al, ap, src, x)
    while its < max_its:
        res = fdm_residual(mesh, al, ap, src, x)
        if not res > tol:
            break
        its += 1
        for axis in (1, 0, 2):
            m = n[axis]
            # sub- and super-diagonal coefficients (S, N), (W, E), (B, T) and the
            # off-line neighbours moved to the right-hand side, (l, di, dj, dk), in the
            # reference's order (fdMatrix.hxx:103-108, 138-143, 173-178)
            lo, hi = {0: (3, 2), 1: (1, 0), 2: (5, 4)}[axis]
            others = [ax for ax in (0, 1, 2) if ax != axis]
            offs = {0: ((0, 0, 1, 0), (1, 0, -1, 0), (4, 0, 0, 1), (5, 0, 0, -1)),
                    1: ((2, 1, 0, 0), (3, -1, 0, 0), (4, 0, 0, 1), (5, 0, 0, -1)),
                    2: ((2, 1, 0, 0), (3, -1, 0, 0), (0, 0, 1, 0), (1, 0, -1, 0))}[axis]
            for p in range(h, n[others[0]] - h):
                for q in range(h, n[others[1]] - h):
                    a, b, c, d = [0.0] * m, [0.0] * m, [0.0] * m, [0.0] * m
                    for t in range(m):
                        idx = [0, 0, 0]
                        idx[axis], idx[others[0]], idx[others[1]] = t, p, q
                        i, j, k = idx
                        if t < h or t >= m - h - 1:
                            a[t], b[t], c[t], d[t] = 0.0, 1.0, 0.0, float(x[i, j, k])
                            continue
                        a[t], b[t], c[t] = float(al[lo][i, j, k]), float(ap[i, j, k]), float(al[hi][i, j, k])
                        v = float(src[i, j, k])
                        for l, di, dj, dk in offs:
                            v = v - float(al[l][i, j, k]) * float(x[i + di, j + dj, k + dk])
                        d[t] = v
                    sol = _tdma(a, b, c, d)
                    for t in range(h, m - h):
                        idx = [0, 0, 0]
                        idx[axis], idx[others[0]], idx[others[1]] = t, p, q
                        x[tuple(idx)] = sol[t]
        x = bc_apply(mesh, x[..., None])[..., 0]
    return x, its, res


def ref_im(mesh, mu, c, xg, fg, tol, max_its):
    """The reference's im::laplacian(mu, x), ap -= c, (M == f).solve(tol, max_its)
    (oracle/_ref/nova_ref im): coefficients and source as built, x after the
    solve, the residual after it and the solve's wall seconds."""
    with tempfile.TemporaryDirectory() as td:
        case = os.path.join(td, "case")
        write_case(case, mesh)
        px, pf = os.path.join(td, "x.bin"), os.path.join(td, "f.bin")
        np.ascontiguousarray(xg, np.float64).tofile(px)
        np.ascontiguousarray(fg, np.float64).tofile(pf)
        out = os.path.join(td, "out")
        subprocess.run([REF_BIN, "im", case, repr(float(mu)), repr(float(c)), px, pf, repr(float(tol)),
                        str(int(max_its)), out, "-m", str(mesh.m)], check=True, stdout=subprocess.DEVNULL)
        rd = lambda k: np.fromfile("%s_%s.bin" % (out, k)).reshape(mesh.n)
        return {"al": np.stack([rd("al%d" % l) for l in range(6)]), "ap": rd("ap"), "src": rd("src"),
                "x": rd("x"), "res": float(open(out + "_res.txt").read()),
                "solve_s": float(open(out + "_time.txt").read())}


# ------------------------------------------------------------- initial data --

def ic_taylor_green(mesh):
    """u = sin x cos y cos z, v = -cos x sin y cos z, w = 0 on the unique points."""
    x, y, z = mesh.coords()
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    return np.stack([np.sin(X) * np.cos(Y) * np.cos(Z), -np.cos(X) * np.sin(Y) * np.cos(Z), np.zeros_like(X)])


def ic_orszag_tang(mesh):
    """u = (-2 sin y, 2 sin x, 0), B = (-2 sin 2y + sin z, 2 sin x + sin z, 0)."""
    x, y, z = mesh.coords()
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    U = np.stack([-2.0 * np.sin(Y), 2.0 * np.sin(X), np.zeros_like(X)])
    B = np.stack([-2.0 * np.sin(2.0 * Y) + np.sin(Z), 2.0 * np.sin(X) + np.sin(Z), np.zeros_like(X)])
    return U, B


def ic_mhd_jet(mesh, seed=1, noise=1e-3):
    """MHD jet (x, y in [-4, 4] about the axis, z periodic): u_z = 0.5 (1 - tanh((r - 1)/0.1)),
    B_z = 0.5, B_theta = 0.2 r exp(-r^2), white noise of amplitude `noise` on u."""
    x, y, z = mesh.coords()
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    r = np.sqrt(X * X + Y * Y)
    zero = np.zeros_like(X)
    U = np.stack([zero, zero, 0.5 * (1.0 - np.tanh((r - 1.0) / 0.1))])
    U = U + noise * np.random.default_rng(seed).standard_normal(U.shape)
    e = 0.2 * np.exp(-r * r)  # B_theta / r
    B = np.stack([-e * Y, e * X, np.full_like(X, 0.5)])
    return U, B


def ic_temporal_shear(mesh, seed=0, noise=1e-3, walls=True, delta=28.0):
    """Temporal shear layer: u = tanh(delta (y - pi)), v = w = 0, plus seed-`seed`
    Gaussian noise of amplitude `noise` on every component, on the stored nodes
    (N1 + 1 rows when y is bounded by walls)."""
    x, y, z = mesh.coords()
    if walls:
        y = mesh.origin[1] + np.arange(mesh.N[1] + 1) * mesh.d[1]
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    zero = np.zeros_like(X)
    U = np.stack([np.tanh(delta * (Y - np.pi)), zero, zero])
    return U + noise * np.random.default_rng(seed).standard_normal(U.shape)


def ghosted_from_stored(mesh, U, spec=None):
    """stored nodes (nc, N0, N1 + 1, N2) of a mesh with y walls -> the ghosted
    reference layout with the BCs of `spec` applied"""
    g = mesh.zeros(U.shape[0])
    h = mesh.h
    N = mesh.N
    g[h:h + N[0], h:h + N[1] + 1, h:h + N[2]] = np.moveaxis(U, 0, -1)
    return bc_apply(mesh, g, spec)


def stored_of(mesh, g):
    """ghosted -> the stored nodes of a mesh with y walls: (nc, N0, N1 + 1, N2)"""
    h = mesh.h
    u = g[h:h + mesh.N[0], h:h + mesh.N[1] + 1, h:h + mesh.N[2]]
    return np.ascontiguousarray(np.moveaxis(u, -1, 0))


def wc_shear_params(mach=0.1):
    """Constants of app/shearLayerWC/shearLayer.cpp:31-44 (Mach as a parameter)."""
    Re0, Ri0, Pr, rho0, c = 1967.0, 0.08, 7.0, 999.57, 0.0417
    u0 = c * mach
    h0, t0 = 0.2, 0.1
    mu = rho0 * u0 * h0 / Re0
    return dict(rho0=rho0, c=c, u0=u0, h0=h0, t0=t0, mu=mu, ka=mu / Pr, gz=-Ri0 * u0 * u0 / t0 / h0)


def ic_wc_shear(mesh, prm, seed=0):
    """U, T of shearLayer.cpp:116-135 on the unique points with z = -7.5 h0 + k dz,
    the reference's std::default_random_engine noise replaced by a seeded
    uniform(-1, 1) generator."""
    u0, h0, t0 = prm["u0"], prm["h0"], prm["t0"]
    x, _, z = mesh.coords()
    z = z - 7.5 * h0
    X, _, Z = np.meshgrid(x, np.zeros(mesh.N[1]), z, indexing="ij")
    rng = np.random.default_rng(seed)
    k0 = 2.0 * 3.1415926536 / (14.0 * h0 / 2.0)
    a, b = 0.005, 0.4177
    th, ch = np.tanh(2.0 * Z / h0), np.cosh(2.0 * Z / h0)
    U = np.zeros((3,) + mesh.N)
    U[0] = u0 / 2.0 * th + a * u0 / 2.0 / k0 * (-np.cos(2 * k0 * X) + 2.0 * b * np.cos(k0 * X)) * th / ch
    U[1] = a * u0 / 2.0 * rng.uniform(-1, 1, mesh.N) / ch / ch
    U[2] = a * u0 / 2.0 * rng.uniform(-1, 1, mesh.N) / ch / ch
    T = t0 / 2.0 * th + a * t0 / 2.0 * rng.uniform(-1, 1, mesh.N) / ch / ch
    return U, T[None]


def ic_tg_compressible(mesh):
    """app/TG/TG.cpp:38-56 on the unique points (x = -pi + i dx): U of Taylor-Green,
    p = 50 + (cos 2x + cos 2y)(cos 2z + 2)/16, rho = (p/50)^0.5."""
    pi = np.pi
    x, y, z = (c - pi for c in mesh.coords())
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    U = np.stack([np.sin(X) * np.cos(Y) * np.cos(Z), -np.cos(X) * np.sin(Y) * np.cos(Z), np.zeros_like(X)])
    p = 50 + 1.0 / 16.0 * (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2)
    return U, np.power(p / 50.0, 0.5)[None], p[None]


def cfl_dt(mesh, fields, cfl=0.3):
    """dt = cfl * min(d) / max(sum_c |f_c|) summed over the given fields (fixed from the IC)."""
    s = sum(np.abs(f).sum(axis=0) for f in fields)
    return cfl * min(mesh.d) / float(s.max())
