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
HIST_COLS = 6


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
        L.orc_maximum.restype = C.c_double
        L.orc_maximum.argtypes = [C.c_void_p, dp]
        L.orc_poisson_solve.argtypes = [C.c_void_p, dp, dp]
        L.orc_poisson_k2.argtypes = [C.c_void_p, dp]
        L.orc_run.restype = C.c_int
        L.orc_run.argtypes = [C.c_void_p, C.POINTER(RunDesc), dp, dp, dp, dp, dp]
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
    Returns (U, B, p, pB, hist[nsteps, 6])."""
    rd = RunDesc()
    rd.model = 1 if model == "mhd" else 0
    rd.rk_mode = 1 if rk_mode == "classical" else 0
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
    bc = bc or {}
    for name, nc in (("U", 3), ("p", 1), ("B", 3), ("pB", 1)):
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


def cfl_dt(mesh, fields, cfl=0.3):
    """dt = cfl * min(d) / max(sum_c |f_c|) summed over the given fields (fixed from the IC)."""
    s = sum(np.abs(f).sum(axis=0) for f in fields)
    return cfl * min(mesh.d) / float(s.max())
