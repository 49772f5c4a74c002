"""ctypes binding of libnova_b200 (include/nova_gpu.h) with the reference's names.

The reference is C++ (``Mesh``, ``Field<T>``, ``ex::grad/div/curl/laplacian``,
``poisson``, ``tools::maximum``); this module gives the same operations to
Python callers over the C ABI.  Everything here is a thin wrapper: every
computation runs in the CUDA library, and importing fails loudly if the
library has not been built.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libnova_b200.so")

OK, E_INVALID, E_CUDA, E_OOM, E_NONFINITE, E_TIMEOUT, E_UNSUPPORTED = range(7)
POISSON_FFT, POISSON_DCT = 0, 1
F64, F32SPLIT = 0, 1
PERIODIC, NEUMANN, DIRICHLET = 0, 1, 2
MODEL_NS, MODEL_MHD = 0, 1
RK_LITERAL, RK_CLASSICAL, RK_SHEARLAYER = 0, 1, 2
# history row (nova_gpu.h NOVA_HIST_COLS): step, t, Ek, Em, max|div U|, max|div B|, omega, Jav,
# Jmax, epsilon, Umax, cfl_x, cfl_y, cfl_z, 1/2<|curl U|^2>, 1/2<|curl B|^2>
HIST_COLS = 16
HIST_NAMES = ("step", "t", "Ek", "Em", "max_div_U", "max_div_B", "omega", "Jav", "Jmax", "epsilon", "Umax",
              "cfl_x", "cfl_y", "cfl_z", "enstrophy_U", "enstrophy_B")
K_STAGE, K_DIV, K_FFT, K_CORRECT, K_DIAG, K_ADJ = range(6)
OBJ_EKIN_FINAL, OBJ_DISSIPATION_WINDOW, OBJ_ETOT_FINAL, OBJ_LINEAR_FINAL = 0, 1, 2, 3
WC_TG, WC_SHEAR = 0, 1
STATUS_NAMES = {0: "NOVA_OK", 1: "NOVA_E_INVALID", 2: "NOVA_E_CUDA", 3: "NOVA_E_OOM", 4: "NOVA_E_NONFINITE",
                5: "NOVA_E_TIMEOUT", 6: "NOVA_E_UNSUPPORTED"}

# every symbol declared in include/nova_gpu.h
EXPORTS = (
    "nova_create", "nova_destroy", "nova_last_error", "nova_set_stream", "nova_synchronize", "nova_mesh_local_n",
    "nova_mesh_metrics", "nova_field_create", "nova_field_destroy", "nova_field_set_bc", "nova_field_get_bc",
    "nova_field_upload", "nova_field_download",
    "nova_field_upload_soa", "nova_field_download_soa", "nova_field_copy_from_device", "nova_field_copy_to_device",
    "nova_grad_s", "nova_grad_v", "nova_curl", "nova_div_v", "nova_div_vf", "nova_laplacian", "nova_poisson_solve",
    "nova_div_t", "nova_div_st", "nova_laplacian_f",
    "nova_field_maxabs", "nova_field_maxabs_noalloc", "nova_advance", "nova_adjoint_grad", "nova_advance_wc",
    "nova_wc_hydrostatic", "nova_checkpoint_write", "nova_checkpoint_read", "nova_ensight_write_geometry",
    "nova_ensight_write_case", "nova_ensight_write_host", "nova_ensight_read_host", "nova_ensight_write_field",
    "nova_ensight_read_field", "nova_profile_enable", "nova_profile_read",
    "nova_launch_count", "nova_im_laplacian", "nova_fdm_add", "nova_fdm_mul", "nova_fdm_scale",
    "nova_fdm_add_source", "nova_fdm_add_diagonal", "nova_fdm_relax", "nova_fdm_set_reference",
    "nova_fdm_residual", "nova_fdm_solve", "nova_fdm_download", "nova_fdm_destroy",
)


class MeshDesc(C.Structure):
    _fields_ = [("N", C.c_int * 3), ("L", C.c_double * 3), ("origin", C.c_double * 3), ("m", C.c_int),
                ("hyperbolic_z", C.c_int), ("s1", C.c_double), ("s2", C.c_double), ("walls", C.c_int * 3)]


class BCDesc(C.Structure):
    _fields_ = [("type", C.c_int * 18), ("val", C.c_double * 18)]


class RunDesc(C.Structure):
    _fields_ = [("model", C.c_int), ("rk_mode", C.c_int), ("precision", C.c_int), ("diag_every", C.c_int),
                ("dt", C.c_double), ("nu", C.c_double), ("eta", C.c_double), ("t0", C.c_double),
                ("poisson", C.c_int), ("reserved", C.c_int)]


class AdjDesc(C.Structure):
    _fields_ = [("run", RunDesc), ("nsteps", C.c_int), ("checkpoint_every", C.c_int), ("objective", C.c_int),
                ("window_start", C.c_int), ("weight", C.c_void_p)]


class State(C.Structure):
    _fields_ = [("U", C.c_void_p), ("p", C.c_void_p), ("B", C.c_void_p), ("pB", C.c_void_p)]


class WcDesc(C.Structure):
    _fields_ = [("wc_case", C.c_int), ("diag_every", C.c_int), ("dt", C.c_double), ("mu", C.c_double),
                ("ka", C.c_double), ("eos_k", C.c_double), ("g", C.c_double * 3), ("t0", C.c_double)]


class WcState(C.Structure):
    _fields_ = [("U", C.c_void_p), ("rho", C.c_void_p), ("p", C.c_void_p), ("T", C.c_void_p)]


class NovaError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), msg))
        self.status = status


_lib = None


def load_library(path: str = LIB_PATH):
    """Load libnova_b200.so; raises if it is missing (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError("libnova_b200.so not built: run `python -m novaclone_b200.build` (%s)" % path)
    L = C.CDLL(path)
    vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
    sig = {
        "nova_create": [C.POINTER(MeshDesc), C.POINTER(C.c_void_p)],
        "nova_destroy": [vp],
        "nova_set_stream": [vp, vp],
        "nova_synchronize": [vp],
        "nova_mesh_local_n": [vp, ip],
        "nova_mesh_metrics": [vp, dp, dp],
        "nova_field_create": [vp, C.c_int, C.c_int, C.POINTER(C.c_void_p)],
        "nova_field_destroy": [vp, vp],
        "nova_field_set_bc": [vp, vp, C.POINTER(BCDesc)],
        "nova_field_get_bc": [vp, vp, C.POINTER(BCDesc)],
        "nova_field_upload": [vp, vp, dp, ip],
        "nova_field_download": [vp, vp, dp, ip, C.POINTER(BCDesc)],
        "nova_field_upload_soa": [vp, vp, dp],
        "nova_field_download_soa": [vp, vp, dp],
        "nova_field_copy_from_device": [vp, vp, vp],
        "nova_field_copy_to_device": [vp, vp, vp],
        "nova_grad_s": [vp, vp, vp],
        "nova_grad_v": [vp, vp, vp],
        "nova_curl": [vp, vp, vp],
        "nova_div_v": [vp, vp, vp],
        "nova_div_vf": [vp, vp, vp, vp],
        "nova_laplacian": [vp, C.c_double, vp, vp],
        "nova_poisson_solve": [vp, vp, vp],
        "nova_div_t": [vp, vp, vp],
        "nova_div_st": [vp, vp, vp, vp],
        "nova_laplacian_f": [vp, vp, vp, vp],
        "nova_field_maxabs": [vp, vp, dp],
        "nova_field_maxabs_noalloc": [vp, vp, dp],
        "nova_advance": [vp, C.POINTER(RunDesc), C.POINTER(State), C.c_int, dp],
        "nova_adjoint_grad": [vp, C.POINTER(AdjDesc), C.POINTER(State), vp, vp, dp],
        "nova_advance_wc": [vp, C.POINTER(WcDesc), C.POINTER(WcState), C.c_int, dp],
        "nova_wc_hydrostatic": [vp, C.POINTER(WcDesc), C.c_double, vp, vp, vp],
        "nova_ensight_write_geometry": [C.POINTER(MeshDesc), C.c_char_p],
        "nova_ensight_write_case": [C.c_char_p, C.c_int, dp],
        "nova_ensight_write_host": [C.POINTER(MeshDesc), dp, C.c_int, C.c_char_p, C.c_char_p, C.c_int],
        "nova_ensight_read_host": [C.POINTER(MeshDesc), dp, C.c_int, C.c_char_p, C.c_char_p, C.c_int],
        "nova_ensight_write_field": [vp, vp, C.c_char_p, C.c_char_p, C.c_int],
        "nova_ensight_read_field": [vp, vp, C.c_char_p, C.c_char_p, C.c_int],
        "nova_checkpoint_write": [vp, C.c_char_p, C.POINTER(State), C.c_double, C.c_longlong],
        "nova_checkpoint_read": [vp, C.c_char_p, C.POINTER(State), C.POINTER(C.c_double), C.POINTER(C.c_longlong)],
        "nova_profile_enable": [vp, C.c_int],
        "nova_profile_read": [vp, C.c_int, dp, C.POINTER(C.c_long), C.c_int],
        "nova_launch_count": [vp, C.POINTER(C.c_long), C.c_int],
        "nova_im_laplacian": [vp, C.c_double, vp, C.POINTER(C.c_void_p)],
        "nova_fdm_add": [vp, vp, C.c_double, vp],
        "nova_fdm_mul": [vp, vp, vp],
        "nova_fdm_scale": [vp, vp, C.c_double],
        "nova_fdm_add_source": [vp, vp, C.c_double, vp],
        "nova_fdm_add_diagonal": [vp, vp, C.c_double],
        "nova_fdm_relax": [vp, vp, C.c_double],
        "nova_fdm_set_reference": [vp, vp, C.c_int, C.c_int, C.c_int, C.c_double],
        "nova_fdm_residual": [vp, vp, dp],
        "nova_fdm_solve": [vp, vp, C.c_double, C.c_int, ip, dp],
        "nova_fdm_download": [vp, vp, dp],
        "nova_fdm_destroy": [vp],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    L.nova_last_error.argtypes = [vp]
    L.nova_last_error.restype = C.c_char_p
    _lib = L
    return L


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _iptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class Mesh:
    """A nova_ctx: the reference's Mesh for one GPU (src/Mesh/Mesh.cpp:24-179)."""

    def __init__(self, N, L=(2 * math.pi,) * 3, origin=(0.0, 0.0, 0.0), m=6, hyperbolic_z=None, walls=(0, 0, 0)):
        self.lib = load_library()
        d = MeshDesc()
        d.walls[:] = [int(v) for v in walls]
        d.N[:] = [int(v) for v in N]
        d.L[:] = [float(v) for v in L]
        d.origin[:] = [float(v) for v in origin]
        d.m = int(m)
        d.hyperbolic_z = int(hyperbolic_z is not None)
        d.s1, d.s2 = hyperbolic_z if hyperbolic_z is not None else (0.0, 0.0)
        h = C.c_void_p()
        st = self.lib.nova_create(C.byref(d), C.byref(h))
        if st != OK:
            raise NovaError(st, "nova_create")
        self.h = h
        self.N = tuple(int(v) for v in N)
        self.L = tuple(float(v) for v in L)
        self.origin = tuple(float(v) for v in origin)
        self.m = int(m)
        self.walls = tuple(int(v) for v in walls)
        # stored nodes per axis: N (periodic) or N + 1 (walls)
        self.shape = tuple(self.N[a] + self.walls[a] for a in range(3))
        n = np.zeros(3, np.int32)
        self.check(self.lib.nova_mesh_local_n(self.h, _iptr(n)))
        self.local_n = tuple(int(v) for v in n)

    def check(self, st, what=""):
        if st != OK:
            raise NovaError(st, self.lib.nova_last_error(self.h).decode() or what)

    def close(self):
        if getattr(self, "h", None):
            self.lib.nova_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def d(self):
        return tuple(self.L[a] / self.N[a] for a in range(3))

    def metrics(self):
        a = np.zeros(self.local_n[2])
        b = np.zeros(self.local_n[2])
        self.check(self.lib.nova_mesh_metrics(self.h, _dptr(a), _dptr(b)))
        return a, b

    def set_stream(self, stream_ptr):
        self.check(self.lib.nova_set_stream(self.h, C.c_void_p(stream_ptr)))

    def synchronize(self):
        self.check(self.lib.nova_synchronize(self.h))

    def profile(self, on=True):
        self.check(self.lib.nova_profile_enable(self.h, int(on)))

    def profile_read(self, cls, reset=False):
        ms = C.c_double()
        n = C.c_long()
        self.check(self.lib.nova_profile_read(self.h, cls, C.byref(ms), C.byref(n), int(reset)))
        return ms.value, n.value

    def launch_count(self, reset=False):
        n = C.c_long()
        self.check(self.lib.nova_launch_count(self.h, C.byref(n), int(reset)))
        return n.value


class Field:
    """Device field with ncomp components (Field<T>, src/Field/Field.h:56-157)."""

    def __init__(self, mesh: Mesh, ncomp: int, precision: int = F64):
        self.mesh = mesh
        self.nc = int(ncomp)
        self.precision = precision
        h = C.c_void_p()
        mesh.check(mesh.lib.nova_field_create(mesh.h, self.nc, precision, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None) and self.mesh.h:
            self.mesh.lib.nova_field_destroy(self.mesh.h, self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # reference Field<T>::ptr() layout
    def upload(self, aos):
        a = np.ascontiguousarray(aos, np.float64)
        if a.shape[:3] != self.mesh.local_n:
            raise ValueError("expected ghosted shape %s, got %s" % (self.mesh.local_n, a.shape))
        n = np.array(self.mesh.local_n, np.int32)
        self.mesh.check(self.mesh.lib.nova_field_upload(self.mesh.h, self.h, _dptr(a), _iptr(n)))
        return self

    def download(self, bc=None, out=None):
        shape = self.mesh.local_n + (self.nc,)
        if out is None:
            out = np.zeros(shape)
        elif out.shape != shape or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of shape %s" % (shape,))
        n = np.array(self.mesh.local_n, np.int32)
        bcp = None
        if bc is not None:
            b = BCDesc()
            b.type[:] = list(bc[0])
            b.val[:] = list(bc[1])
            bcp = C.byref(b)
        self.mesh.check(self.mesh.lib.nova_field_download(self.mesh.h, self.h, _dptr(out), _iptr(n), bcp))
        return out

    # device-native layout [c][i][j][k]
    def set_bc(self, types, vals=None):
        """types/vals: 18 entries indexed face + 6*comp (north, south, east, west, top, bottom)."""
        b = BCDesc()
        b.type[:] = [int(t) for t in types] + [0] * (18 - len(types))
        v = list(vals) if vals is not None else [0.0] * len(types)
        b.val[:] = [float(x) for x in v] + [0.0] * (18 - len(v))
        self.mesh.check(self.mesh.lib.nova_field_set_bc(self.mesh.h, self.h, C.byref(b)))
        return self

    def upload_soa(self, soa):
        a = np.ascontiguousarray(soa, np.float64)
        if a.size != self.nc * int(np.prod(self.mesh.shape)):
            raise ValueError("wrong size")
        self.mesh.check(self.mesh.lib.nova_field_upload_soa(self.mesh.h, self.h, _dptr(a)))
        return self

    def download_soa(self):
        out = np.zeros((self.nc,) + self.mesh.shape)
        self.mesh.check(self.mesh.lib.nova_field_download_soa(self.mesh.h, self.h, _dptr(out)))
        return out

    def copy_from_device(self, dev_ptr):
        self.mesh.check(self.mesh.lib.nova_field_copy_from_device(self.mesh.h, self.h, C.c_void_p(dev_ptr)))

    def copy_to_device(self, dev_ptr):
        self.mesh.check(self.mesh.lib.nova_field_copy_to_device(self.mesh.h, self.h, C.c_void_p(dev_ptr)))


class ex:
    """The reference's explicit operators (src/ex), each one C-ABI call."""

    @staticmethod
    def grad(f: Field) -> Field:
        M = f.mesh
        if f.nc == 1:
            out = Field(M, 3)
            M.check(M.lib.nova_grad_s(M.h, f.h, out.h))
        else:
            out = Field(M, 9)
            M.check(M.lib.nova_grad_v(M.h, f.h, out.h))
        return out

    @staticmethod
    def div(U: Field, f: Field = None) -> Field:
        """div(vector), div(vector, T), div(tensor), div(symmTensor), div(scalar, tensor)."""
        M = U.mesh
        if f is None and U.nc in (6, 9):
            out = Field(M, 3)
            M.check(M.lib.nova_div_t(M.h, U.h, out.h))
        elif f is None:
            out = Field(M, 1)
            M.check(M.lib.nova_div_v(M.h, U.h, out.h))
        elif U.nc == 1:
            out = Field(M, 3)
            M.check(M.lib.nova_div_st(M.h, U.h, f.h, out.h))
        else:
            out = Field(M, f.nc)
            M.check(M.lib.nova_div_vf(M.h, U.h, f.h, out.h))
        return out

    @staticmethod
    def curl(U: Field) -> Field:
        M = U.mesh
        out = Field(M, 3)
        M.check(M.lib.nova_curl(M.h, U.h, out.h))
        return out

    @staticmethod
    def laplacian(nu, f: Field) -> Field:
        """laplacian(scalar nu, T) or laplacian(Field<scalar> nu, T)."""
        M = f.mesh
        out = Field(M, f.nc)
        if isinstance(nu, Field):
            M.check(M.lib.nova_laplacian_f(M.h, nu.h, f.h, out.h))
        else:
            M.check(M.lib.nova_laplacian(M.h, float(nu), f.h, out.h))
        return out


class poisson:
    """poisson(p): rhs(f) then solve() writes p (src/poisson/poisson.h:36-115)."""

    def __init__(self, p: Field):
        self.p = p
        self._rhs = None

    def rhs(self, f: Field):
        self._rhs = f

    def solve(self):
        M = self.p.mesh
        M.check(M.lib.nova_poisson_solve(M.h, self._rhs.h, self.p.h))


class FdMatrix:
    """The reference's fdMatrix<scalar> (src/im/fdMatrix): per-node coefficients
    al[0..5] (neighbours j+1, j-1, i+1, i-1, k+1, k-1), ap and the source b of
    A x = b, and the transported field x that solve() updates in place."""

    def __init__(self, mesh: Mesh, x: Field, h):
        self.mesh, self.x, self.h = mesh, x, h

    def close(self):
        """release the matrix's device memory now"""
        if getattr(self, "h", None) and self.mesh.lib is not None:
            self.mesh.lib.nova_fdm_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    def add(self, other: "FdMatrix", alpha: float = 1.0) -> "FdMatrix":
        """self += alpha other (operator+ / operator-)"""
        self.mesh.check(self.mesh.lib.nova_fdm_add(self.mesh.h, self.h, float(alpha), other.h))
        return self

    def mul(self, other: "FdMatrix") -> "FdMatrix":
        """self *= other node by node (operator*=)"""
        self.mesh.check(self.mesh.lib.nova_fdm_mul(self.mesh.h, self.h, other.h))
        return self

    def scale(self, s: float) -> "FdMatrix":
        """coefficients and source times s (s = -1: unary operator-)"""
        self.mesh.check(self.mesh.lib.nova_fdm_scale(self.mesh.h, self.h, float(s)))
        return self

    def eq(self, f: Field, alpha: float = 1.0) -> "FdMatrix":
        """operator==: the source += alpha f"""
        self.mesh.check(self.mesh.lib.nova_fdm_add_source(self.mesh.h, self.h, float(alpha), f.h))
        return self

    def add_diagonal(self, d: float) -> "FdMatrix":
        """ap() += d"""
        self.mesh.check(self.mesh.lib.nova_fdm_add_diagonal(self.mesh.h, self.h, float(d)))
        return self

    def relax(self, urf: float) -> "FdMatrix":
        """fdMatrix::relax(urf): source += (1 - urf)/urf ap x, then ap /= urf (urf > 0)"""
        self.mesh.check(self.mesh.lib.nova_fdm_relax(self.mesh.h, self.h, float(urf)))
        return self

    def set_reference(self, i: int, j: int, k: int, val: float) -> "FdMatrix":
        """fdMatrix::setReference at the unique node (i, j, k): source += 1e15 val, ap *= 1e15"""
        self.mesh.check(self.mesh.lib.nova_fdm_set_reference(self.mesh.h, self.h, int(i), int(j), int(k),
                                                             float(val)))
        return self

    def residual(self) -> float:
        """fdMatrix::residual: the RMS of b - A x over the reference's (N0+1)(N1+1)(N2+1) nodes"""
        r = C.c_double()
        self.mesh.check(self.mesh.lib.nova_fdm_residual(self.mesh.h, self.h, C.byref(r)))
        return r.value

    def solve(self, tol: float, max_its: int):
        """Line relaxation on x until the residual is not above tol; returns (iterations, residual)."""
        its, r = C.c_int(), C.c_double()
        self.mesh.check(self.mesh.lib.nova_fdm_solve(self.mesh.h, self.h, float(tol), int(max_its), C.byref(its),
                                                     C.byref(r)))
        return its.value, r.value

    def download(self):
        """(al (6, N0, N1, N2), ap, b) on the unique nodes"""
        out = np.zeros((8,) + tuple(self.mesh.N))
        self.mesh.check(self.mesh.lib.nova_fdm_download(self.mesh.h, self.h, _dptr(out)))
        return out[:6], out[6], out[7]


class im:
    """The reference's implicit operators (src/im)."""

    @staticmethod
    def laplacian(mu: float, x: Field) -> FdMatrix:
        M = x.mesh
        h = C.c_void_p()
        M.check(M.lib.nova_im_laplacian(M.h, float(mu), x.h, C.byref(h)))
        return FdMatrix(M, x, h)


class tools:
    @staticmethod
    def maximum(f: Field) -> float:
        M = f.mesh
        v = C.c_double()
        M.check(M.lib.nova_field_maxabs(M.h, f.h, C.byref(v)))
        return v.value

    @staticmethod
    def maximum_noalloc(f: Field) -> float:
        """maximum() through the allocation-free entry point (fixed static
        scratch, at most NOVA_MAXABS_NOALLOC_MAX_NODES stored nodes; calls on one
        device must not overlap in time)."""
        M = f.mesh
        v = C.c_double()
        M.check(M.lib.nova_field_maxabs_noalloc(M.h, f.h, C.byref(v)))
        return v.value


def run_desc(model="ns", rk_mode="classical", precision=F64, dt=0.01, nu=0.0, eta=0.0, diag_every=1, t0=0.0,
             poisson="fft"):
    r = RunDesc()
    r.poisson = POISSON_DCT if poisson == "dct" else POISSON_FFT
    r.model = MODEL_MHD if model == "mhd" else MODEL_NS
    r.rk_mode = {"literal": RK_LITERAL, "classical": RK_CLASSICAL, "shear": RK_SHEARLAYER}[rk_mode]
    r.precision = precision
    r.diag_every = diag_every
    r.dt, r.nu, r.eta, r.t0 = float(dt), float(nu), float(eta), float(t0)
    return r


def advance(mesh: Mesh, rd: RunDesc, U: Field, p: Field, B: Field = None, pB: Field = None, nsteps: int = 1,
            history: bool = True):
    """nsteps of the reference loop body; returns the (nsteps, HIST_COLS) history or None."""
    st = State(U.h, p.h, B.h if B is not None else None, pB.h if pB is not None else None)
    hist = np.zeros((max(nsteps, 1), HIST_COLS)) if history else None
    mesh.check(mesh.lib.nova_advance(mesh.h, C.byref(rd), C.byref(st), int(nsteps),
                                     _dptr(hist) if history else None))
    return hist


def adjoint_grad(mesh: Mesh, rd: RunDesc, U0: Field, nsteps: int, checkpoint_every: int = 20,
                 window_start: int = None, B0: Field = None, total_energy: bool = False, weight: Field = None):
    """Gradient of J by the discrete adjoint.  J = Ek(nsteps); with total_energy
    (MHD) Ek + Em; with window_start = n0 the dissipation over steps n0+1..nsteps,
    E(n0) - E(nsteps) (E = Ek, or Ek + Em for MHD); with a weight field w
    (Navier-Stokes, FP64) J = <w, U(nsteps)> / N^3.  Returns (J, dJ/dU0) for
    Navier-Stokes and (J, dJ/dU0, dJ/dB0) for MHD (rd.model MHD, B0 given).
    With rd.precision F32SPLIT (U0, B0 split fields) the trajectory is the split
    path's and the adjoint stages run in FP32; the gradients are FP64."""
    a = AdjDesc()
    a.run = rd
    a.nsteps = int(nsteps)
    a.checkpoint_every = int(checkpoint_every)
    a.weight = weight.h if weight is not None else None
    if weight is not None:
        a.objective = OBJ_LINEAR_FINAL
    elif window_start is not None:
        a.objective = OBJ_DISSIPATION_WINDOW
    else:
        a.objective = OBJ_ETOT_FINAL if total_energy else OBJ_EKIN_FINAL
    a.window_start = 0 if window_start is None else int(window_start)
    grad = Field(mesh, 3)
    gradB = Field(mesh, 3) if B0 is not None else None
    st = State(U0.h, None, B0.h if B0 is not None else None, None)
    J = C.c_double()
    mesh.check(mesh.lib.nova_adjoint_grad(mesh.h, C.byref(a), C.byref(st), grad.h,
                                          gradB.h if gradB is not None else None, C.byref(J)))
    return (J.value, grad) if gradB is None else (J.value, grad, gradB)


def _state(U=None, p=None, B=None, pB=None):
    return State(*(f.h if f is not None else None for f in (U, p, B, pB)))


def checkpoint_write(mesh: Mesh, path: str, U=None, p=None, B=None, pB=None, t: float = 0.0, step: int = 0):
    """Lossless FP64 restart file of the given fields (nova_checkpoint_write)."""
    st = _state(U, p, B, pB)
    mesh.check(mesh.lib.nova_checkpoint_write(mesh.h, os.fsencode(path), C.byref(st), float(t), int(step)))


def checkpoint_read(mesh: Mesh, path: str, U=None, p=None, B=None, pB=None):
    """Fill the given fields from a restart file of the same mesh; returns (t, step)."""
    st = _state(U, p, B, pB)
    t, step = C.c_double(), C.c_longlong()
    mesh.check(mesh.lib.nova_checkpoint_read(mesh.h, os.fsencode(path), C.byref(st), C.byref(t), C.byref(step)))
    return t.value, step.value


def wc_desc(case="shear", dt=0.01, mu=0.0, ka=0.0, eos_k=50.0, g=(0.0, 0.0, 0.0), diag_every=1, t0=0.0):
    """nova_wc_desc: case "tg" (app/TG) or "shear" (app/shearLayerWC)."""
    d = WcDesc()
    d.wc_case = WC_SHEAR if case == "shear" else WC_TG
    d.diag_every, d.dt, d.mu, d.ka, d.eos_k, d.t0 = int(diag_every), dt, mu, ka, eos_k, t0
    d.g[:] = [float(v) for v in g]
    return d


def advance_wc(mesh: Mesh, wd: WcDesc, U: Field, rho: Field, p: Field, T: Field = None, nsteps: int = 1):
    """nsteps of the weakly-compressible loop bodies; returns the diagnostics rows."""
    st = WcState(U.h, rho.h, p.h, T.h if T is not None else None)
    hist = np.zeros((nsteps, HIST_COLS))
    mesh.check(mesh.lib.nova_advance_wc(mesh.h, C.byref(wd), C.byref(st), int(nsteps), _dptr(hist)))
    return hist


def wc_hydrostatic(mesh: Mesh, wd: WcDesc, rho0: float, T: Field, p: Field, rho: Field):
    """Initial p and rho of the weakly-compressible shear layer for a given T."""
    mesh.check(mesh.lib.nova_wc_hydrostatic(mesh.h, C.byref(wd), float(rho0), T.h, p.h, rho.h))


# ----------------------------------------------------------------- EnSight --
class ensight:
    """EnSight Gold files in the reference's layout (src/Mesh/Mesh.cpp:224-355,
    src/Field/Field.hxx:404-485).  The host functions need no GPU."""

    @staticmethod
    def mesh_desc(N, L=(2 * math.pi,) * 3, origin=(0.0, 0.0, 0.0), m=6, hyperbolic_z=None, walls=(0, 0, 0)):
        d = MeshDesc()
        d.N[:] = [int(v) for v in N]
        d.L[:] = [float(v) for v in L]
        d.origin[:] = [float(v) for v in origin]
        d.m = int(m)
        d.hyperbolic_z = int(hyperbolic_z is not None)
        d.s1, d.s2 = hyperbolic_z if hyperbolic_z is not None else (0.0, 0.0)
        d.walls[:] = [int(v) for v in walls]
        return d

    @staticmethod
    def _check(st, what):
        if st != OK:
            raise NovaError(st, what)

    @staticmethod
    def write_geometry(md: MeshDesc, dir: str):
        ensight._check(load_library().nova_ensight_write_geometry(C.byref(md), os.fsencode(dir)), dir)

    @staticmethod
    def write_case(dir: str, times):
        t = np.ascontiguousarray(times, np.float64)
        ensight._check(load_library().nova_ensight_write_case(os.fsencode(dir), len(t), _dptr(t)), dir)

    @staticmethod
    def write_host(md: MeshDesc, soa, dir: str, name: str, num: int):
        a = np.ascontiguousarray(soa, np.float64)
        nc = a.shape[0] if a.ndim == 4 else 1
        ensight._check(load_library().nova_ensight_write_host(C.byref(md), _dptr(a), nc, os.fsencode(dir),
                                                              name.encode(), int(num)), name)

    @staticmethod
    def read_host(md: MeshDesc, nc: int, dir: str, name: str, num: int):
        shape = (nc,) + tuple(md.N[a] + md.walls[a] for a in range(3))
        out = np.zeros(shape)
        ensight._check(load_library().nova_ensight_read_host(C.byref(md), _dptr(out), nc, os.fsencode(dir),
                                                             name.encode(), int(num)), name)
        return out

    @staticmethod
    def write_field(f: Field, dir: str, name: str, num: int):
        M = f.mesh
        M.check(M.lib.nova_ensight_write_field(M.h, f.h, os.fsencode(dir), name.encode(), int(num)))

    @staticmethod
    def read_field(f: Field, dir: str, name: str, num: int):
        M = f.mesh
        M.check(M.lib.nova_ensight_read_field(M.h, f.h, os.fsencode(dir), name.encode(), int(num)))
        return f
