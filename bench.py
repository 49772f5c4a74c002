#!/usr/bin/env python
"""Benchmark of the explicit time advance: Mpoint-steps/s on one B200.

Workload: Taylor-Green vortex, incompressible, periodic [0,2pi]^3 at 256^3,
classical RK4 (four fused stage kernels) + one FFT pressure projection per
step, nu = 1/1600, dt fixed from CFL 0.3 of the initial field.  A step is one
call of the reference's loop body (app/TG_Piosson/RKLoop.H in its
stage-refreshed form).  Synthetic data: the analytic initial field.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--n 256]

One JSON line on rank 0.  `value` is the FP64 path with the state resident in
HBM; the FP32-split path (FP32 stencils, (hi,lo) state, FP64 projection) is
reported beside it with its error against FP64.  `e2e` runs the same steps
through the reference-layout C ABI with host buffers: the ghosted
array-of-structs field is uploaded from pinned memory, the diagnostics row is
read back every step and the final field is downloaded, all inside the timed
region.  With N > 1 GPUs each rank advances its own replica (the reference
path does not shard on one GPU per rank here), timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mpoint-steps/s at 256^3: FP64 vs FP32-split (stated err); adjoint/fwd time ratio"
UNIT = "Mpoint-steps/s"
NU = 1.0 / 1600.0
MHD_NU = 1.0 / 1000.0
CFL = 0.3
# algorithmic HBM bytes per grid point for one classical RK4 step of the NS
# stage kernels (3 components): FP64 stages 72 + 120 + 120 + 72; FP32-split
# stages 36 + 60 + 60 + 72 (see the stage-kernel epilogue in nova_stage.cu)
STAGE_BYTES = {"f64": 384.0, "f32split": 228.0}
STAGE_LAUNCHES_PER_STEP = 4
# fdMatrix::solve, FP64 bytes per node per iteration that the algorithm must
# move: the residual reads the 8 matrix fields and x (72); each of the three
# line sweeps reads the 8 matrix fields (source, ap, the two coefficients along
# the line, the four off it) and x, and writes x (80)
IM_BYTES = 72.0 + 3 * 80.0


def workload_config(n, extra=None):
    c = {"workload": "Taylor-Green vortex, incompressible, periodic [0,2pi]^3, %d^3, classical RK4 + FFT "
                     "projection per step, nu=1/1600, CFL 0.3" % n,
         "grid": [n, n, n], "rk": "classical", "stencil_order": 6,
         "l2": "inputs larger than L2 (FP64 state %.0f MB)" % (3 * 8 * n ** 3 / 1e6),
         "parallelism": "replicas"}
    if extra:
        c.update(extra)
    return c


def tg_field(n):
    x = np.arange(n) * (2 * math.pi / n)
    s, c = np.sin(x), np.cos(x)
    u = s[:, None, None] * c[None, :, None] * c[None, None, :]
    v = -c[:, None, None] * s[None, :, None] * c[None, None, :]
    return np.stack([u, v, np.zeros_like(u)])


def ot_fields(n):
    """Orszag-Tang: u = (-2 sin y, 2 sin x, 0), B = (-2 sin 2y + sin z, 2 sin x + sin z, 0)."""
    x = np.arange(n) * (2 * math.pi / n)
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    U = np.stack([-2.0 * np.sin(Y), 2.0 * np.sin(X), np.zeros_like(X)])
    B = np.stack([-2.0 * np.sin(2.0 * Y) + np.sin(Z), 2.0 * np.sin(X) + np.sin(Z), np.zeros_like(X)])
    return U, B


def shear_layer_field(N, L, seed=0, noise=1e-3, delta=28.0):
    """Temporal shear layer on the stored nodes of a mesh with y walls (N1 + 1
    rows): u = tanh(delta (y - pi)), v = w = 0, plus seed-`seed` Gaussian noise
    of amplitude `noise` on every component."""
    y = np.arange(N[1] + 1) * (L[1] / N[1])
    u = np.broadcast_to(np.tanh(delta * (y - math.pi))[None, :, None], (N[0], N[1] + 1, N[2]))
    U = np.stack([u, np.zeros_like(u), np.zeros_like(u)])
    return U + noise * np.random.default_rng(seed).standard_normal(U.shape)


def mhd_jet_fields(N, L, origin, seed=1, noise=1e-3):
    """MHD jet about the z axis: u_z = 0.5 (1 - tanh((r - 1)/0.1)), B_z = 0.5,
    B_theta = 0.2 r exp(-r^2), seed-`seed` white noise of amplitude `noise` on u."""
    x, y, z = (origin[a] + np.arange(N[a]) * (L[a] / N[a]) for a in range(3))
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    r = np.sqrt(X * X + Y * Y)
    zero = np.zeros_like(X)
    U = np.stack([zero, zero, 0.5 * (1.0 - np.tanh((r - 1.0) / 0.1))])
    U = U + noise * np.random.default_rng(seed).standard_normal(U.shape)
    e = 0.2 * np.exp(-r * r)
    return U, np.stack([-e * Y, e * X, np.full_like(X, 0.5)])


def wc_shear_setup(N, mach, seed=0):
    """The weakly-compressible shear layer of app/shearLayerWC/shearLayer.cpp:31-44,
    116-135 (Mach as a parameter; its std::default_random_engine noise replaced by
    a seeded uniform(-1, 1) generator) on [0, 14 h0) x [0, 1.7 h0) x [-7.5 h0, 7.5 h0):
    returns (constants, L, U, T)."""
    Re0, Ri0, Pr, rho0, c = 1967.0, 0.08, 7.0, 999.57, 0.0417
    u0, h0, t0 = c * mach, 0.2, 0.1
    mu = rho0 * u0 * h0 / Re0
    prm = dict(rho0=rho0, c=c, u0=u0, h0=h0, t0=t0, mu=mu, ka=mu / Pr, gz=-Ri0 * u0 * u0 / t0 / h0)
    L = (14.0 * h0, 1.7 * h0, 15.0 * h0)
    x = np.arange(N[0]) * (L[0] / N[0])
    z = np.arange(N[2]) * (L[2] / N[2]) - 7.5 * h0
    X, _, Z = np.meshgrid(x, np.zeros(N[1]), z, indexing="ij")
    rng = np.random.default_rng(seed)
    k0 = 2.0 * 3.1415926536 / (14.0 * h0 / 2.0)
    a, b = 0.005, 0.4177
    th, ch = np.tanh(2.0 * Z / h0), np.cosh(2.0 * Z / h0)
    U = np.zeros((3,) + tuple(N))
    U[0] = u0 / 2.0 * th + a * u0 / 2.0 / k0 * (-np.cos(2 * k0 * X) + 2.0 * b * np.cos(k0 * X)) * th / ch
    U[1] = a * u0 / 2.0 * rng.uniform(-1, 1, N) / ch / ch
    U[2] = a * u0 / 2.0 * rng.uniform(-1, 1, N) / ch / ch
    T = t0 / 2.0 * th + a * t0 / 2.0 * rng.uniform(-1, 1, N) / ch / ch
    return prm, L, U, T[None]


def unit_directions(n, count, seed):
    """Seeded random vector fields of unit RMS amplitude on the n^3 grid, one at
    a time: white noise, so every Fourier mode carries a random phase and no
    symmetry of the base state annihilates a direction."""
    rng = np.random.default_rng(seed)
    for _ in range(count):
        v = rng.standard_normal((3, n, n, n))
        yield v / math.sqrt(float(np.mean(v * v)))


def final_energy(nova, GM, rd, U0, nsteps, B0=None):
    """E_kin (+ E_mag with B0) after nsteps, from the solver's own diagnostics row."""
    U = nova.Field(GM, 3).upload_soa(U0)
    p = nova.Field(GM, 1)
    B = pB = None
    if B0 is not None:
        B, pB = nova.Field(GM, 3).upload_soa(B0), nova.Field(GM, 1)
    rd.diag_every = nsteps
    h = nova.advance(GM, rd, U, p, B, pB, nsteps=nsteps, history=True)
    rd.diag_every = 0
    for f in (U, p, B, pB):
        if f is not None:
            f.close()
    return float(h[-1, 2] + (h[-1, 3] if B0 is not None else 0.0))


def fd_check(nova, GM, rd, U0, grads, nsteps, count, eps=1e-6, B0=None, seed=2024):
    """Finite differences of the objective along `count` seeded unit directions
    (white noise in U, and in B for MHD) against the adjoint gradient.  The
    check uses the fourth-order central difference
    (8 (J(+e) - J(-e)) - (J(+2e) - J(-2e))) / 12e, whose O(e^2) term cancels;
    the second-order one, (J(+e) - J(-e)) / 2e, carries e^2 J'''[v,v,v] / 6 and
    is stated beside it (fd2).  Per direction |fd - grad J . v| / |grad J . v|,
    every direction counted (max_rel_err), and the projection against a random
    direction's typical one, |grad J| |v| / sqrt(dim)."""
    gnorm = math.sqrt(sum(float(np.sum(g * g)) for g in grads))
    dim = sum(g.size for g in grads)
    n = U0.shape[1]
    dirs = unit_directions(n, count * (2 if B0 is not None else 1), seed)
    rows = []
    for _ in range(count):
        v = next(dirs)
        w = next(dirs) if B0 is not None else None

        def J(s):
            return final_energy(nova, GM, rd, U0 + s * v, nsteps, None if B0 is None else B0 + s * w)

        d1 = J(eps) - J(-eps)
        d2 = J(2 * eps) - J(-2 * eps)
        fd2 = d1 / (2 * eps)
        fd = (8 * d1 - d2) / (12 * eps)
        ad = float(np.sum(grads[0] * v)) + (float(np.sum(grads[1] * w)) if B0 is not None else 0.0)
        vnorm = math.sqrt(float(np.sum(v * v)) + (float(np.sum(w * w)) if B0 is not None else 0.0))
        typical = gnorm * vnorm / math.sqrt(dim)

        def rel(x):
            return abs(x - ad) / abs(ad) if ad else float("inf")

        rows.append({"fd": fd, "adjoint": ad, "rel_err": rel(fd), "fd2": fd2, "rel_err_fd2": rel(fd2),
                     "projection_vs_typical": abs(ad) / typical})
    worst = max(r["rel_err"] for r in rows)
    return {"directions": count, "eps": eps, "checked": count, "max_rel_err": worst, "max_rel_err_all": worst,
            "max_rel_err_fd2": max(r["rel_err_fd2"] for r in rows), "passes_1e-6": bool(worst <= 1e-6),
            "stencil": "fourth-order central (+-e, +-2e)", "direction_kind": "seeded white noise, unit RMS",
            "per_direction": rows, "objective_from": "the solver's diagnostics row after the same steps"}


def ghosted(U, h=3):
    """(3, n, n, n) unique nodes -> the reference's ghosted AoS Field<vector> layout (periodic images)."""
    n = U.shape[1]
    idx = (np.arange(n + 1 + 2 * h) - h) % n
    g = U[:, idx][:, :, idx][:, :, :, idx]
    return np.ascontiguousarray(np.moveaxis(g, 0, -1))


def cfl_dt(n, U, B=None):
    s = np.abs(U).sum(axis=0) + (0.0 if B is None else np.abs(B).sum(axis=0))
    return CFL * (2 * math.pi / n) / float(s.max())


def max_over_ranks(x, dist, device="cuda"):
    """The largest of a per-rank float over all ranks (the identity without a process group)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_value(name, key):
    """A 'key: value' line of a committed ncu summary under profiles/, if any."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith(key + ":"):
            return float(line.split(":")[1])
    return None


def profiled_traffic():
    """DRAM bytes per grid point per stage launch from the committed ncu summary, if any."""
    return profiled_value("stage_kernel_ns_f64.md", "dram_bytes_per_point_per_launch")


class ClockSampler:
    """NVML SM clock and throttle-reason samples while the timed region runs."""
    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, cuda_index):
        self.cuda_index = cuda_index
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nvml = pynvml
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            ids = [v.strip() for v in vis.split(",") if v.strip()]
            if ids and self.cuda_index < len(ids):
                sel = ids[self.cuda_index]
                if sel.isdigit():
                    self._h = pynvml.nvmlDeviceGetHandleByIndex(int(sel))
                else:
                    self._h = pynvml.nvmlDeviceGetHandleByUUID(sel)
            else:
                self._h = pynvml.nvmlDeviceGetHandleByIndex(self.cuda_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self._nvml = None
            return self
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def _run(self):
        nv = self._nvml
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for bit, name in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.01)

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


# ------------------------------------------------------------ reference arm --

def reference_bin(omp=False):
    """The reference compiled in place: its supported configuration, the serial
    build on one thread (the reference's CMake rejects OpenMP), or with omp the
    build with its own #pragma omp loops on every host thread (experimental)."""
    path = os.path.join(ROOT, "oracle", "_ref", "nova_ref_omp" if omp else "nova_ref")
    if not os.path.exists(path):
        return None, 0
    return path, (os.cpu_count() or 1) if omp else 1


def run_reference(n, nsteps, omp=False):
    """Run the reference's own loop body (compiled in place) on an n^3 Taylor-Green field.
    Returns (per-step wall seconds of the loop bodies, threads, binary)."""
    from oracle import oracle as O
    exe, cores = reference_bin(omp)
    if exe is None:
        raise RuntimeError("reference not built (make -C oracle ref ref-omp)")
    M = O.Mesh((n, n, n))
    U = O.ic_taylor_green(M)
    dt = cfl_dt(n, U)
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(cores)
    with tempfile.TemporaryDirectory() as td:
        case = os.path.join(td, "case")
        O.write_case(case, M)
        M.to_ghosted(U).tofile(os.path.join(td, "U.bin"))
        out = os.path.join(td, "out")
        subprocess.run([exe, "run", case, "ns", "classical", str(nsteps), repr(dt), repr(NU), "0",
                        os.path.join(td, "U.bin"), "-", out], check=True, stdout=subprocess.DEVNULL, env=env)
        return [float(v) for v in open(out + "_time.txt").read().split()], cores, exe


def reference_arm(args, rank):
    """The reference's own loop body on the host: its supported configuration
    (serial build, one thread, one rank), on a bounded 64^3 sample of the
    256^3 workload (per-point throughput measured size-independent: 64^3,
    128^3 and 256^3 within 7%); beside it, the build with its #pragma omp loops
    on every host thread, which the reference's CMake rejects (experimental)."""
    if rank != 0:
        return 0
    exe, cores = reference_bin()
    if exe is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference not compiled (make -C oracle ref)"}))
        return 0
    n = args.ref_n
    if args.warmup + args.steps > 60:  # keep the whole reference run within a few minutes
        n = 48 if args.warmup + args.steps <= 150 else 32
    times, cores, exe = run_reference(n, args.warmup + args.steps)
    t = sum(times[args.warmup:])
    value = n ** 3 * args.steps / t / 1e6
    sample = ("TG %d^3 (of 256^3), %d+%d steps, reference RKLoop body, serial build, 1 thread"
              % (n, args.warmup, args.steps))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic: analytic Taylor-Green field",
            "config": workload_config(args.n, {"sample_grid": [n, n, n], "threads": 1}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    exe_omp, threads = reference_bin(omp=True)
    if exe_omp is not None:
        to, threads, _ = run_reference(n, 1 + min(args.steps, 10), omp=True)
        line["experimental_omp"] = {"value": n ** 3 * (len(to) - 1) / sum(to[1:]) / 1e6, "unit": UNIT,
                                    "threads": threads, "sample": "the same loop body with the reference's own "
                                    "#pragma omp loops enabled (its CMake rejects OpenMP), %d^3" % n}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ our arm --

def time_device(nova, torch, GM, U, p, rd, steps, warmup, dist, stage_bytes):
    """Warm up, then time exactly `steps` device-resident steps; returns (seconds, stage stats, launches, clocks)."""
    nova.advance(GM, rd, U, p, nsteps=warmup, history=False)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    GM.profile(True)
    GM.profile_read(nova.K_STAGE, reset=True)
    GM.launch_count(reset=True)
    dev = torch.cuda.current_device()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        torch.cuda.synchronize()
        ev0.record()
        nova.advance(GM, rd, U, p, nsteps=steps, history=False)
        ev1.record()
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    GM.profile(False)
    sec = ev0.elapsed_time(ev1) / 1e3
    st_ms, st_n = GM.profile_read(nova.K_STAGE, reset=True)
    launches = GM.launch_count(reset=True)
    return sec, (st_ms, st_n), launches, clk.summary()


def time_e2e(nova, torch, GM, U, p, rd, U0_aos_pinned, out_pinned, steps, dist):
    """Same steps through the reference-layout ABI with host buffers, copies inside the timed region."""
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    hist_rows = 0
    ev0.record()
    U.upload(U0_aos_pinned)
    hist = nova.advance(GM, rd, U, p, nsteps=steps, history=True)
    hist_rows = hist.shape[0]
    U.download(out=out_pinned)
    ev1.record()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    sec = ev0.elapsed_time(ev1) / 1e3
    h2d = U0_aos_pinned.nbytes
    d2h = out_pinned.nbytes + hist_rows * nova.HIST_COLS * 8
    return sec, h2d, d2h


def mhd_legs(args, nova, torch, dist, world):
    """Secondary MHD numbers: Orszag-Tang at args.mhd_n^3 for args.mhd_steps steps
    (U loop then B loop with its cleaning projection, classical RK4, nu = eta =
    1/1000), FP64 and FP32-split with the split error at the end, and the MHD
    adjoint / forward ratio at args.mhd_adj_n^3 with its finite-difference check."""
    def maxover(x):
        return max_over_ranks(x, dist)

    def timed(fn):
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r = fn()
        e1.record()
        torch.cuda.synchronize()
        return maxover(e0.elapsed_time(e1) / 1e3), r

    n, steps = args.mhd_n, args.mhd_steps
    U0, B0 = ot_fields(n)
    dt = cfl_dt(n, U0, B0)
    GM = nova.Mesh((n, n, n))
    GM.set_stream(torch.cuda.current_stream().cuda_stream)
    p, pB = nova.Field(GM, 1), nova.Field(GM, 1)
    out, finals = {}, {}
    for prec_name, prec in (("f64", nova.F64), ("f32split", nova.F32SPLIT)):
        U, B = nova.Field(GM, 3, prec).upload_soa(U0), nova.Field(GM, 3, prec).upload_soa(B0)
        rd = nova.run_desc(model="mhd", rk_mode="classical", precision=prec, dt=dt, nu=MHD_NU, eta=MHD_NU,
                           diag_every=0)
        nova.advance(GM, rd, U, p, B, pB, nsteps=3, history=False)
        GM.launch_count(reset=True)
        sec, _ = timed(lambda: nova.advance(GM, rd, U, p, B, pB, nsteps=steps, history=False))
        out[prec_name] = {"value": world * n ** 3 * steps / sec / 1e6, "unit": UNIT,
                          "ms_per_step": 1e3 * sec / steps, "gpu_launches": GM.launch_count(reset=True)}
        finals[prec_name] = np.concatenate([U.download_soa(), B.download_soa()])
        U.close()
        B.close()
    out["f32split"]["rel_l2_vs_fp64"] = float(np.linalg.norm(finals["f32split"] - finals["f64"]) /
                                              np.linalg.norm(finals["f64"]))
    out["f32split"]["speedup_vs_fp64"] = out["f64"]["ms_per_step"] / out["f32split"]["ms_per_step"]
    p.close()
    pB.close()
    res = {"workload": "Orszag-Tang, periodic [0,2pi]^3, %d^3, classical RK4 U loop + FFT projection, then B "
                       "loop + cleaning projection, nu=eta=1/1000, CFL 0.3 on |u|+|B|; %d timed steps after 3"
                       % (n, steps), **out}
    if not args.no_adjoint:
        na, M, K = args.mhd_adj_n, args.adj_steps, args.adj_checkpoint
        U0, B0 = ot_fields(na)
        dt = cfl_dt(na, U0, B0)
        AM = nova.Mesh((na, na, na))
        AM.set_stream(torch.cuda.current_stream().cuda_stream)
        U, B = nova.Field(AM, 3).upload_soa(U0), nova.Field(AM, 3).upload_soa(B0)
        p, pB = nova.Field(AM, 1), nova.Field(AM, 1)
        rd = nova.run_desc(model="mhd", rk_mode="classical", dt=dt, nu=MHD_NU, eta=MHD_NU, diag_every=0)
        for r in nova.adjoint_grad(AM, rd, U, M, checkpoint_every=K, B0=B, total_energy=True)[1:]:
            r.close()  # warm-up: the same call, which also sizes the checkpoint pool
        t_fwd, _ = timed(lambda: nova.advance(AM, rd, U, p, B, pB, nsteps=M, history=False))
        U.upload_soa(U0)
        B.upload_soa(B0)
        t_adj, r = timed(lambda: nova.adjoint_grad(AM, rd, U, M, checkpoint_every=K, B0=B, total_energy=True))
        grads = [r[1].download_soa(), r[2].download_soa()]
        for f in list(r[1:]) + [U, B, p, pB]:
            f.close()
        fd = fd_check(nova, AM, rd, U0, grads, M, args.fd_dirs, B0=B0) if args.fd_dirs > 0 else None
        res["adjoint"] = {"ratio": t_adj / t_fwd, "forward_s": t_fwd, "adjoint_s": t_adj, "grid": [na] * 3,
                          "steps": M, "checkpoint_every": K, "objective": "E_kin + E_mag at the final step",
                          "gradients": "dJ/dU0 and dJ/dB0", "dtype": "f64", "J": r[0], "fd_check": fd}
        # the FP32-split adjoint of the same case against its own forward solve and the FP64 gradients
        U, B = nova.Field(AM, 3, nova.F32SPLIT).upload_soa(U0), nova.Field(AM, 3, nova.F32SPLIT).upload_soa(B0)
        p, pB = nova.Field(AM, 1), nova.Field(AM, 1)
        rd = nova.run_desc(model="mhd", rk_mode="classical", precision=nova.F32SPLIT, dt=dt, nu=MHD_NU, eta=MHD_NU,
                           diag_every=0)
        for f in nova.adjoint_grad(AM, rd, U, M, checkpoint_every=K, B0=B, total_energy=True)[1:]:
            f.close()
        t_fwd, _ = timed(lambda: nova.advance(AM, rd, U, p, B, pB, nsteps=M, history=False))
        U.upload_soa(U0)
        B.upload_soa(B0)
        t_adj, r = timed(lambda: nova.adjoint_grad(AM, rd, U, M, checkpoint_every=K, B0=B, total_energy=True))
        g32 = [r[1].download_soa(), r[2].download_soa()]
        for f in list(r[1:]) + [U, B, p, pB]:
            f.close()
        res["adjoint"]["f32split"] = {
            "ratio": t_adj / t_fwd, "forward_s": t_fwd, "adjoint_s": t_adj, "J": r[0],
            "grad_rel_l2_vs_fp64": [float(np.linalg.norm(a - b) / np.linalg.norm(b)) for a, b in zip(g32, grads)],
            "dtype": "f32 adjoint stages and stage states, f64 adjoint state and projections"}
    return res


def timed_advance(torch, dist, fn):
    """CUDA-event seconds of fn() on the current stream, max over ranks."""
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    r = fn()
    e1.record()
    torch.cuda.synchronize()
    return max_over_ranks(e0.elapsed_time(e1) / 1e3, dist), r


def hbm_roof(alg_bytes, sec, what):
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / sec / 1e9
    return {"bound": "hbm", "kernel": what, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind}


# algorithmic HBM bytes per point and step of the configuration legs (one read
# of every input stream and one write of every output stream per fused pass;
# projection = divergence 3s+8, spectral solve 32, correction 8+3s+3s):
#   shear-layer loop (app/shearLayer/UEqn.H), per stage: the stage kernel
#   reads the stage state and the base and writes U* (FP64 72, split 60: U*
#   leaves in FP64 either way), then a projection of 136: the divergence 32,
#   the wall Poisson solve 48 (2-D (i, k) transform of the stored rows, the
#   DCT-I pass along y, the inverse transform: one read and one write of the
#   spectrum each) and the correction 56 (the split one writes the (hi, lo) pair)
SHEAR_STAGE_BYTES = {"f64": 72.0, "f32split": 60.0}
SHEAR_STEP_BYTES = {k: 4 * (v + 32 + 48 + 56) for k, v in SHEAR_STAGE_BYTES.items()}
#   MHD jet, the app's scheme (literal U loop: one stage reading U, B and
#   writing U*; projection; classical B loop with U frozen: 96, 144, 144, 96
#   FP64 / 48, 72, 72, 84 split; cleaning projection)
JET_STEP_BYTES = {"f64": 72 + 120 + 96 + 144 + 144 + 96 + 120, "f32split": 60 + 120 + 48 + 72 + 72 + 84 + 120}
#   weakly compressible: 5 evolved components at 136 B each (4 RK stages)
WC_STEP_BYTES = 5 * 136.0


def shear_leg(args, nova, torch, dist, world):
    """The temporal shear layer 256 x 256 x 128 with y walls: u = tanh(28 (y - pi))
    + seed-0 noise 1e-3, nu = 1/2000, the reference app's loop
    (app/shearLayer/UEqn.H: RK4 weights as stage coefficients, a projection per
    stage) with the wall Poisson solve on the even extension (DCT), dt from CFL
    0.3; args.shear_steps timed steps per precision after 3 warm-up steps, and
    the FP32-split error against FP64 after them."""
    N, L = (256, 256, 128), (2 * math.pi, 2 * math.pi, math.pi)
    steps = args.shear_steps
    U0 = shear_layer_field(N, L)
    dt = CFL * (L[0] / N[0]) / float(np.abs(U0).sum(axis=0).max())
    GM = nova.Mesh(N, L=L, walls=(0, 1, 0))
    GM.set_stream(torch.cuda.current_stream().cuda_stream)
    ubc = [0] * 18
    for c in range(3):  # u, w Neumann 0, v Dirichlet 0 on the north and south walls
        ubc[0 + 6 * c] = ubc[1 + 6 * c] = (2 if c == 1 else 1)
    pbc = [1, 1] + [0] * 16
    npts = N[0] * N[1] * N[2]
    out, finals = {}, {}
    for prec_name, prec in (("f64", nova.F64), ("f32split", nova.F32SPLIT)):
        U = nova.Field(GM, 3, prec).set_bc(ubc)
        p = nova.Field(GM, 1).set_bc(pbc)
        rd = nova.run_desc(model="ns", rk_mode="shear", precision=prec, dt=dt, nu=1.0 / 2000.0, poisson="dct",
                           diag_every=0)
        U.upload_soa(U0)
        nova.advance(GM, rd, U, p, nsteps=3, history=False)
        U.upload_soa(U0)
        GM.profile(True)
        GM.profile_read(nova.K_STAGE, reset=True)
        GM.launch_count(reset=True)
        sec, _ = timed_advance(torch, dist, lambda: nova.advance(GM, rd, U, p, nsteps=steps, history=False))
        GM.profile(False)
        st_ms, st_n = GM.profile_read(nova.K_STAGE, reset=True)
        out[prec_name] = {"value": world * npts * steps / sec / 1e6, "unit": UNIT, "ms_per_step": 1e3 * sec / steps,
                          "gpu_launches": GM.launch_count(reset=True),
                          "roofline": hbm_roof(SHEAR_STEP_BYTES[prec_name] * npts * steps, sec,
                                               "whole step, %g B/point-step" % SHEAR_STEP_BYTES[prec_name]),
                          "stage_kernel": hbm_roof(SHEAR_STAGE_BYTES[prec_name] * npts * st_n, st_ms / 1e3,
                                                   "shear-loop stage kernel (walls; FP64 on the march, split on "
                                                   "the TMA pipeline), %g B/point" % SHEAR_STAGE_BYTES[prec_name])}
        finals[prec_name] = U.download_soa()
        U.close()
        p.close()
    err = float(np.linalg.norm(finals["f32split"] - finals["f64"]) / np.linalg.norm(finals["f64"]))
    out["f32split"]["rel_l2_vs_fp64"] = err
    out["f32split"]["speedup_vs_fp64"] = out["f64"]["ms_per_step"] / out["f32split"]["ms_per_step"]
    return {"workload": "temporal shear layer %dx%dx%d, y walls (DCT Poisson), app/shearLayer loop, nu=1/2000, "
                        "CFL 0.3; %d timed steps (t = %.3f)" % (N + (steps, steps * dt)), **out}


def jet_leg(args, nova, torch, dist, world):
    """The MHD jet 192 x 192 x 384 (x, y in [-4, 4), z in [0, 16)), nu = eta =
    1/1500, the reference app's scheme (literal U loop, refreshed B loop, both
    projected), dt from CFL 0.3 on |u| + |B|: args.jet_steps timed steps per
    precision after 3 warm-up steps, the FP32-split error against FP64 after them."""
    N, L, org = (192, 192, 384), (8.0, 8.0, 16.0), (-4.0, -4.0, 0.0)
    steps = args.jet_steps
    U0, B0 = mhd_jet_fields(N, L, org)
    dt = CFL * (L[0] / N[0]) / float((np.abs(U0).sum(axis=0) + np.abs(B0).sum(axis=0)).max())
    GM = nova.Mesh(N, L=L, origin=org)
    GM.set_stream(torch.cuda.current_stream().cuda_stream)
    npts = N[0] * N[1] * N[2]
    out, finals = {}, {}
    p, pB = nova.Field(GM, 1), nova.Field(GM, 1)
    for prec_name, prec in (("f64", nova.F64), ("f32split", nova.F32SPLIT)):
        U, B = nova.Field(GM, 3, prec), nova.Field(GM, 3, prec)
        rd = nova.run_desc(model="mhd", rk_mode="literal", precision=prec, dt=dt, nu=1 / 1500, eta=1 / 1500,
                           diag_every=0)
        U.upload_soa(U0)
        B.upload_soa(B0)
        nova.advance(GM, rd, U, p, B, pB, nsteps=3, history=False)
        U.upload_soa(U0)
        B.upload_soa(B0)
        GM.launch_count(reset=True)
        sec, _ = timed_advance(torch, dist, lambda: nova.advance(GM, rd, U, p, B, pB, nsteps=steps, history=False))
        out[prec_name] = {"value": world * npts * steps / sec / 1e6, "unit": UNIT, "ms_per_step": 1e3 * sec / steps,
                          "gpu_launches": GM.launch_count(reset=True),
                          "roofline": hbm_roof(JET_STEP_BYTES[prec_name] * npts * steps, sec,
                                               "whole step, %g B/point-step" % JET_STEP_BYTES[prec_name])}
        finals[prec_name] = np.concatenate([U.download_soa(), B.download_soa()])
        U.close()
        B.close()
    p.close()
    pB.close()
    out["f32split"]["rel_l2_vs_fp64"] = float(np.linalg.norm(finals["f32split"] - finals["f64"]) /
                                              np.linalg.norm(finals["f64"]))
    out["f32split"]["speedup_vs_fp64"] = out["f64"]["ms_per_step"] / out["f32split"]["ms_per_step"]
    return {"workload": "MHD jet %dx%dx%d periodic, literal U loop + B loop, both projected, nu=eta=1/1500, "
                        "CFL 0.3 on |u|+|B|; %d timed steps (t = %.3f)" % (N + (steps, steps * dt)), **out}


def wc_leg(args, nova, torch, dist, world):
    """The weakly-compressible shear layer (app/shearLayerWC) at 256^3, Mach 0.1:
    hydrostatic initialisation on the GPU, then args.wc_steps timed steps (U,
    rho + EOS, T loops) after 3 warm-up steps, FP64."""
    n, steps, mach = 256, args.wc_steps, 0.1
    prm, L, U0, T0 = wc_shear_setup((n, n, n), mach)
    GM = nova.Mesh((n, n, n), L=L)
    GM.set_stream(torch.cuda.current_stream().cuda_stream)
    dt = CFL * min(L[a] / n for a in range(3)) / (prm["u0"] / mach + prm["u0"] / 2.0)  # shearLayer.cpp:182
    K = prm["c"] * prm["c"] / 2.0 / prm["rho0"]
    wd = nova.wc_desc("shear", dt=dt, mu=prm["mu"], ka=prm["ka"], eos_k=K, g=(0.0, 0.0, prm["gz"]))
    U, rho, p, T = nova.Field(GM, 3).upload_soa(U0), nova.Field(GM, 1), nova.Field(GM, 1), nova.Field(GM, 1)
    T.upload_soa(T0)
    nova.wc_hydrostatic(GM, wd, prm["rho0"], T, p, rho)
    wd.diag_every = 0
    nova.advance_wc(GM, wd, U, rho, p, T, nsteps=3)
    GM.launch_count(reset=True)
    sec, _ = timed_advance(torch, dist, lambda: nova.advance_wc(GM, wd, U, rho, p, T, nsteps=steps))
    launches = GM.launch_count(reset=True)
    ok = bool(np.all(np.isfinite(rho.download_soa())))
    for f in (U, rho, p, T):
        f.close()
    return {"workload": "weakly-compressible shear layer (app/shearLayerWC) %d^3, Mach %g, U/rho/T loops with the "
                        "EOS, dt from shearLayer.cpp:182 at CFL 0.3; %d timed steps" % (n, mach, steps),
            "value": world * n ** 3 * steps / sec / 1e6, "unit": UNIT, "ms_per_step": 1e3 * sec / steps,
            "gpu_launches": launches, "dtype": "f64", "finite": ok,
            "roofline": hbm_roof(WC_STEP_BYTES * n ** 3 * steps, sec, "whole step, %g B/point-step" % WC_STEP_BYTES)}


def im_leg(args, nova, torch, dist, world):
    """The implicit Laplacian of src/im: im::laplacian(mu, x), ap -= c, (M == f)
    and fdMatrix::solve with tol = 0, so that exactly args.im_its iterations run
    (residual check, then line sweeps along j, i, k), on a periodic args.im_n^3
    mesh; beside it the reference's own solve on the host (serial, as written)."""
    n, its = args.im_n, args.im_its
    mu, c = 1e-3, 1.0
    rng = np.random.default_rng(11)
    x0, f0 = rng.standard_normal((1, n, n, n)), rng.standard_normal((1, n, n, n))
    GM = nova.Mesh((n, n, n))
    GM.set_stream(torch.cuda.current_stream().cuda_stream)
    x, f = nova.Field(GM, 1).upload_soa(x0), nova.Field(GM, 1).upload_soa(f0)
    A = nova.im.laplacian(mu, x)
    A.add_diagonal(-c)
    A.eq(f)
    A.solve(0.0, 3)  # warm-up: scratch and line factors
    res0 = A.residual()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    GM.launch_count(reset=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    done, _ = A.solve(0.0, its)
    e1.record()
    torch.cuda.synchronize()
    sec = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist)
    launches = GM.launch_count(reset=True)
    res1 = A.residual()
    A.close()
    x.close()
    f.close()
    peak, peak_kind = measured_peaks()
    achieved = IM_BYTES * n ** 3 * its / sec / 1e9
    tr = profiled_value("fdm_solve_256.md", "dram_bytes_per_node_iteration")
    out = {"workload": "im::laplacian(1e-3, x) - 1 == f on a periodic [0,2pi]^3 %d^3 mesh, random x and f; "
                       "fdMatrix::solve(tol=0, %d) timed after 3 iterations" % (n, its),
           "value": world * n ** 3 * its / sec / 1e6, "unit": "Mnode-iterations/s", "iterations": done,
           "ms_per_iteration": 1e3 * sec / its, "gpu_launches": launches, "dtype": "f64",
           "residual_before_after": [res0, res1],
           "roofline": {"bound": "hbm", "kernel": "one solve iteration (residual + three line sweeps)",
                        "alg_bytes_per_node_iteration": IM_BYTES, "achieved": achieved, "peak": peak,
                        "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                        "traffic": None if tr is None else tr * n ** 3,
                        "traffic_per": "iteration (DRAM bytes from the committed ncu summary)"}}
    if world == 1 and not args.no_cpu_baseline and reference_bin()[0] is not None:
        from oracle import oracle as O
        nc, ic = args.im_cpu_n, args.im_cpu_its
        M = O.Mesh((nc, nc, nc), L=(2 * np.pi,) * 3)
        r = O.ref_im(M, mu, c, M.to_ghosted(x0[:, :nc, :nc, :nc]), M.to_ghosted(f0[:, :nc, :nc, :nc]), 0.0, ic)
        out["cpu_baseline"] = {"value": nc ** 3 * ic / r["solve_s"] / 1e6, "unit": "Mnode-iterations/s",
                               "cores": 1, "kind": "reference",
                               "sample": "the reference's fdMatrix::solve (serial as written), %d^3, %d iterations"
                                         % (nc, ic)}
    return out


def our_arm(args, rank, world, dist):
    import torch
    from novaclone_b200 import nova

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    # one explicit stream for the library and for torch's timing events
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    n = args.n
    U0 = tg_field(n)
    dt = cfl_dt(n, U0)
    GM = nova.Mesh((n, n, n))
    GM.set_stream(torch.cuda.current_stream().cuda_stream)
    p = nova.Field(GM, 1)

    def maxover(x):
        return max_over_ranks(x, dist)

    res = {}
    finals = {}
    for prec_name, prec in (("f64", nova.F64), ("f32split", nova.F32SPLIT)):
        U = nova.Field(GM, 3, prec).upload_soa(U0)
        rd = nova.run_desc(model="ns", rk_mode="classical", precision=prec, dt=dt, nu=NU, diag_every=0)
        sec, (st_ms, st_n), launches, clocks = time_device(nova, torch, GM, U, p, rd, args.steps, args.warmup, dist,
                                                           STAGE_BYTES[prec_name])
        finals[prec_name] = U.download_soa()
        sec = maxover(sec)
        res[prec_name] = {"sec": sec, "stage_ms": st_ms, "stage_launches": st_n, "launches": launches,
                          "clocks": clocks, "value": world * n ** 3 * args.steps / sec / 1e6,
                          "ms_per_step": 1e3 * sec / args.steps}
        U.close()

    err = float(np.linalg.norm(finals["f32split"] - finals["f64"]) / np.linalg.norm(finals["f64"]))
    # the split error at t = 1: the smallest step count that reaches it
    n1 = int(math.ceil(1.0 / dt - 1e-9))
    for prec_name, prec in (() if args.no_t1 else (("f64", nova.F64), ("f32split", nova.F32SPLIT))):
        U = nova.Field(GM, 3, prec).upload_soa(U0)
        rd = nova.run_desc(model="ns", rk_mode="classical", precision=prec, dt=dt, nu=NU, diag_every=0)
        nova.advance(GM, rd, U, p, nsteps=n1, history=False)
        finals[prec_name] = U.download_soa()
        U.close()
    err_t1 = None if args.no_t1 else float(np.linalg.norm(finals["f32split"] - finals["f64"]) /
                                           np.linalg.norm(finals["f64"]))
    del finals

    # adjoint / forward wall-time ratio: gradient of E_kin after M steps with
    # checkpoints every K steps, against an M-step forward solve of the same
    # precision (FP64, then FP32-split, whose gradient is compared with FP64's)
    adj = None
    if not args.no_adjoint:
        M, K = args.adj_steps, args.adj_checkpoint
        adj_runs = {}
        for prec_name, prec in (("f64", nova.F64), ("f32split", nova.F32SPLIT)):
            U = nova.Field(GM, 3, prec).upload_soa(U0)
            rd = nova.run_desc(model="ns", rk_mode="classical", precision=prec, dt=dt, nu=NU, diag_every=0)
            # warm-up: the same call, which also sizes the checkpoint pool (a
            # one-time device allocation of about (M/K + 4K + 5) fields)
            nova.adjoint_grad(GM, rd, U, M, checkpoint_every=K)[1].close()
            torch.cuda.synchronize()
            e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            e[0].record()
            nova.advance(GM, rd, U, p, nsteps=M, history=False)
            e[1].record()
            U.upload_soa(U0)
            torch.cuda.synchronize()
            e[2].record()
            J, grad = nova.adjoint_grad(GM, rd, U, M, checkpoint_every=K)
            e[3].record()
            torch.cuda.synchronize()
            t_fwd = maxover(e[0].elapsed_time(e[1]) / 1e3)
            t_adj = maxover(e[2].elapsed_time(e[3]) / 1e3)
            adj_runs[prec_name] = {"ratio": t_adj / t_fwd, "forward_s": t_fwd, "adjoint_s": t_adj, "J": J,
                                   "grad": grad.download_soa()}
            grad.close()
            U.close()
        f, s32 = adj_runs["f64"], adj_runs["f32split"]
        fd = None
        if args.fd_dirs > 0:
            rd = nova.run_desc(model="ns", rk_mode="classical", precision=nova.F64, dt=dt, nu=NU, diag_every=0)
            fd = fd_check(nova, GM, rd, U0, [f["grad"]], M, args.fd_dirs)
        adj = {"ratio": f["ratio"], "forward_s": f["forward_s"], "adjoint_s": f["adjoint_s"], "steps": M,
               "checkpoint_every": K, "objective": "E_kin at the final step", "dtype": "f64", "J": f["J"],
               "fd_check": fd,
               "f32split": {"ratio": s32["ratio"], "forward_s": s32["forward_s"], "adjoint_s": s32["adjoint_s"],
                            "J": s32["J"], "grad_rel_l2_vs_fp64": float(np.linalg.norm(s32["grad"] - f["grad"]) /
                                                                        np.linalg.norm(f["grad"])),
                            "dtype": "f32 adjoint stages and stage states, f64 adjoint state and projection"}}
        del adj_runs
    t_end = (args.warmup + args.steps) * dt

    # e2e through the reference-layout ABI (ghosted AoS host buffers, pinned)
    e2e = {}
    if not args.no_e2e:
        aos = ghosted(U0)
        pin_in = torch.empty(aos.shape, dtype=torch.float64, pin_memory=True).numpy()
        pin_in[...] = aos
        pin_out = torch.empty(aos.shape, dtype=torch.float64, pin_memory=True).numpy()
        for prec_name, prec in (("f64", nova.F64), ("f32split", nova.F32SPLIT)):
            U = nova.Field(GM, 3, prec)
            rd = nova.run_desc(model="ns", rk_mode="classical", precision=prec, dt=dt, nu=NU, diag_every=1)
            U.upload(pin_in)
            nova.advance(GM, rd, U, p, nsteps=1, history=True)  # warm the path (plans, buffers)
            sec, h2d, d2h = time_e2e(nova, torch, GM, U, p, rd, pin_in, pin_out, args.steps, dist)
            sec = maxover(sec)
            e2e[prec_name] = {"value": world * n ** 3 * args.steps / sec / 1e6, "unit": UNIT,
                              "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                              "ms_per_step": 1e3 * sec / args.steps}
            U.close()

    mhd = None if args.no_mhd else mhd_legs(args, nova, torch, dist, world)
    im = None if args.no_im else im_leg(args, nova, torch, dist, world)
    configs = None
    if not args.no_configs:
        configs = {"shear_layer": shear_leg(args, nova, torch, dist, world),
                   "mhd_jet": jet_leg(args, nova, torch, dist, world),
                   "wc_shear": wc_leg(args, nova, torch, dist, world)}

    if rank != 0:
        return 0

    peak, peak_kind = measured_peaks()

    def roof(prec_name):
        r = res[prec_name]
        if r["stage_launches"] == 0:
            return None
        bytes_total = STAGE_BYTES[prec_name] * n ** 3 * r["stage_launches"] / STAGE_LAUNCHES_PER_STEP
        achieved = bytes_total / (r["stage_ms"] / 1e3) / 1e9
        tr = profiled_traffic() if prec_name == "f64" else None
        return {"bound": "hbm", "kernel": "k_stage (fused RHS + RK stage update), NS %s" % prec_name,
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "avg_launch_ms": r["stage_ms"] / r["stage_launches"],
                "alg_bytes_per_launch": STAGE_BYTES[prec_name] * n ** 3 / STAGE_LAUNCHES_PER_STEP,
                "traffic": None if tr is None else tr * n ** 3, "stage_share_of_step": r["stage_ms"] / (1e3 * r["sec"])}

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        exe, cores = reference_bin()
        if exe is not None:
            ns = args.cpu_n
            times, cores, exe = run_reference(ns, args.cpu_steps + 1)
            t = sum(times[1:])
            cpu = {"value": ns ** 3 * args.cpu_steps / t / 1e6, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": "TG %d^3 (of 256^3), %d steps after 1, reference loop body, serial build, 1 thread"
                             % (ns, args.cpu_steps)}
            exe_omp, _ = reference_bin(omp=True)
            if exe_omp is not None:
                to, threads, _ = run_reference(ns, args.cpu_steps + 1, omp=True)
                cpu["experimental_omp"] = {"value": ns ** 3 * args.cpu_steps / sum(to[1:]) / 1e6, "threads": threads,
                                           "sample": "the same with the reference's own #pragma omp loops"}

    f64 = res["f64"]
    f32 = res["f32split"]
    line = {
        "metric": METRIC, "value": f64["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": f64["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic: analytic Taylor-Green initial field",
        "config": workload_config(n),
        "roofline": roof("f64"),
        "cpu_baseline": cpu,
        "e2e": e2e.get("f64"),
        "gpu_launches": f64["launches"],
        "clocks": f64["clocks"],
        "fp32split": {"value": f32["value"], "unit": UNIT, "ms_per_step": f32["ms_per_step"],
                      "speedup_vs_fp64": f64["ms_per_step"] / f32["ms_per_step"],
                      "rel_l2_vs_fp64": err, "at_time": t_end, "steps_compared": args.warmup + args.steps,
                      "rel_l2_vs_fp64_t1": err_t1, "t1": n1 * dt, "t1_steps": n1,
                      "dtype": "f32 stencils, (hi,lo) f32 state, f64 projection", "roofline": roof("f32split"),
                      "e2e": e2e.get("f32split"), "gpu_launches": f32["launches"], "clocks": f32["clocks"]},
        "adjoint_fwd_ratio": None if adj is None else adj["ratio"],
        "adjoint": adj,
        "mhd": mhd,
        "im": im,
        "configs": configs,
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--ref-n", type=int, default=64, help="grid of the reference arm's bounded sample")
    ap.add_argument("--cpu-n", type=int, default=64)
    ap.add_argument("--cpu-steps", type=int, default=6)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--adj-steps", type=int, default=200)
    ap.add_argument("--adj-checkpoint", type=int, default=20)
    ap.add_argument("--no-mhd", action="store_true")
    ap.add_argument("--mhd-n", type=int, default=128)
    ap.add_argument("--mhd-steps", type=int, default=200)
    ap.add_argument("--mhd-adj-n", type=int, default=128)
    ap.add_argument("--no-im", action="store_true")
    ap.add_argument("--im-n", type=int, default=256)
    ap.add_argument("--im-its", type=int, default=20)
    ap.add_argument("--im-cpu-n", type=int, default=128)
    ap.add_argument("--im-cpu-its", type=int, default=30)
    ap.add_argument("--fd-dirs", type=int, default=8, help="finite-difference checks of each FP64 adjoint")
    ap.add_argument("--no-configs", action="store_true", help="skip the shear-layer, MHD-jet and WC legs")
    ap.add_argument("--no-t1", action="store_true", help="skip the FP32-split error run to t = 1")
    ap.add_argument("--shear-steps", type=int, default=500)
    ap.add_argument("--jet-steps", type=int, default=200)
    ap.add_argument("--wc-steps", type=int, default=50)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank)
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        return our_arm(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
