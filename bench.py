#!/usr/bin/env python
"""bench.py -- cell-steps/s of the projected SSP-RK3 dynamical-core step.

Workload (default "cbl", the dry convective boundary layer): anelastic
core, 256 x 256 x 128 cells on 5120 m x 5120 m x 2000 m with tanh-stretched
z (first cell 8 m), rho0(z) = 1.2 exp(-z/8000), theta 300 K to 1 km then
+3 K and 3 K/km, seeded uniform +-0.1 K theta noise in the lowest 10 levels,
surface heat flux 0.1 K m/s, Smagorinsky C_s = 0.17 (Pr_t = 1/3), walls in
z, FFT-xy + tridiagonal-z pressure solve, dt = 1 s.  Synthetic inputs from
the Philox generator (no dataset exists for this case).

One "step" = one projected SSP-RK3 step of the whole grid.  `value` is the
FP32-mixed step (stencils and horizontal FFTs in FP32, the column solve and
reductions in FP64) timed with CUDA events on the library's stream with the
state resident in HBM; the FP64 step is measured the same way and reported
beside it.  `e2e` is the same metric through the C-ABI with the state copied
from pinned host memory and back every step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--workload cbl|tgv|urban|hit|urban_step|tracer]

The default line also carries "pcg": the other half of the headline metric,
the time to a 1e-8 relative residual of the cut-cell urban pressure problem
(256 x 256 x 96 at 2 m, 40 floor-standing boxes, multigrid-preconditioned CG
in FP64 and FP32-mixed).  `--workload urban` reports that solve as the line's
own metric (ms to 1e-8, lower is better) with its roofline, e2e and CPU
baseline.  `--workload hit` is the decaying isotropic turbulence of 512^3
cells (WENO-Z5, no SGS, adaptive dt at CFL 0.5): the FP64 run steps
adaptively, the FP32-mixed run repeats its dt sequence, and the line reports
the FP32-mixed cell-steps/s beside the FP64 rate with the fields' relative L2
difference and the kinetic-energy difference after `--hit-steps` steps.

`--workload urban_step` is the large urban convective case: 1024 x 1024 x
192 cells of 2 m, 600 seeded floor-standing boxes, surface heat flux
0.15 K m/s, WENO-JS5 with Smagorinsky, the projection by the
multigrid-preconditioned CG on the cut-cell apertures to a 1e-8 relative
residual; FP32-mixed against FP64 (cell-steps/s, CG iterations and solve
time, field error after `--urban-steps` steps), with the learned U-Net
preconditioner in the FP32-mixed run when `--learned` is given.

Under torchrun every rank runs an independent replica of the workload (the
step has no data-path collective on one domain; weak scaling) and rank 0
prints one JSON line with the max-over-ranks time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "aeolus.jl_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

HBM_FALLBACK_GBS = 6650.0
# DRAM bytes (read + write) of one sweep launch of the CBL 256x256x128 FP32-mixed
# step, from an ncu capture of `python bench.py --steps 2 --warmup 3`
# (profiles/sweep_pair_kernel_cbl256_fp32.md)
CBL_SWEEP_DRAM_BYTES = 315824640 + 109399552
# ... and of one finest red-black colour pass of the urban 256x256x96 FP32-mixed
# solve (profiles/mg_vcycle_urban256x256x96_fp32.md): 69.4 MB read + 1.3 MB written
URBAN_RBGS_DRAM_BYTES = 70.7e6


# ----------------------------------------------------------------------------- workloads

def workload(name):
    from aeolus_b200 import CoreSpec, regular_grid, stretched_grid, tanh_beta_for_first_cell, tanh_faces
    from aeolus_b200.inputs import cbl_initial, cbl_theta_profile, taylor_green
    from aeolus_b200.reference_state import anelastic_profiles, exponential_density

    if name == "cbl":
        nx, nz, lz = 256, 128, 2000.0
        beta = tanh_beta_for_first_cell(nz, lz, 8.0)
        g = stretched_grid((nx, nx, nz), (5120.0, 5120.0, lz), tanh_faces(nz, lz, beta))
        prof = anelastic_profiles(g, exponential_density(g), cbl_theta_profile(g.znodes("c")))

        def spec(prec):
            return CoreSpec(grid=g, core="anelastic", c_s=0.17, pr_t=1 / 3, flux_bot=0.1, precision=prec,
                            wc=prof["wc"], wf=prof["wf"], thf=prof["thf"])

        u, v, w, th, _ = cbl_initial(g, seed=1, noise=0.1, noise_levels=10)
        desc = {"workload": "dry CBL, anelastic, 256x256x128, tanh z (dz1=8 m, beta=%.4f), Cs=0.17, "
                            "F=0.1 K m/s, dt=1 s, FFT-xy + tridiagonal-z" % beta,
                "grid": [nx, nx, nz], "dt": 1.0, "advection": "centred (W-weighted flux form)",
                "sgs": "Smagorinsky Cs=0.17 Prt=1/3", "l2": "inputs larger than L2 (state ~0.5 GB)"}
        return g, spec, (u, v, w, th), 1.0, desc, False
    if name == "tgv":
        n = 256
        g = regular_grid((n, n, n), (2 * np.pi,) * 3)

        def spec(prec):
            return CoreSpec(grid=g, advection="weno_js5", nu=1 / 1600, precision=prec)

        state = taylor_green(g, seed=1, amp=1e-3)
        desc = {"workload": "Taylor-Green vortex 256^3 triply periodic, WENO-JS5, nu=1/1600, dt=0.01, FFT projection",
                "grid": [n, n, n], "dt": 0.01, "l2": "inputs larger than L2"}
        return g, spec, state, 0.01, desc, True
    raise SystemExit(f"unknown workload {name}")


URBAN_N = (256, 256, 96)
URBAN_H = 2.0


def urban_problem(n=URBAN_N, seed=1, nboxes=40):
    """The cut-cell urban pressure problem: n cells of 2 m, `nboxes`
    floor-standing boxes (Philox-seeded centres, footprints U(10, 40) m,
    heights U(10, 60) m), sampled with nsub = 4; the right-hand side is
    vol_eff times the cut-cell divergence of a log-profile inflow (5 m/s at
    10 m, z0 = 0.1 m) plus seeded uniform +-0.5 m/s noise.  Returns the face
    coefficients a^2, the right-hand side and a description."""
    from aeolus_b200 import regular_grid
    from aeolus_b200.cutcell import box_geometry, face_coefficients, pressure_rhs, random_boxes, urban_velocity
    g = regular_grid(n, tuple(URBAN_H * v for v in n), halo=(3, 3, 3), bc_z="wall")
    geom = box_geometry(g, random_boxes(g, nboxes, seed=seed), nsub=4)
    u, v, w = urban_velocity(g, geom, seed=seed)
    b = pressure_rhs(geom, u, v, w)
    desc = {"workload": f"cut-cell urban pressure solve {n[0]}x{n[1]}x{n[2]} at 2 m, {nboxes} boxes (seed {seed}), "
                        "MG-preconditioned CG (V(2,2) RB-GS, a^2 faces) to ||r|| <= 1e-8 ||b||",
            "grid": list(n), "solid_fraction": round(float(geom.is_solid[g.interior].mean()), 4),
            "rhs": "vol_eff * cut-cell divergence of a log-profile inflow (5 m/s at 10 m, z0 0.1 m) "
                   "+ seeded +-0.5 m/s noise",
            "l2": "inputs larger than L2 (solver state ~0.4 GB)"}
    return face_coefficients(geom), b, desc


def pcg_solves(coeffs, b, reps, precisions=("fp64", "fp32_mixed")):
    """Device ms of one solve to 1e-8 (graph launches, b resident), plus the
    iteration count, for each precision."""
    from aeolus_b200.multigrid import MGPreconditionedCG
    out = {}
    for prec in precisions:
        s = MGPreconditionedCG(URBAN_N, (URBAN_H,) * 3, coeffs=coeffs, tol=1e-8, precision=prec)
        x, st = s.solve(b)
        ms = s.profile("solve", reps)
        out[prec] = {"ms": ms, "iterations": st["iterations"], "relative_residual": st["relative_residual"],
                     "status": st["status"], "handle": s}
    return out


# algorithmic bytes per cell of one launch of each kernel class (field passes
# P, one compulsory read or write of one interior scalar field), averaged over
# the three substages; the spectrum holds (nx/2+1)/nx complex per cell.
def class_passes(cls, g, sgs):
    sp = 2.0 * (g.nx // 2 + 1) / g.nx  # real words of the spectrum per cell
    return {
        "sweep": (8 + 9 + 9) / 3.0,            # R u,v,w,theta (+theta0); W u*,v*,w*,theta
        "sgs": 4.0,                           # R u,v,w; W nut
        "div_fftx": 3.0 + sp,                 # R u*,v*,w*; W spectrum (the divergence + r2c pair)
        "ffty": 2.0 * sp,                     # R+W spectrum
        "zsolve": 2.0 * sp,                   # R+W spectrum
        "ifftx": sp + 1.0,                    # R spectrum; W phi
        "correct": (8 + 11 + 11) / 3.0,       # R u*,v*,w*,phi (+u0,v0,w0); W u,v,w,p
        "halo": 0.0,
    }[cls]


LAUNCHES_PER_STEP = {"sweep": 3, "sgs": 6, "div_fftx": 3, "ffty": 6, "zsolve": 3, "ifftx": 3, "correct": 3, "halo": 3}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """SM clocks and clock-event reasons sampled during the timed region:
    read-only NVML queries every 2 ms from a thread (the GPU found by its PCI
    address), so even a timed region of a few milliseconds has samples;
    nvidia-smi at 100 ms when NVML is not importable."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown", 0x8),
             ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
             ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
             ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap", 0x4))

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.nvml = None
        self.lines = []
        self.sm = []
        self.smax = None
        self.reasons = set()

    def _nvml_sample(self):
        m = self.nvml
        self.sm.append(float(m.nvmlDeviceGetClockInfo(self.h, m.NVML_CLOCK_SM)))
        r = m.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        for name, const, bit in self.NAMES:
            if r & getattr(m, const, bit):
                self.reasons.add(name)

    def _poll(self):
        while not self.halt.is_set():
            try:
                self._nvml_sample()
            except Exception:
                return
            time.sleep(0.002)

    def start(self):
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            p = torch.cuda.get_device_properties(self.device)
            bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
            self.h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            self.nvml = pynvml
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
            self._nvml_sample()
            self.halt = threading.Event()
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml:
            self.halt.set()
            self.t.join(timeout=5)
            try:
                self._nvml_sample()
            except Exception:
                pass
            return {"sm_mhz": statistics.median(self.sm) if self.sm else None, "sm_max_mhz": self.smax,
                    "reasons": sorted(self.reasons), "samples": len(self.sm), "source": "nvml, 2 ms"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = [n for n, _, _ in self.NAMES]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi, 100 ms"}


# ----------------------------------------------------------------------------- distributed
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "gloo"
        if torch.cuda.is_available():   # one rank per GPU; gloo for the host-only (CPU) runs
            torch.cuda.set_device(local)
            backend = "nccl"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------------------- timing
def timed_steps(sim, dt, k, world):
    import torch
    stream = torch.cuda.ExternalStream(sim.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    sim.synchronize()
    torch.cuda.synchronize()
    e0.record(stream)
    sim.step_rk3_async(dt, k)
    e1.record(stream)
    sim.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    return e0.elapsed_time(e1)


def e2e_steps(sim, state, dt, k, f32=False):
    """Through the C-ABI with host buffers: every step uploads u, v, w, theta
    from pinned host memory, steps, and downloads them again -- FP64 host
    arrays, or with f32 the FP32 ones of aeo_set_field_f32 / aeo_get_field_f32
    (an FP32-mixed domain's host mirror)."""
    import torch
    dt_host = torch.float32 if f32 else torch.float64
    pinned = []
    for a in state:
        t = torch.empty(a.shape, dtype=dt_host, pin_memory=True)
        t.numpy()[...] = a
        pinned.append(t.numpy())
    outs = [torch.empty(a.shape, dtype=dt_host, pin_memory=True).numpy() for a in state]
    put = sim.set_field_f32 if f32 else sim.set_field
    get = sim.get_field_f32 if f32 else sim.get_field
    stream = torch.cuda.ExternalStream(sim.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sim.synchronize()
    e0.record(stream)
    for _ in range(k):
        for n, a in zip(("u", "v", "w", "theta"), pinned):
            put(n, a)
        sim.step_rk3(dt, 1)
        for n, o in zip(("u", "v", "w", "theta"), outs):
            get(n, o)
    e1.record(stream)
    sim.synchronize()
    nbytes = sum(a.nbytes for a in pinned)
    return e0.elapsed_time(e1) / k, nbytes, sum(o.nbytes for o in outs)


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_oracle_rate(spec, state, dt, min_seconds=10.0, max_steps=20, threads=None):
    """The oracle (CPU restatement) on the host cores (all of them, or
    `threads`), full grid."""
    from oracle.oracle import OracleSimulation, set_threads
    cores = threads or os.cpu_count() or 1
    set_threads(cores)
    o = OracleSimulation(spec)
    o.set_state(*state)
    o.step_rk3(dt, 1)  # warm-up
    n, t0 = 0, time.perf_counter()
    while True:
        o.step_rk3(dt, 1)
        n += 1
        el = time.perf_counter() - t0
        if el >= min_seconds or n >= max_steps:
            break
    o.close()
    return spec.grid.ncells * n / el, cores, n, el


# ----------------------------------------------------------------------------- arms
def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    g, mkspec, state, dt, desc, _ = workload(args.workload)
    spec = mkspec("fp64")
    from oracle.oracle import OracleSimulation, set_threads
    cores = os.cpu_count() or 1
    set_threads(cores)
    o = OracleSimulation(spec)
    o.set_state(*state)
    o.step_rk3(dt, max(1, args.warmup))
    t0 = time.perf_counter()
    o.step_rk3(dt, args.steps)
    el = time.perf_counter() - t0
    value = g.ncells * args.steps / el
    line = {
        "impl": "reference", "metric": "cell-steps/s", "value": value, "unit": "cell-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": desc,
        "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": cores, "kind": "port",
                         "sample": f"{args.steps} RK3 steps of the full {desc['grid']} grid after {max(1, args.warmup)} "
                                   f"warm-up steps; the reference is Julia (not installable), this is the "
                                   f"C/OpenMP FP64 restatement of its step"},
        "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_reference_urban(args):
    """The oracle's MG-preconditioned CG (serial C restatement) on the urban
    problem: one warm-up solve, then min(steps, 3) timed solves."""
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    from oracle.mgpcg import OracleMGPCG
    coeffs, b, desc = urban_problem()
    o = OracleMGPCG(URBAN_N, (URBAN_H,) * 3, coeffs=coeffs, tol=1e-8)
    x, st = o.solve(b)
    k = max(1, min(args.steps, 3))
    t0 = time.perf_counter()
    for _ in range(k):
        o.solve(b)
    ms = 1e3 * (time.perf_counter() - t0) / k
    line = {
        "impl": "reference", "metric": "PCG time-to-1e-8", "value": ms, "unit": "ms", "n_gpus": args.gpus,
        "steps": k, "warmup": 1, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": desc,
        "iterations": st["iterations"], "relative_residual": st["relative_residual"],
        "cpu_baseline": {"value": ms, "unit": "ms", "cores": 1, "kind": "port",
                         "sample": f"{k} full solves after one warm-up; the reference is Julia (not installable), "
                                   "this is the serial C FP64 restatement of its MGPreconditionedCG"},
        "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_b200_urban(args):
    world, rank, local = dist_setup()
    import torch
    torch.cuda.set_device(local)
    from aeolus_b200.multigrid import MGPreconditionedCG
    coeffs, b, desc = urban_problem()
    hbm, hbm_kind = measured_peaks()
    n = int(np.prod(URBAN_N))
    res = {}
    for prec in ("fp32_mixed", "fp64"):
        s = MGPreconditionedCG(URBAN_N, (URBAN_H,) * 3, coeffs=coeffs, tol=1e-8, precision=prec, device=local)
        for _ in range(args.warmup):
            x, st = s.solve(b)
        clk = ClockSampler(local)
        clk.start()
        barrier(world)
        ms = s.profile("solve", args.steps)
        barrier(world)
        clocks = clk.stop()
        ms = max_over_ranks(ms, world)
        parts = {p: s.profile(p, 20) for p in ("vcycle", "apply", "sweep", "rbgs", "restrict", "coarsest")}
        # e2e: the C-ABI call with pinned host arrays, copies inside
        bh = torch.empty(b.shape, dtype=torch.float64, pin_memory=True).numpy()
        bh[...] = b
        xh = torch.empty(b.shape, dtype=torch.float64, pin_memory=True).numpy()
        t0 = time.perf_counter()
        ke = max(2, min(args.steps, 5))
        for _ in range(ke):
            _, st = s.solve(bh, out=xh)
        e2e = max_over_ranks(1e3 * (time.perf_counter() - t0) / ke, world)
        res[prec] = dict(ms=ms, st=st, parts=parts, clocks=clocks, e2e=e2e, lpi=s.launches_per_iteration)
        del s
    if rank != 0:
        barrier(world)
        return 0
    m = res["fp32_mixed"]
    rb_bytes = 11.0 * n          # one colour pass, FP32: phi 4 + b 2 + codes 3 + write 2 bytes/cell
    ach = rb_bytes / (m["parts"]["rbgs"] * 1e-3) / 1e9
    line = {
        "metric": "PCG time-to-1e-8", "value": m["ms"], "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": m["ms"], "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32-mixed (FP32 multigrid cycle; FP64 Krylov vectors, operator, reductions)",
        "data": "synthetic (Philox-seeded boxes and inflow)",
        "config": dict(desc, parallelism=f"replicas x{world}" if world > 1 else "1 GPU"),
        "iterations": m["st"]["iterations"], "relative_residual": m["st"]["relative_residual"],
        "fp64": {"ms": res["fp64"]["ms"], "iterations": res["fp64"]["st"]["iterations"],
                 "relative_residual": res["fp64"]["st"]["relative_residual"], "e2e_ms": res["fp64"]["e2e"]},
        "e2e": {"value": m["e2e"], "unit": "ms", "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n + 64},
        "roofline": {"bound": "hbm", "kernel": "mg_rbgs_kernel (finest level, one colour pass)",
                     "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s", "frac": round(ach / hbm, 4),
                     "peak_kind": hbm_kind, "bytes_per_launch": rb_bytes,
                     "traffic": URBAN_RBGS_DRAM_BYTES if tuple(URBAN_N) == (256, 256, 96) else None,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one finest colour "
                                       "pass at 256x256x96 (profiles/mg_vcycle_urban256x256x96_fp32.md)"},
        "parts_ms": {k: round(v, 4) for k, v in m["parts"].items()},
        "gpu_launches": (m["st"]["iterations"] + 1) * m["lpi"] * args.steps,
        "clocks": m["clocks"],
        "learned": learned_pcg(coeffs, b, args),
    }
    if world == 1 and not args.no_cpu_baseline:
        from oracle.mgpcg import OracleMGPCG
        o = OracleMGPCG(URBAN_N, (URBAN_H,) * 3, coeffs=coeffs, tol=1e-8)
        t0 = time.perf_counter()
        _, sto = o.solve(b)
        el = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": 1e3 * el, "unit": "ms", "cores": 1, "kind": "port",
                                "sample": f"one full solve ({sto['iterations']} iterations), serial FP64 oracle"}
    print(json.dumps(line), flush=True)
    barrier(world)
    return 0


def learned_pcg(coeffs, b, args):
    """The learned U-Net preconditioner on the urban problem, trained in this
    run on the run's own snapshots: `--learned-steps` (200) projected RK3
    steps of the same setup (256 x 256 x 96 at 2 m, 40 boxes of a training
    seed, the log-profile inflow, dt = 0.1 s), after each step the right-hand
    side of its last projection solved again by the plain MG-preconditioned
    CG with its first 10 residual -> error pairs used for Adam steps (2,000
    pairs); then used in flexible CG on the test geometry (seed 1, a fresh
    seed).  Compared with CG without a preconditioner (the method without the
    network), with Jacobi-preconditioned CG (the density-weighted
    projection's solver) and with the multigrid preconditioner."""
    from aeolus_b200.learned import train_from_run, transfer, urban_flow, urban_geometry
    from aeolus_b200.multigrid import MGPreconditionedCG
    t0 = time.perf_counter()
    sim, tg, tgeom = urban_flow(URBAN_N, seed=101, nboxes=40)
    net, losses, used = train_from_run(sim, steps=args.learned_steps, dt=0.1, cap=10,
                                       fluid=(~tgeom.is_solid[tg.interior]).astype(np.float32))
    sim.close()
    del sim, tgeom
    train_s = time.perf_counter() - t0
    g, geom = urban_geometry(URBAN_N, 1, 40)
    fluid = (~geom.is_solid[g.interior]).astype(np.float32)
    big = transfer(net, URBAN_N, fluid)
    k = min(50, len(losses) // 4) or 1
    out = {"training": {"pairs": used, "seconds": round(train_s, 1), "loss_first": float(losses[:k].mean()),
                        "loss_last": float(losses[-k:].mean()), "grid": list(URBAN_N),
                        "source": f"{args.learned_steps} spin-up steps of the urban flow (training seed 101, 40 "
                                  "boxes, dt 0.1 s), pairs of each step's last projection re-solved by plain MG-PCG",
                        "step_ms": big.profile("train", 3)},
           "unet_forward_ms": big.profile("forward", 10)}
    for name, pc in (("learned", "vcycle"), ("plain_cg", "identity"), ("jacobi_cg", "jacobi"), ("mg", "vcycle")):
        s = MGPreconditionedCG(URBAN_N, (URBAN_H,) * 3, coeffs=coeffs, tol=1e-8, precision="fp32_mixed", maxit=4000,
                               precond=pc)
        if name == "learned":
            s.set_learned(big, stagnation=0.9)
        x, st = s.solve(b)
        out[name] = {"ms": s.profile("solve", 3), "iterations": st["iterations"],
                     "relative_residual": st["relative_residual"], "status": st["status"],
                     "fallback_at": st["fallback_at"]}
    return out


def run_reference_hit(args):
    """The oracle (all host cores) on the HIT workload: the field generated on
    the host by the same spectral construction, projected, then timed steps
    at the first adaptive dt (each step is a bounded sample of the workload)."""
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    from aeolus_b200 import CoreSpec, regular_grid
    from aeolus_b200.inputs import isotropic_turbulence
    from aeolus_b200.simulation import CFLConstraints
    from oracle.oracle import OracleSimulation, set_threads
    n = args.hit_n
    g = regular_grid((n, n, n), (2 * np.pi,) * 3)
    cores = os.cpu_count() or 1
    set_threads(cores)
    o = OracleSimulation(CoreSpec(grid=g, advection="weno_z5", nu=0.0))
    u, v, w = isotropic_turbulence(g, 1.0, 4.0, seed=1)
    o.set_state(u, v, w, g.zeros())
    del u, v, w
    o.project()
    dt, _ = o.adaptive_dt(CFLConstraints(C_advective=0.5, growth_max=1.1))
    k = max(1, min(args.steps, 2))
    t0 = time.perf_counter()
    o.step_rk3(dt, k)
    el = time.perf_counter() - t0
    value = g.ncells * k / el
    line = {"impl": "reference", "metric": "cell-steps/s", "value": value, "unit": "cell-steps/s",
            "n_gpus": args.gpus, "steps": k, "warmup": 0, "ms_per_step": 1e3 * el / k, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"decaying isotropic turbulence {n}^3, WENO-Z5, no SGS", "grid": [n, n, n]},
            "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": cores, "kind": "port",
                             "sample": f"{k} RK3 steps of the full grid at the first adaptive dt, FP64 oracle"},
            "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def precision_comparison(s32, s64, g, theta_ref=None):
    """FP32-mixed against FP64 after the same steps from the same state: per
    prognostic field the relative L2 difference, the max abs difference and
    that max relative to the FP64 field's max; theta also as its departure
    from `theta_ref` (the initial profile), whose differences are not hidden
    behind the 300 K level; kinetic energies and max divergences."""
    rel, mx, mxr = {}, {}, {}
    names = ("u", "v", "w") + (("theta",) if theta_ref is not None else ())
    for f in names:
        a, b = s32.get_field(f)[g.interior], s64.get_field(f)[g.interior]
        keys = [(f, a, b)]
        if f == "theta":
            keys.append(("theta_departure", a - theta_ref, b - theta_ref))
        for k, x, y in keys:
            d = np.abs(x - y)
            ny_ = float(np.linalg.norm(y))
            rel[k] = float(np.linalg.norm(x - y) / ny_) if ny_ > 0 else float(np.linalg.norm(x - y))
            mx[k] = float(d.max())
            ym = float(np.abs(y).max())
            mxr[k] = mx[k] / ym if ym > 0 else mx[k]
        del a, b, keys
    return {"relative_l2": rel, "max_abs": mx, "max_relative": mxr,
            "ke_fp64": s64.kinetic_energy(), "ke_fp32": s32.kinetic_energy(),
            "max_divergence_fp64": s64.max_divergence(), "max_divergence_fp32": s32.max_divergence()}


def ke_change(cmp, ke0_64, ke0_32):
    """Kinetic-energy drift of the FP32-mixed run against FP64: the relative
    difference of the final energies and of the energy change over the run
    (the decay of a decaying flow, the growth of a convecting one)."""
    k64, k32 = cmp["ke_fp64"], cmp["ke_fp32"]
    d64, d32 = k64 - ke0_64, k32 - ke0_32
    cmp.update({"ke_initial_fp64": ke0_64, "ke_initial_fp32": ke0_32,
                "ke_relative_difference": abs(k32 - k64) / abs(k64) if k64 else None,
                "ke_change_fp64": d64, "ke_change_fp32": d32,
                "ke_change_relative_difference": abs(d32 - d64) / abs(d64) if d64 else None})
    return cmp


def hit_run(n, nsteps, args, local, world):
    """Config 3, decaying isotropic turbulence on n^3 cells: the FP64 run steps
    adaptively (CFL 0.5, growth 1.1) for `nsteps` steps, the FP32-mixed run
    repeats its dt sequence from the same start, the two are compared; then
    both are timed at the last dt (the captured graph) and adaptively."""
    import torch
    from aeolus_b200 import CoreSpec, regular_grid
    from aeolus_b200.simulation import CFLConstraints, Simulation
    g = regular_grid((n, n, n), (2 * np.pi,) * 3)

    def spec(prec):
        return CoreSpec(grid=g, advection="weno_z5", nu=0.0, precision=prec)

    s64 = Simulation(spec("fp64"), device=local)
    s64.init_isotropic(u_rms=1.0, k_peak=4.0, seed=1, project=True, target_rms=1.0)
    state0 = s64.get_state()
    ke0 = s64.kinetic_energy()
    c = CFLConstraints(C_advective=0.5, growth_max=1.1)
    dts, dt_prev = [], None
    for _ in range(nsteps):
        st = s64.step_adaptive(c, 1, dt_prev)
        dts.append(st["dt"])
        dt_prev = st["dt"]
    s32 = Simulation(spec("fp32_mixed"), device=local)
    s32.set_state(*state0)
    del state0
    ke0_32 = s32.kinetic_energy()
    for dt in dts:
        s32.step_rk3(dt, 1)
    cmp = ke_change(precision_comparison(s32, s64, g), ke0, ke0_32)
    cmp["ke_decay_relative_difference"] = cmp["ke_change_relative_difference"]
    cmp.update({"steps": nsteps, "t_end": float(np.sum(dts)), "dt_first": dts[0], "dt_last": dts[-1]})
    dt = dts[-1]
    res = {}
    for name, sim in (("fp32_mixed", s32), ("fp64", s64)):
        sim.step_rk3(dt, args.warmup)
        clk = ClockSampler(local)
        clk.start()
        ms = timed_steps(sim, dt, args.steps, world) / args.steps
        clocks = clk.stop()
        prof = sim.profile_step(dt)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ka = max(3, min(args.steps, 10))
        # the guard's divergence bound is the reference's FP64 round-off bound (1e-6);
        # an FP32 projection leaves ~1e-7 relative to the velocity gradients
        ca = c if name == "fp64" else CFLConstraints(C_advective=0.5, growth_max=1.1, divergence_tol=1e-2)
        sim.synchronize()
        e0.record(torch.cuda.ExternalStream(sim.stream))
        sim.step_adaptive(ca, ka, dt)
        e1.record(torch.cuda.ExternalStream(sim.stream))
        sim.synchronize()
        res[name] = {"ms": max_over_ranks(ms, world), "clocks": clocks, "prof": prof,
                     "adaptive_ms": e0.elapsed_time(e1) / ka, "launches": sim.launches_per_step()}
    s32.close()
    s64.close()
    return g, cmp, res


def run_b200_hit(args):
    world, rank, local = dist_setup()
    import torch
    torch.cuda.set_device(local)
    n = args.hit_n
    hbm, hbm_kind = measured_peaks()
    g, cmp, res = hit_run(n, args.hit_steps, args, local, world)
    if rank != 0:
        barrier(world)
        return 0
    ncell = g.ncells
    m = res["fp32_mixed"]
    prof = m["prof"]
    per_launch_ms = prof["sweep"] / LAUNCHES_PER_STEP["sweep"]
    sweep_bytes = class_passes("sweep", g, False) * 4 * ncell
    ach = sweep_bytes / (per_launch_ms * 1e-3) / 1e9
    line = {
        "metric": "cell-steps/s", "value": world * ncell / (m["ms"] * 1e-3), "unit": "cell-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": m["ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32-mixed (FP32 stencils/FFT, FP64 reductions)", "data": "synthetic (Passot-Pouquet spectrum, seed 1)",
        "config": {"workload": f"decaying isotropic turbulence {n}^3, triply periodic, WENO-Z5, no SGS, nu = 0, "
                               f"adaptive dt CFL 0.5 (growth 1.1), E(k) ~ k^4 exp(-2 (k/4)^2), u_rms = 1",
                   "grid": [n, n, n], "l2": "inputs larger than L2",
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
        "fp64": {"value": world * ncell / (res["fp64"]["ms"] * 1e-3), "ms_per_step": res["fp64"]["ms"],
                 "adaptive_ms_per_step": res["fp64"]["adaptive_ms"]},
        "adaptive_ms_per_step": m["adaptive_ms"],
        "fp32_vs_fp64": cmp,
        "roofline": {"bound": "hbm", "kernel": "sweep", "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
                     "frac": round(ach / hbm, 4), "peak_kind": hbm_kind, "bytes_per_launch": sweep_bytes,
                     "traffic": None},
        "gpu_launches": m["launches"] * args.steps,
        "clocks": m["clocks"],
    }
    print(json.dumps(line), flush=True)
    barrier(world)
    return 0


def run_tracer(args):
    """Positivity-preserving WENO-Z5 tracer advection (advect_positive!) on
    device arrays in the reference storage layout: 256^3 triply periodic,
    random face velocities at a first-order CFL of 0.9, a non-negative field
    with zero regions and blocks (the limiter active); FP32-mixed and FP64;
    the oracle on a 128^3 sample on the host cores as the CPU baseline (the
    reference arm prints only that)."""
    import torch
    from aeolus_b200 import CoreSpec, regular_grid
    from aeolus_b200.inputs import tracer_case as case

    def grid(n):
        return regular_grid(n, (1.0, 1.0, 1.0), halo=(3, 3, 3), bc_z="periodic")

    def spec(g, precision="fp64"):
        return CoreSpec(grid=g, advection="weno_z5", precision=precision)

    n = args.tracer_n
    g = grid((n, n, n))
    u, v, w, phi, dt = case(g, 1)
    ncell = g.ncells
    line = {"metric": "cell-updates/s", "unit": "cell-updates/s", "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "data": "synthetic (seeded velocities and field)",
            "config": {"workload": f"advect_positive WENO-Z5 tracer, {n}^3 triply periodic, first-order CFL 0.9, "
                                   "limiter active (zero regions and blocks)", "grid": [n, n, n],
                       "l2": "inputs larger than L2"}}
    if args.impl == "reference":
        world, rank, _ = dist_setup()
        if rank != 0:
            return 0
        from oracle.oracle import OracleSimulation, set_threads
        cores = os.cpu_count() or 1
        set_threads(cores)
        gs = grid((128, 128, 128))
        us, vs, ws, ps, _ = case(gs, 1)
        o = OracleSimulation(spec(gs))
        o.advect_positive(us, vs, ws, ps, dt)
        k = max(1, min(args.steps, 3))
        t0 = time.perf_counter()
        for _ in range(k):
            o.advect_positive(us, vs, ws, ps, dt)
        el = (time.perf_counter() - t0) / k
        rate = gs.ncells / el
        line.update({"impl": "reference", "value": rate, "n_gpus": args.gpus, "steps": k, "warmup": 1,
                     "ms_per_step": 1e3 * el, "dtype": "f64",
                     "cpu_baseline": {"value": rate, "unit": "cell-updates/s", "cores": cores, "kind": "port",
                                      "sample": f"{k} calls on a 128^3 sample of the workload, FP64 oracle, "
                                                f"{cores} OpenMP threads"},
                     "e2e": {"value": rate, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                             "d2h_bytes_per_step": 0}})
        print(json.dumps(line), flush=True)
        return 0
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    from aeolus_b200.simulation import Simulation
    hbm, hbm_kind = measured_peaks()
    res = {}
    for prec, dtype, word in (("fp32_mixed", torch.float32, 4), ("fp64", torch.float64, 8)):
        s = Simulation(spec(g, prec), device=local)
        dev = [torch.from_numpy(a).to(dtype).cuda() for a in (u, v, w, phi)]
        tend = torch.zeros(g.storage_shape, dtype=dtype, device="cuda")
        stream = torch.cuda.ExternalStream(s.stream)
        for _ in range(args.warmup):
            s.advect_positive_device(*dev, tend, dt)
        clk = ClockSampler(local)
        clk.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.synchronize()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            s.advect_positive_device(*dev, tend, dt)
        e1.record(stream)
        s.synchronize()
        clocks = clk.stop()
        ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
        # e2e: the host-array entry point (u, v, w, phi, tend up, tend down)
        t0 = time.perf_counter()
        ke = max(2, min(args.steps, 5))
        out = np.zeros(g.storage_shape)
        for _ in range(ke):
            out = s.advect_positive(u, v, w, phi, dt, tend=out)
        e2e_ms = 1e3 * (time.perf_counter() - t0) / ke
        res[prec] = dict(ms=ms, e2e_ms=e2e_ms, clocks=clocks, word=word)
        s.close()
    if rank != 0:
        return 0
    m = res["fp32_mixed"]
    # algorithmic bytes: read u, v, w, phi and tend, write tend (the fluxes and
    # ratios between the three kernels are the implementation's own traffic)
    byts = 6 * m["word"] * ncell
    ach = byts / (m["ms"] * 1e-3) / 1e9
    hb = 5 * 8 * int(np.prod(g.storage_shape))
    line.update({"value": world * ncell / (m["ms"] * 1e-3), "n_gpus": world, "steps": args.steps,
                 "warmup": args.warmup, "ms_per_step": m["ms"], "dtype": "f32 (FP32 arithmetic on FP32 arrays)",
                 "fp64": {"value": world * ncell / (res["fp64"]["ms"] * 1e-3), "ms_per_step": res["fp64"]["ms"]},
                 "e2e": {"value": ncell / (m["e2e_ms"] * 1e-3), "unit": "cell-updates/s",
                         "h2d_bytes_per_step": hb, "d2h_bytes_per_step": 8 * int(np.prod(g.storage_shape))},
                 "roofline": {"bound": "hbm", "kernel": "advect_positive (three kernels, whole call)",
                              "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s", "frac": round(ach / hbm, 4),
                              "peak_kind": hbm_kind, "bytes_per_launch": byts, "traffic": None},
                 "gpu_launches": 3 * args.steps, "clocks": m["clocks"]})
    print(json.dumps(line), flush=True)
    return 0


URBAN_STEP_N = (1024, 1024, 192)


def urban_step_case(n, nboxes, seed=1, core="anelastic"):
    """The large urban convective case: n cells of 2 m horizontally, `nboxes`
    floor-standing boxes (Philox-seeded centres, footprints U(10, 40) m,
    heights U(10, 60) m) as a solid mask (a cell is solid when its centre is
    inside a box) and its staircase geometry (0/1 apertures, the obstacle
    model of the urban cases), surface heat flux 0.15 K m/s, Smagorinsky
    C_s = 0.17, the projection by the multigrid-preconditioned CG on the
    cut-cell apertures, dt = 1 s.  core = "anelastic" (the configuration):
    the sound-proof core on a tanh-stretched column (first cell 2 m, depth
    2.5 m x nz), rho0 = 1.2 exp(-z/8000), theta_bar = 300 K, the
    density-weighted cut-cell projection, centred advection (the reference
    defines WENO on uniform Boussinesq grids only).  core = "boussinesq":
    the uniform 2 m column with theta0 = 300 K and WENO-JS5.  Initial state:
    at rest, theta = 300 K plus seeded uniform +-0.1 K noise in the lowest
    10 levels.  Returns the grid, the apertures, the fluid mask, a spec
    maker, the state and a description."""
    from aeolus_b200 import CoreSpec, regular_grid, stretched_grid, tanh_beta_for_first_cell, tanh_faces
    from aeolus_b200.cutcell import box_solid_mask, face_coefficients, random_boxes, staircase_geometry
    from aeolus_b200.inputs import philox_uniform
    from aeolus_b200.reference_state import anelastic_profiles, exponential_density
    nx, ny, nz = n
    if core == "anelastic":
        lz = 2.5 * nz
        beta = tanh_beta_for_first_cell(nz, lz, URBAN_H)
        g = stretched_grid(n, (URBAN_H * nx, URBAN_H * ny, lz), tanh_faces(nz, lz, beta))
        prof = anelastic_profiles(g, exponential_density(g), np.full(nz, 300.0))
    else:
        g = regular_grid(n, tuple(URBAN_H * v for v in n), halo=(3, 3, 3), bc_z="wall")
    geom = staircase_geometry(g, box_solid_mask(g, random_boxes(g, nboxes, seed=seed)))
    ap = face_coefficients(geom, power=1)
    fluid = ~geom.is_solid[g.interior]
    del geom
    kn = min(10, nz)
    th = np.full(g.storage_shape, 300.0)
    hx, hy, hz = g.halo
    th[hz:hz + kn, hy:hy + ny, hx:hx + nx] += (
        0.1 * (2.0 * philox_uniform(seed, 3, nx * ny * kn) - 1.0)).reshape(kn, ny, nx)
    zero = g.zeros()
    state = (zero, zero, zero, th)

    def mkspec(prec):
        if core == "anelastic":
            return CoreSpec(grid=g, core="anelastic", c_s=0.17, nu=0.0, flux_bot=0.15, solver="pcg",
                            precision=prec, wc=prof["wc"], wf=prof["wf"], thf=prof["thf"])
        return CoreSpec(grid=g, advection="weno_js5", c_s=0.17, nu=0.0, theta0=300.0, flux_bot=0.15,
                        solver="pcg", precision=prec)

    if core == "anelastic":
        dz = np.diff(g.zf)
        column = (f"anelastic, tanh-stretched z ({nz} levels over {lz:.0f} m, dz {dz[0]:.2f} -> {dz[-1]:.2f} m, "
                  f"max ratio {float(np.max(dz[1:] / dz[:-1])):.4f}), rho0 = 1.2 exp(-z/8000), theta_bar 300 K, "
                  "centred advection + Smagorinsky 0.17, density-weighted cut-cell MG-PCG projection")
    else:
        column = "Boussinesq (theta0 300 K), uniform 2 m z, WENO-JS5 + Smagorinsky 0.17, cut-cell MG-PCG projection"
    desc = {"workload": f"urban convective {nx}x{ny}x{nz} at 2 m, {nboxes} boxes (seed {seed}, footprints "
                        "U(10,40) m, heights U(10,60) m, staircase solid mask), heated surface 0.15 K m/s, "
                        f"{column} to 1e-8, dt = 1 s",
            "grid": [nx, ny, nz], "core": core, "solid_fraction": round(float(1.0 - fluid.mean()), 4),
            "l2": "inputs larger than L2"}
    return g, ap, fluid, mkspec, state, desc


def urban_step_learned(sim, n, fluid, dt, k):
    """The learned U-Net preconditioner in the FP32-mixed step: trained on the
    GPU as for the urban pressure problem (2000 residual -> error pairs of
    128 x 128 x 48 problems, seeds 101..120), transferred to this grid with
    its fluid mask; k steps timed, the last solve's statistics."""
    import torch
    from aeolus_b200.learned import train_streaming, transfer
    t0 = time.perf_counter()
    net, losses, used = train_streaming((128, 128, 48), seeds=range(101, 121), rhs_per_geometry=10, nboxes=10,
                                        pairs_total=2000)
    train_s = time.perf_counter() - t0
    big = transfer(net, n, fluid.astype(np.float32))
    sim.set_learned(big, 0.9)
    sim.step_rk3(dt, 1)
    stream = torch.cuda.ExternalStream(sim.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sim.synchronize()
    e0.record(stream)
    sim.step_rk3_async(dt, k)
    e1.record(stream)
    sim.synchronize()
    ms = e0.elapsed_time(e1) / k
    prof = sim.profile_step(dt)
    st = sim.pcg_stats()
    sim.set_learned(None)
    return {"ms_per_step": ms, "solve_ms": prof["zsolve"] / 3, "iterations_last_solve": st["iterations"],
            "status": st["status"], "relative_residual": st["relative_residual"],
            "training": {"pairs": used, "seconds": round(train_s, 1),
                         "loss_first50": float(losses[:50].mean()), "loss_last50": float(losses[-50:].mean())},
            "unet_forward_ms": big.profile("forward", 3)}


def run_b200_urban_step(args):
    world, rank, local = dist_setup()
    import torch
    torch.cuda.set_device(local)
    from aeolus_b200.simulation import Simulation
    n = tuple(args.urban_n) if args.urban_n else URBAN_STEP_N
    nboxes = args.urban_boxes
    t0 = time.perf_counter()
    g, ap, fluid, mkspec, state, desc = urban_step_case(n, nboxes, core=args.urban_core)
    setup_s = time.perf_counter() - t0
    hbm, hbm_kind = measured_peaks()
    dt, S = 1.0, args.urban_steps
    fields = ("u", "v", "w", "theta")
    res, ref = {}, None
    for prec in ("fp64", "fp32_mixed"):
        sim = Simulation(mkspec(prec), device=local)
        sim.set_pcg(ap, tol=1e-8, maxit=500)
        sim.set_state(*state)
        sim.project()
        # the trajectory: S steps from the common initial state, as one launch of
        # the multi-step graph (a WHILE node over two-step bodies)
        ms_traj = timed_steps(sim, dt, S, world) / S
        fin = [sim.get_field(f)[g.interior].copy() for f in fields]
        ke, div = sim.kinetic_energy(), sim.max_divergence()
        if ref is None:
            ref = fin
            rel = None
        else:
            rel = {f: float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)) for f, a, b in zip(fields, fin, ref)}
        del fin
        sim.step_rk3(dt, args.warmup)
        clk = ClockSampler(local)
        clk.start()
        ms = max_over_ranks(timed_steps(sim, dt, args.steps, world) / args.steps, world)
        clocks = clk.stop()
        prof = sim.profile_step(dt)
        st = sim.pcg_stats()
        launches = sim.launches_per_step()
        e2e_ms, h2d, d2h = e2e_steps(sim, state, dt, 2)   # Float64 host arrays, the reference's Field.data
        out = dict(ms=ms, ms_traj=ms_traj, prof=prof, st=st, launches=launches, clocks=clocks, rel=rel, ke=ke,
                   div=div, e2e_ms=max_over_ranks(e2e_ms, world), h2d=h2d, d2h=d2h)
        if prec == "fp32_mixed" and args.learned:
            out["learned"] = urban_step_learned(sim, n, fluid, dt, max(2, min(args.steps, 5)))
        res[prec] = out
        sim.close()
        del sim
    del ref
    if rank != 0:
        barrier(world)
        return 0
    ncell = g.ncells
    m, d = res["fp32_mixed"], res["fp64"]
    prof = m["prof"]
    per_launch_ms = prof["sweep"] / LAUNCHES_PER_STEP["sweep"]
    sweep_bytes = class_passes("sweep", g, True) * 4 * ncell
    ach = sweep_bytes / (per_launch_ms * 1e-3) / 1e9

    def solve(r):
        return {"ms_per_solve": round(r["prof"]["zsolve"] / 3, 3), "iterations_last_solve": r["st"]["iterations"],
                "status": r["st"]["status"], "relative_residual": r["st"]["relative_residual"]}

    line = {
        "metric": "cell-steps/s", "value": world * ncell / (m["ms"] * 1e-3), "unit": "cell-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": m["ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32-mixed (FP32 stencils and multigrid cycle; FP64 CG vectors, operator, reductions)",
        "data": "synthetic (Philox-seeded boxes and theta noise)",
        "config": dict(desc, parallelism=f"replicas x{world}" if world > 1 else "1 GPU"),
        "pcg": solve(m),
        "fp64": {"value": world * ncell / (d["ms"] * 1e-3), "ms_per_step": d["ms"], "pcg": solve(d),
                 "e2e": world * ncell / (d["e2e_ms"] * 1e-3), "max_divergence": d["div"]},
        "fp32_vs_fp64": {"steps": S, "relative_l2": m["rel"], "ke_fp64": d["ke"], "ke_fp32": m["ke"],
                         "ke_relative_difference": abs(m["ke"] - d["ke"]) / abs(d["ke"]) if d["ke"] else None,
                         "max_divergence_fp32": m["div"], "max_divergence_fp64": d["div"],
                         "trajectory_ms_per_step": {"fp32_mixed": m["ms_traj"], "fp64": d["ms_traj"]},
                         "trajectory_graph_launches": 1 if S >= 2 else S},
        "kernels_ms_per_step": {k: round(v, 3) for k, v in prof.items() if v > 0},
        "e2e": {"value": world * ncell / (m["e2e_ms"] * 1e-3), "unit": "cell-steps/s",
                "h2d_bytes_per_step": m["h2d"], "d2h_bytes_per_step": m["d2h"]},
        "roofline": {"bound": "hbm", "kernel": "sweep", "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
                     "frac": round(ach / hbm, 4), "peak_kind": hbm_kind, "bytes_per_launch": sweep_bytes,
                     "traffic": None},
        "gpu_launches": m["launches"] * args.steps,
        "clocks": m["clocks"],
        "setup_seconds": round(setup_s, 1),
        "learned": m.get("learned"),
    }
    print(json.dumps(line), flush=True)
    barrier(world)
    return 0


def run_reference_urban_step(args):
    """The oracle's cut-cell step (all host threads for the stencils, the
    serial multigrid CG) on a bounded sample of the urban convective case:
    128 x 128 x 48 cells of 2 m holding the case's box density (9 boxes),
    one warm-up step and min(steps, 2) timed steps."""
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    from oracle.oracle import OracleSimulation, set_threads
    n = (128, 128, 48)
    g, ap, fluid, mkspec, state, desc = urban_step_case(n, 9, core=args.urban_core)
    cores = os.cpu_count() or 1
    set_threads(cores)
    o = OracleSimulation(mkspec("fp64"))
    o.set_pcg(ap, tol=1e-8, maxit=500)
    o.set_state(*state)
    o.project()
    o.step_rk3(1.0, 1)
    k = max(1, min(args.steps, 2))
    t0 = time.perf_counter()
    o.step_rk3(1.0, k)
    el = time.perf_counter() - t0
    rate = g.ncells * k / el
    line = {
        "impl": "reference", "metric": "cell-steps/s", "value": rate, "unit": "cell-steps/s", "n_gpus": args.gpus,
        "steps": k, "warmup": 1, "ms_per_step": 1e3 * el / k, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": dict(desc, sample=list(n)),
        "cpu_baseline": {"value": rate, "unit": "cell-steps/s", "cores": cores, "kind": "port",
                         "sample": f"{k} steps of a 128x128x48 sample (9 boxes) after one warm-up, FP64 oracle, "
                                   f"{cores} OpenMP threads for the stencils, serial multigrid CG"},
        "e2e": {"value": rate, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_b200(args):
    world, rank, local = dist_setup()
    import torch
    torch.cuda.set_device(local)
    from aeolus_b200 import _lib
    from aeolus_b200.simulation import Simulation

    g, mkspec, state, dt, desc, _ = workload(args.workload)
    hbm, hbm_kind = measured_peaks()
    results = {}
    for prec in ("fp32_mixed", "fp64"):
        sim = Simulation(mkspec(prec), device=local)
        sim.set_state(*state)
        sim.step_rk3(dt, args.warmup)
        prof = sim.profile_step(dt)           # per-kernel-class device time, one un-graphed step
        sim.step_rk3(dt, 1)
        clk = ClockSampler(local)
        clk.start()
        ms_total = timed_steps(sim, dt, args.steps, world)
        clocks = clk.stop()
        ms_total = max_over_ranks(ms_total, world)
        ms = ms_total / args.steps
        # e2e through the reference's binding: Float64 Field.data host arrays
        ke2e = max(2, min(args.steps, 5))
        e2e_ms, h2d, d2h = e2e_steps(sim, state, dt, ke2e)
        e2e_ms = max_over_ranks(e2e_ms, world)
        r = dict(ms=ms, prof=prof, clocks=clocks, e2e_ms=e2e_ms, h2d=h2d, d2h=d2h,
                 launches=sim.launches_per_step(), div=sim.max_divergence(), ke=sim.kinetic_energy())
        if prec == "fp32_mixed":   # and through the FP32 host mirror of an FP32-mixed domain
            e2e32_ms, h2d32, d2h32 = e2e_steps(sim, state, dt, ke2e, f32=True)
            r.update(e2e32_ms=max_over_ranks(e2e32_ms, world), h2d32=h2d32, d2h32=d2h32)
        results[prec] = r
        sim.close()
        del sim
    # FP32-mixed against FP64 over the configured run (500 steps of 1 s)
    sims = {p: Simulation(mkspec(p), device=local) for p in ("fp64", "fp32_mixed")}
    for sim in sims.values():
        sim.set_state(*state)
    ke0 = {p: sim.kinetic_energy() for p, sim in sims.items()}
    for sim in sims.values():
        sim.step_rk3(dt, args.cbl_steps)
    theta_ref = state[3][g.interior]
    cbl_cmp = ke_change(precision_comparison(sims["fp32_mixed"], sims["fp64"], g, theta_ref=theta_ref),
                        ke0["fp64"], ke0["fp32_mixed"])
    cbl_cmp["ke_growth_relative_difference"] = cbl_cmp["ke_change_relative_difference"]
    cbl_cmp.update({"steps": args.cbl_steps, "t_end": dt * args.cbl_steps})
    for sim in sims.values():
        sim.close()
    del sims
    # the other half of the metric: PCG time to 1e-8 on the urban problem
    coeffs, b, udesc = urban_problem()
    pcg = pcg_solves(coeffs, b, reps=max(3, min(args.steps, 10)))
    for v in pcg.values():
        v["ms"] = max_over_ranks(v["ms"], world)
        del v["handle"]
    # the learned preconditioner on the same problem (trained in this run), beside the plain solves
    learned = None if args.no_learned else learned_pcg(coeffs, b, args)
    # config 3 beside it: decaying isotropic turbulence, FP32-mixed against FP64
    hit = None
    if args.hit_steps > 0:
        hg, hcmp, hres = hit_run(args.hit_n, args.hit_steps, args, local, world)
        hit = {"config": f"decaying isotropic turbulence {args.hit_n}^3, WENO-Z5, no SGS, nu = 0, adaptive dt "
                         f"CFL 0.5 (growth 1.1), Passot-Pouquet spectrum k_p = 4, u_rms = 1, seed 1",
               "value": world * hg.ncells / (hres["fp32_mixed"]["ms"] * 1e-3), "unit": "cell-steps/s",
               "ms_per_step": hres["fp32_mixed"]["ms"],
               "fp64": {"value": world * hg.ncells / (hres["fp64"]["ms"] * 1e-3), "ms_per_step": hres["fp64"]["ms"]},
               "adaptive_ms_per_step": {"fp32_mixed": hres["fp32_mixed"]["adaptive_ms"],
                                        "fp64": hres["fp64"]["adaptive_ms"]},
               "fp32_vs_fp64": hcmp, "clocks": hres["fp32_mixed"]["clocks"]}
        hprof = hres["fp32_mixed"]["prof"]
        if hprof.get("sweep", 0) > 0:
            hb = class_passes("sweep", hg, False) * 4 * hg.ncells
            hach = hb / (hprof["sweep"] / LAUNCHES_PER_STEP["sweep"] * 1e-3) / 1e9
            hbm_h, hbm_kind_h = measured_peaks()
            hit["roofline"] = {"bound": "hbm", "kernel": "sweep (sweep_wpair_kernel)", "achieved": round(hach, 1),
                               "peak": hbm_h, "unit": "GB/s", "frac": round(hach / hbm_h, 4),
                               "peak_kind": hbm_kind_h, "bytes_per_launch": hb}
    if rank != 0:
        barrier(world)
        return 0
    main = results["fp32_mixed"]
    ncell = g.ncells
    value = world * ncell / (main["ms"] * 1e-3)
    sgs = True
    # roofline of the dominant kernel class
    prof = main["prof"]
    dom = max(prof, key=lambda c: prof[c])
    s = 4  # fp32 words
    passes = class_passes(dom, g, sgs)
    per_launch_ms = prof[dom] / LAUNCHES_PER_STEP[dom]
    bytes_per_launch = passes * s * ncell
    achieved = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9 if per_launch_ms > 0 else 0.0
    kernels = {}
    for c, v in prof.items():
        if v <= 0:
            continue
        pl = v / LAUNCHES_PER_STEP[c]
        b = class_passes(c, g, sgs) * s * ncell
        kernels[c] = {"ms_per_step": round(v, 4), "share": round(v / sum(prof.values()), 4),
                      "GBps_per_launch": round(b / (pl * 1e-3) / 1e9, 1) if b > 0 else None}
    step_bytes = 392.0 * ncell  # FP32-mixed algorithmic bytes per cell-step
    fp64 = results["fp64"]
    line = {
        "metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": main["ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32-mixed (FP32 stencils/FFT, FP64 column solve and reductions)",
        "data": "synthetic (Philox-seeded CBL initial state)",
        "config": dict(desc, parallelism=f"replicas x{world}" if world > 1 else "1 GPU"),
        "fp64": {"value": world * ncell / (fp64["ms"] * 1e-3), "ms_per_step": fp64["ms"],
                 "e2e": world * ncell / (fp64["e2e_ms"] * 1e-3), "max_divergence": fp64["div"]},
        "e2e": {"value": world * ncell / (main["e2e_ms"] * 1e-3), "unit": "cell-steps/s",
                "h2d_bytes_per_step": main["h2d"], "d2h_bytes_per_step": main["d2h"],
                "host_arrays": "Float64 storage arrays (the reference's Field.data) through aeo_set_field / "
                               "aeo_get_field, pinned"},
        "e2e_fp32_host": {"value": world * ncell / (main["e2e32_ms"] * 1e-3), "unit": "cell-steps/s",
                          "h2d_bytes_per_step": main["h2d32"], "d2h_bytes_per_step": main["d2h32"],
                          "host_arrays": "Float32 mirrors through aeo_set_field_f32 / aeo_get_field_f32"},
        "fp32_vs_fp64": cbl_cmp,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": hbm,
                     "unit": "GB/s", "frac": round(achieved / hbm, 4), "peak_kind": hbm_kind,
                     "bytes_per_launch": bytes_per_launch, "traffic": CBL_SWEEP_DRAM_BYTES,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one sweep launch of "
                                       "this workload (profiles/sweep_pair_kernel_cbl256_fp32.md)"},
        "step_roofline": {"algorithmic_bytes_per_cell_step": 392, "achieved_GBps": round(
            step_bytes / (main["ms"] * 1e-3) / 1e9, 1), "frac": round(step_bytes / (main["ms"] * 1e-3) / 1e9 / hbm, 4)},
        "kernels": kernels,
        "gpu_launches": main["launches"] * args.steps,
        "clocks": main["clocks"],
        "max_divergence": main["div"],
        "pcg": {"metric": "PCG time-to-1e-8", "unit": "ms", "config": udesc,
                "plain_fp32_mixed": pcg["fp32_mixed"], "plain_fp64": pcg["fp64"], "learned": learned},
        "hit": hit,
    }
    if world == 1 and not args.no_cpu_baseline:
        rate, cores, n, el = cpu_oracle_rate(mkspec("fp64"), state, dt)
        rate1, _, n1, el1 = cpu_oracle_rate(mkspec("fp64"), state, dt, threads=1, min_seconds=8.0, max_steps=2)
        line["cpu_baseline"] = {"value": rate, "unit": "cell-steps/s", "cores": cores, "kind": "port",
                                "cpu_model": cpu_model(),
                                "sample": f"{n} RK3 steps of the full grid ({el:.1f} s), FP64 oracle, "
                                          f"{cores} OpenMP threads",
                                "one_thread": {"value": rate1, "sample": f"{n1} RK3 steps of the full grid "
                                                                         f"({el1:.1f} s), 1 thread"}}
    print(json.dumps(line), flush=True)
    barrier(world)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="cbl", choices=["cbl", "tgv", "urban", "hit", "urban_step", "tracer"])
    ap.add_argument("--tracer-n", type=int, default=256)
    ap.add_argument("--hit-n", type=int, default=512)
    ap.add_argument("--hit-steps", type=int, default=200)
    ap.add_argument("--cbl-steps", type=int, default=500)
    ap.add_argument("--urban-n", type=int, nargs=3, default=None)
    ap.add_argument("--urban-boxes", type=int, default=600)
    ap.add_argument("--urban-steps", type=int, default=10)
    ap.add_argument("--urban-core", default="anelastic", choices=["anelastic", "boussinesq"])
    ap.add_argument("--learned", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--learned-steps", type=int, default=200)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "urban":
        rc = run_reference_urban(args) if args.impl == "reference" else run_b200_urban(args)
    elif args.workload == "tracer":
        rc = run_tracer(args)
    elif args.workload == "urban_step":
        rc = run_reference_urban_step(args) if args.impl == "reference" else run_b200_urban_step(args)
    elif args.workload == "hit":
        rc = run_reference_hit(args) if args.impl == "reference" else run_b200_hit(args)
    else:
        rc = run_reference(args) if args.impl == "reference" else run_b200(args)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
