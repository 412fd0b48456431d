#!/usr/bin/env python
"""Benchmark: FP64 zone-cycles/s of KORAL's per-step hot path on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload ot128]

A step is one full time step of the workload (RK2, ko.c:571-626: two explicit
operators and two inversions with fixups and boundary conditions; RK2IMEX,
ko.c:444-570, with radiation).  Workloads:

  radtorus  (default) the torus below on 256x128x64 with M1 radiation: a step
          is one RK2IMEX step (implicit source solve in every substep,
          batched solver with the learned warm start, one CUDA graph per
          step); the line adds the same steps without the network, with the
          persistent solver and with one thread per cell, and the flow's own
          one-ulp sensitivity over those steps
  torus   3D magnetised Kerr torus, 192x96x64: spin 0.9, MKS2
          coordinates, r in [1.8, 1000], Fishbone-Moncrief torus r_in = 6,
          r_max = 12, Gamma = 13/9, beta_min = 100, 2% seeded pressure noise,
          density floor 1e-4 r^-1.5, MP5 + HLL + flux-CT, RK2, CFL 0.5
  ot128   relativistic Orszag-Tang vortex, 128x128, PPM + LLF + flux-CT,
          Minkowski, Gamma = 5/3, CFL 0.5 (the reference's CPU-runnable case)
  radcells  2^22 independent radiating cells: a step is one batched implicit
          gas-radiation source solve (metric "implicit solves/s"); the line
          adds the one-thread-per-cell form, the learned warm start and the
          MHD inversion's learned warm start

value  = cells x timed steps / device time (CUDA events on the library's own
         stream, L2 flushed between steps, inputs resident in HBM)
e2e    = same metric through the C-ABI with host buffers: every step uploads
         u and p from pinned host memory, runs the step and downloads u and p
N > 1  : one process per GPU (torchrun), each rank runs its own replica of the
         workload (the path is one subdomain per GPU: replicas only), device
         time is the maximum over ranks, value counts the cells of all ranks.
--impl reference times the reference KORAL sources themselves (oracle/_ref,
OpenMP build) on the host cores, same workload and metric.
The line also carries the roofline of the dominant kernel (HBM, and FP64
for the face flux), the per-kernel shares, the clocks sampled during the
timed region and the set-up time of the workload (metric and initial state
computed on the device).
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FP64 zone-cycles/s (1 B200)"
UNIT = "zone-cycles/s"

WORKLOADS = {
    "torus": dict(desc="3D magnetised Kerr torus 192x96x64 (a=0.9 MKS2, FM torus r_in=6 r_max=12, Gamma 13/9, "
                       "beta_min 100, 2% noise, MP5+HLL+flux-CT, RK2, CFL 0.5)",
                  shape=(192, 96, 64), ref_lib="libkref_fmtorus_omp.so", ref_serial="libkref_fmtorus.so",
                  ref_sample_steps=4, ref_max_steps=20, ref_max_warmup=5),
    "ot128": dict(desc="relativistic Orszag-Tang vortex 128x128 (Minkowski, PPM+LLF+flux-CT, RK2, CFL 0.5, Gamma 5/3)",
                  shape=(128, 128, 1), ref_lib="libkref_orszagrel_128_omp.so", ref_serial="libkref_orszagrel_128.so",
                  ref_sample_steps=40, ref_max_steps=100, ref_max_warmup=10),
    "radtorus": dict(desc="3D magnetised radiative Kerr torus 256x128x64 (the torus above plus M1 radiation in LTE "
                          "with the gas at one temperature, Kramers + electron scattering, M = 1e16 Msun, faint "
                          "atmosphere radiation 1e-6 u; MP5+HLL+flux-CT, RK2IMEX with the implicit source solve "
                          "every substep, batched solver + learned warm start, one CUDA graph per step, CFL 0.5)",
                     shape=(256, 128, 64), ref_lib="libkref_radtorus_omp.so", ref_serial="libkref_radtorus_omp.so",
                     ref_sample_lib="libkref_radtorus_wedge_omp.so", ref_sample_desc="a 256x128x8 phi wedge of the "
                     "torus (its first 8 of 64 phi columns, same cells, periodic in phi)",
                     ref_max_steps=40, ref_max_warmup=5, radiation=True),
    "radcells": dict(desc="batched implicit gas-radiation source solve, 2^22 independent cells (Kerr-Schild a=0.9, "
                          "r log-U[2,100] M, theta U[0.1,pi-0.1], log-U rho [1e-8,1], T [1e4,1e12] K, "
                          "E_rad/rho [1e-10,1e2], tau [1e-3,1e5], gas Lorentz factor [1,20], flux fraction [0,0.99], "
                          "Kramers + electron scattering, M = 10 Msun, Gamma 13/9, Newton to 1e-10, seed 2026)",
                     ncells=1 << 22, ref_lib="libkref_radcells_omp.so", ref_serial="libkref_radcells.so",
                     ref_sample_cells=1 << 17),
}
RAD_METRIC = "implicit solves/s (1 B200)"

# From the ncu capture of the x-face flux kernel on the 192x96x64 torus
# (profiles/k_flux_x_torus_192x96x64.md): FP64 operations per face (DADD +
# DMUL + 2 DFMA thread instructions / faces).  That capture's DRAM bytes
# (971 MB per launch, mostly register spill) belong to the build before the
# magnetic floor moved to k_flux_fix, which cut the spills; the current
# build's traffic has not been captured, so the line reports none.
FLUX_FP64_PER_FACE = 1895.5


def flux_roofline(prof, nx, ny, nz, hbm_peak, peak_src, fp64_peak):
    """HBM roofline of the x-face flux (algorithmic bytes 16 NV per face
    over the event time of k_flux_x and its magnetic-floor pass k_flux_fix,
    timed as one), and its FP64 rate."""
    nfaces = (nx + 1) * (ny + 2) * (nz + 2)
    flux_ms = prof["k_flux_x"][0] / max(1, prof["k_flux_x"][1])
    flux_gbs = 16 * 9 * nfaces / (flux_ms / 1e3) / 1e9 if flux_ms > 0 else None
    tflops = FLUX_FP64_PER_FACE * nfaces / (flux_ms / 1e3) / 1e12 if flux_ms > 0 else None
    return {"kernel": "k_flux_x", "bound": "hbm", "achieved": flux_gbs, "peak": hbm_peak, "unit": "GB/s",
            "frac": (flux_gbs / hbm_peak) if flux_gbs else None,
            "traffic": None,
            "traffic_source": "not captured for this build (the previous build's 971 MB per launch was "
                              "register spill; deferring the magnetic floor cut the spill loads 4.5x)",
            "peak_source": peak_src, "algorithmic_bytes_per_launch": 16 * 9 * nfaces,
            "fp64": {"achieved_tflops": tflops, "peak_tflops": fp64_peak,
                     "frac": (tflops / fp64_peak) if (tflops and fp64_peak) else None,
                     "flop_per_face": FLUX_FP64_PER_FACE,
                     "note": "the kernel is FP64-latency bound: 13.1 FLOP per algorithmic byte"}}


def fp64_peak_tflops(k):
    peak = ctypes.c_double()
    k._check(k.lib().kgpu_fp64_peak(ctypes.byref(peak)), "kgpu_fp64_peak")
    return peak.value / 1e12
RAD_UNIT = "solves/s"


def max_over_ranks(x, dist, device):
    """The largest value of x over all ranks (x itself on a single rank);
    every rank takes part and receives the result."""
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, steps, world, ms_slowest):
    """Units of all ranks per second, over the slowest rank's time."""
    return units_per_rank * steps * world / (ms_slowest / 1e3)


def make_subdomain(kgpu, name):
    """The workload's subdomain; its set-up time (context allocation, grid,
    metric tables and initial state computed on the device, boundaries,
    first dt) is kept as s.setup_s."""
    wl = WORKLOADS[name]
    nx, ny, nz = wl["shape"]
    t0 = time.perf_counter()
    if name == "torus":
        s = kgpu.fm_torus(nx, ny, nz)
    elif name == "radtorus":
        s = kgpu.radtorus(nx, ny, nz)
    else:
        s = kgpu.orszag_tang(nx)
    s.setup_s = time.perf_counter() - t0
    return s


def setup_record(s):
    return {"seconds": s.setup_s, "where": "device",
            "covers": "context allocation, grid, metric tables and initial state computed on the device, "
                      "boundaries, first dt"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="radtorus", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-solve", choices=["plain", "batched", "persistent"], default=None,
                    help="a profiling aid: radtorus: after the warm-up steps solve the cells of the last implicit "
                         "step again with this solver; radcells: solve the first cells of the batched-solve "
                         "distribution; print the solver's counters as JSON (no bench line)")
    ap.add_argument("--profile-cells", type=int, default=0,
                    help="with --profile-solve: solve only the first this many cells (0: all)")
    ap.add_argument("--profile-file", default=None,
                    help="with --profile-solve on the radiative torus: the cells are read from this .npz when it "
                         "exists (no warm-up steps), else written to it after the warm-up")
    return ap.parse_args()


def profile_solve(args):
    """A profiling aid for the implicit solve.  Radiative torus: after the
    warm-up steps, the cells of the last implicit step (their inputs, as the
    step gathered them; the first --profile-cells of them, or all); batched-
    solve workload: the first --profile-cells cells of its distribution
    (seed 2026).  They are solved once
    with the given solver through kgpu_rad_implicit_cells_device_ex, for an
    ncu capture of its kernels; prints the solver's counters (solves, Newton
    iterations, residual evaluations, nested inversion work) and its event
    time as JSON, so that per-evaluation figures can be formed from the
    capture."""
    import torch
    import koral_b200 as k
    from koral_b200 import build
    build.build()
    torch.cuda.set_device(0)
    if args.workload == "radcells":
        rp = k.rad_params()
        m = args.profile_cells if args.profile_cells > 0 else WORKLOADS["radcells"]["ncells"]
        d = [torch.from_numpy(a).cuda() for a in k.rad_cells(m, 2026, rp)]
    elif args.profile_file and os.path.exists(args.profile_file):
        import numpy as np
        f = np.load(args.profile_file)
        m = args.profile_cells if args.profile_cells > 0 else f["uu"].shape[0]
        d = [torch.from_numpy(f[key][:m]).cuda() for key in ("uu", "pp", "g", "G", "dt")]
        rp = k.rad_params(mass=k.RADTORUS_MASS, gamma=13.0 / 9.0)
    else:
        s = make_subdomain(k, "radtorus")
        mlp, _ = warmstart_network(k)
        s.set_implicit_options(warm_attempts=WARM_ATTEMPTS_RADTORUS, skip=SKIP_RADTORUS)
        s.set_implicit_solver(k.RAD_BATCHED, mlp)
        s.rk2imex_steps(max(1, args.warmup), graph=True)
        n, b = s.implicit_buffers()
        m = min(n, args.profile_cells) if args.profile_cells > 0 else n

        class Dev:
            def __init__(self, ptr, shape):
                self.__cuda_array_interface__ = {"shape": shape, "typestr": "<f8", "data": (ptr, False),
                                                 "version": 3}

        d = [torch.as_tensor(Dev(b[key], shape), device="cuda")[:m].clone()
             for key, shape in (("uu_in", (n, 13)), ("pp_in", (n, 13)), ("g20", (n, 20)), ("G20", (n, 20)),
                                ("dt", (n,)))]
        rp = s._rp
        s.close()
        if args.profile_file:
            import numpy as np
            np.savez(args.profile_file, **{key: t.cpu().numpy() for key, t in zip(("uu", "pp", "g", "G", "dt"), d)})
    mode = {"plain": k.RAD_PLAIN, "batched": k.RAD_BATCHED, "persistent": k.RAD_PERSISTENT}[args.profile_solve]
    torch.cuda.synchronize()
    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    out = k.rad_solve_device(rp, *d, mode=mode, nstats=7)
    e.record()
    torch.cuda.synchronize()
    st = out[5]
    print(json.dumps({"solver": args.profile_solve, "warmup_steps": args.warmup, "cells": m, "ms": a.elapsed_time(e),
                      "newton_iterations": int(st[0]), "launches_with_work": int(st[1]), "evaluations": int(st[3]),
                      "nested_newton_steps": int(st[4]), "nested_w_evaluations": int(st[5]),
                      "evaluations_handed_to_a_warp": int(st[6])}))


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.samples.append([x.strip() for x in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit())
        mx = max(float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, nm in enumerate(names):
                if len(s) > 5 + k and s[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# reference CPU path (oracle/_ref builds of the reference sources)
# ---------------------------------------------------------------------------
REF_CHILD = r"""
import ctypes, json, os, sys, time
sys.path.insert(0, {root!r})
from oracle.koral_oracle import RefKoral
R = RefKoral({lib!r}); R.init()
R.step({warm})
t0 = time.perf_counter(); R.step({steps}); t1 = time.perf_counter()
print(json.dumps({{"seconds": t1 - t0, "cells": R.nx * R.ny * R.nz, "steps": {steps}}}))
"""


def run_reference_cpu(wl, steps, warm, threads):
    lib = wl["ref_lib"] if threads > 1 else wl["ref_serial"]
    path = os.path.join(ROOT, "oracle", "_ref", lib)
    if not os.path.exists(path):
        return None, f"{lib} not built (needs the reference tree at build time)"
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    code = REF_CHILD.format(root=ROOT, lib=lib, warm=warm, steps=steps)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=1800)
    line = [l for l in r.stdout.splitlines() if l.startswith("{")]
    if r.returncode != 0 or not line:
        return None, (r.stderr or r.stdout)[-300:]
    d = json.loads(line[-1])
    return d["cells"] * d["steps"] / d["seconds"], None


RAD_REF_CHILD = r"""
import json, sys, time
import numpy as np
sys.path.insert(0, {root!r})
import koral_b200 as k
from oracle.koral_oracle import RefRadCells, _p, _i
R = RefRadCells({lib!r})
rp = k.rad_params()
pp, g, G, tau = k.rad_cell_draws({n}, 2026, rp)
uu, kabs, kes = R.prepare(pp, g, G)
dt = 0.5 * tau / (kabs + kes)
st = np.zeros({n}, np.int32)
B = R.batch
t0 = time.perf_counter()
for s in range(0, {n}, B):
    m = min(B, {n} - s)
    R.L.kref_rad_implicit_timed(m, _p(uu[s:]), _p(pp[s:]), _p(g[s:]), _p(G[s:]), _p(dt[s:]), _i(st[s:]))
t1 = time.perf_counter()
print(json.dumps({{"seconds": t1 - t0, "cells": {n}, "ok": float(np.mean(st == 0))}}))
"""


def run_reference_radcells(wl, ncells, threads):
    lib = wl["ref_lib"] if threads > 1 else wl["ref_serial"]
    path = os.path.join(ROOT, "oracle", "_ref", lib)
    if not os.path.exists(path):
        return None, f"{lib} not built (needs the reference tree at build time)"
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    code = RAD_REF_CHILD.format(root=ROOT, lib=lib, n=ncells)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=1800)
    line = [l for l in r.stdout.splitlines() if l.startswith("{")]
    if r.returncode != 0 or not line:
        return None, (r.stderr or r.stdout)[-300:]
    d = json.loads(line[-1])
    return d["cells"] / d["seconds"], None


def cells_of(wl):
    nx, ny, nz = wl["shape"]
    return nx * ny * nz


def reference_arm_radcells(args, wl, threads):
    n = wl["ref_sample_cells"]
    val, err = run_reference_radcells(wl, n, threads)
    if val is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return
    line = {
        "metric": RAD_METRIC, "value": val, "unit": RAD_UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": wl["ncells"] / val * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl["desc"], "parallelism": "openmp host threads"},
        "cpu_baseline": {"value": val, "unit": RAD_UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{n} cells of the same distribution, one solve_implicit_lab each"},
        "e2e": {"value": val, "unit": RAD_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def reference_arm(args, wl, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    if "ncells" in wl:
        reference_arm_radcells(args, wl, threads)
        return
    # The reference's own time steps on all host cores, from its own initial
    # state: the same W warm-up steps as the GPU arm (capped where a CPU step
    # takes long), then the timed steps, at most ref_max_steps of them;
    # "steps" and "warmup" report what was run.  The radiative torus runs on
    # a phi wedge (its first 8 of 64 phi columns, periodic in phi): a bounded
    # sample of the same cells at the same resolution.
    nsteps = max(1, min(args.steps, wl["ref_max_steps"]))
    warm = max(0, min(args.warmup, wl["ref_max_warmup"]))
    lib = wl.get("ref_sample_lib", wl["ref_lib"])
    val, err = run_reference_cpu(dict(wl, ref_lib=lib), nsteps, warm, threads)
    if val is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return
    sample = wl.get("ref_sample_desc", "the whole grid")
    line = {
        "metric": METRIC, "value": val, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": nsteps, "warmup": warm, "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": cells_of(wl) / val * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl["desc"], "parallelism": "openmp host threads", "sample": sample},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "reference", "cpu": cpu_model(),
                         "sample": f"{nsteps} time steps of {sample} after {warm} warm-up step(s), "
                                   f"reference sources built with gcc -O3 -fopenmp"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def our_arm(args, wl, rank, world, local_rank):
    import numpy as np
    import torch
    import koral_b200

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    from koral_b200 import build
    build.build()

    s = make_subdomain(koral_b200, args.workload)
    ext = torch.cuda.ExternalStream(s.stream, device=dev)
    nx, ny, nz = wl["shape"]
    cells = nx * ny * nz
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # 256 MB > 126 MB L2

    dist = None
    if world > 1:
        import torch.distributed as dist_
        dist = dist_

    def barrier():
        if dist is not None:
            dist.barrier()

    # warm-up (graph capture happens here), then the autotuner's choice of
    # launch shapes on the state reached (the same arithmetic whatever it
    # picks)
    s.rk2_steps(max(1, args.warmup), graph=True)
    tuning = None
    if args.workload == "torus":
        t_tune = time.perf_counter()
        tuned, tune_ms = s.autotune(steps=2)
        tuning = {"chosen": tuned.as_dict(), "seconds": time.perf_counter() - t_tune,
                  "ms_per_step_before": tune_ms[0], "ms_per_step_after": tune_ms[1],
                  "by": "kgpu_autotune on the warmed-up state"}
        s.rk2_steps(1, graph=True)   # capture the step with the chosen shapes

    def timed_steps(k, profile=False):
        """k steps, L2 flushed before each; returns summed device ms."""
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(k)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(k)]
        if profile:
            s.profile(True)
            s.profile_reset()
        for i in range(k):
            with torch.cuda.stream(ext):
                flush.fill_(float(i))
                starts[i].record(ext)
            if profile:
                s.rk2_steps(1, graph=False)
            else:
                s.rk2_steps(1, graph=True)
            with torch.cuda.stream(ext):
                ends[i].record(ext)
        torch.cuda.synchronize(dev)
        if profile:
            s.profile(False)
        return sum(a.elapsed_time(b) for a, b in zip(starts, ends))

    barrier()
    torch.cuda.synchronize(dev)
    launches0 = s.launches
    with ClockSampler(local_rank) as clk:
        ms = timed_steps(args.steps)
    launches = s.launches - launches0
    torch.cuda.synchronize(dev)
    ms_max = max_over_ranks(ms, dist, dev)
    value = whole_job_rate(cells, args.steps, world, ms_max)

    # per-kernel device times (events around each launch, separate pass)
    timed_steps(min(args.steps, 50), profile=True)
    prof = s.profile_read()
    total = sum(v[0] for v in prof.values())
    top = max(prof.items(), key=lambda kv: kv[1][0])

    # e2e through the C-ABI with pinned host buffers
    shape = s.shape
    hu = torch.empty(shape, dtype=torch.float64, pin_memory=True)
    hp = torch.empty(shape, dtype=torch.float64, pin_memory=True)
    u0, p0 = s.download_state()
    hu.numpy()[...] = u0
    hp.numpy()[...] = p0
    L = koral_b200.lib()
    dp = ctypes.POINTER(ctypes.c_double)
    pu = ctypes.cast(hu.data_ptr(), dp)
    pp = ctypes.cast(hp.data_ptr(), dp)
    ke = max(1, min(args.steps, 100))
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(ext):
        e0.record(ext)
    for _ in range(ke):
        koral_b200._check(L.kgpu_upload_state(s.h, pu, pp), "upload")
        koral_b200._check(L.kgpu_rk2_steps(s.h, 1), "step")
        koral_b200._check(L.kgpu_download_state(s.h, pu, pp), "download")
    with torch.cuda.stream(ext):
        e1.record(ext)
    torch.cuda.synchronize(dev)
    e2e_value = whole_job_rate(cells, ke, world, max_over_ranks(e0.elapsed_time(e1), dist, dev))
    state_bytes = 2 * int(np.prod(shape)) * 8

    if rank != 0:
        return
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    # algorithmic bytes of the face-flux kernels: 16*NV bytes per face
    # (read the primitives once, write the face flux once)
    nv = 9
    nfaces = (nx + 1) * (ny + 2 if ny > 1 else 1) * (nz + 2 if nz > 1 else 1)
    flux_ms = prof["k_flux_x"][0] / max(1, prof["k_flux_x"][1])
    flux_gbs = 16 * nv * nfaces / (flux_ms / 1e3) / 1e9 if flux_ms > 0 else None
    roof = (flux_roofline(prof, nx, ny, nz, hbm_peak, peak_src, fp64_peak_tflops(koral_b200))
            if args.workload == "torus" else
            {"kernel": "k_flux_x", "bound": "hbm", "achieved": flux_gbs, "peak": hbm_peak, "unit": "GB/s",
             "frac": (flux_gbs / hbm_peak) if flux_gbs else None, "traffic": None, "peak_source": peak_src,
             "algorithmic_bytes_per_launch": 16 * nv * nfaces})

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl["desc"], "cells_per_gpu": cells, "l2": "flushed (256 MB write) before every step",
                   "parallelism": "replicas" if world > 1 else "single subdomain", "graph": "one CUDA graph per RK2 step",
                   "tuning": tuning},
        "roofline": roof,
        "kernels": {k: {"ms_per_launch": v[0] / max(1, v[1]), "share": v[0] / total if total else 0.}
                    for k, v in prof.items() if v[1]},
        "top_kernel": top[0],
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "setup": setup_record(s),
    }
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        ns = max(1, wl["ref_sample_steps"] // 2)
        val, err = run_reference_cpu(wl, ns, 1, threads)
        if val is not None:
            line["cpu_baseline"] = {"value": val, "unit": UNIT, "cores": threads, "kind": "reference",
                                    "sample": f"{ns} full RK2 steps of the same workload after 1 warm-up step"}
        else:
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": threads, "kind": "reference",
                                    "sample": f"unavailable: {err}"}
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# our arm, radiative torus (RK2IMEX)
# ---------------------------------------------------------------------------
def warmstart_network(k):
    """The warm-start network for the radiative torus: the weights trained on
    the torus's own implicit solves when present, else those trained on the
    batched-solve distribution."""
    from koral_b200 import train_warmstart as tw
    for name in ("warmstart_radtorus.npz", "warmstart_mlp.npz"):
        path = os.path.join(ROOT, "koral_b200", "data", name)
        if os.path.exists(path):
            return tw.load(k, path), name
    return None, None


# attempts of the cascade a warm-started torus cell runs from the prediction
# before the reference cascade (the torus's solves start close to the
# previous state: past the first two attempts a failed warm start is better
# served by the reference cascade; measured 236 against 365 ms per implicit
# step with all six)
WARM_ATTEMPTS_RADTORUS = 2
# on the torus only the cells the network expects to fail their first
# attempt start from its prediction (kgpu_rad_solver_opts.skip = 2).  With
# skip = 1 (every cell from the prediction, beginning with the attempt the
# network expects to succeed) 10 settled steps (21-30) from one state took
# 146.7 ms per step against 179.0 with skip = 2 and 177.0 without the
# network, but the run from the initial torus reached states where both
# solvers fail 50 times more solves (62074 against 1161 without the network
# over steps 6-105) and every step costs more (11.32 M zone-cycles/s
# against 11.69 M): the prediction sends some cells of the transient to
# another solution of the same equations; skip = 2 keeps the reference's
# start for the cells it expects to succeed
SKIP_RADTORUS = 2
# the implicit solver of the timed radiative-torus steps
MAIN_SOLVER = "batched"
# FP64 work of one residual evaluation of the implicit solve on the torus's
# own cells, nested MHD inversion included: DADD + DMUL + 2 DFMA thread
# instructions of the one-thread-per-cell solver over its counted
# evaluations (ncu capture of the first 262144 cells of the implicit step
# after 3 time steps, profiles/k_rad_plain_fp64_per_evaluation.md)
IMP_FP64_PER_EVAL = 2884.5
# the same figure on the batched-solve cells (the first 65536 of the 2^22,
# seed 2026; profiles/k_rad_plain_fp64_per_evaluation.md)
IMP_FP64_PER_EVAL_CELLS = 2838.5

CPU_REF_CHILD = r"""
import json, sys, time
import numpy as np
sys.path.insert(0, {root!r})
from oracle.koral_oracle import RefKoral
R = RefKoral({lib!r}); R.init()
st = np.load({state!r})
u, p = R.array("u"), R.array("p")
u[...] = st["u"][:u.shape[0]]
p[...] = st["p"][:p.shape[0]]
R.set_scalar("tstepdenmax", float(st["tsd"]))
t0 = time.perf_counter(); R.step({steps}); t1 = time.perf_counter()
print(json.dumps({{"seconds": t1 - t0, "cells": R.nx * R.ny * R.nz, "steps": {steps}}}))
"""


def cpu_baseline_from_state(wl, u, p, tsd, steps, threads):
    """The reference's own time steps on the host cores, started from the
    GPU run's state (its first phi columns, for the wedge build): a bounded
    sample of the same steps the GPU timed."""
    import tempfile
    import numpy as np
    lib = wl.get("ref_sample_lib", wl["ref_lib"])
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", lib)):
        return None, f"{lib} not built (needs the reference tree at build time)"
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "state.npz")
        np.savez(path, u=u, p=p, tsd=tsd)
        code = CPU_REF_CHILD.format(root=ROOT, lib=lib, state=path, steps=steps)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=1800)
    line = [l for l in r.stdout.splitlines() if l.startswith("{")]
    if r.returncode != 0 or not line:
        return None, (r.stderr or r.stdout)[-300:]
    d = json.loads(line[-1])
    return d["cells"] * d["steps"] / d["seconds"], None


def our_arm_radtorus(args, wl, rank, world, local_rank):
    import numpy as np
    import torch
    import koral_b200 as k

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    from koral_b200 import build
    build.build()
    s = make_subdomain(k, args.workload)
    mlp, mlp_name = warmstart_network(k)
    s.set_implicit_options(warm_attempts=WARM_ATTEMPTS_RADTORUS, skip=SKIP_RADTORUS)
    main_mode = {"persistent": k.RAD_PERSISTENT, "batched": k.RAD_BATCHED}[MAIN_SOLVER]
    other_mode, other_name = ((k.RAD_BATCHED, "batched") if main_mode == k.RAD_PERSISTENT
                              else (k.RAD_PERSISTENT, "persistent"))
    ext = torch.cuda.ExternalStream(s.stream, device=dev)
    nx, ny, nz = wl["shape"]
    cells = nx * ny * nz
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # 256 MB > 126 MB L2
    dist = None
    if world > 1:
        import torch.distributed as dist_
        dist = dist_

    def barrier():
        if dist is not None:
            dist.barrier()

    def dmax(ms):
        return max_over_ranks(ms, dist, dev)

    def timed_steps(kk, graph=True, profile=False):
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(kk)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(kk)]
        if profile:
            s.profile(True)
            s.profile_reset()
        for i in range(kk):
            with torch.cuda.stream(ext):
                flush.fill_(float(i))
                starts[i].record(ext)
            s.rk2imex_steps(1, graph=graph and not profile)
            with torch.cuda.stream(ext):
                ends[i].record(ext)
        torch.cuda.synchronize(dev)
        if profile:
            s.profile(False)
        return sum(a.elapsed_time(b) for a, b in zip(starts, ends))

    def restart():
        s.upload_state(u_start.copy(), p_start.copy())
        s.tstepdenmax = tsd_start
        s.reset_counters()

    def leg(mode, warm, kk):
        """kk steps from the saved state with the given solver; device ms,
        solver statistics and the end state"""
        s.set_implicit_solver(mode, warm)
        restart()
        barrier()
        ms = dmax(timed_steps(kk))
        c = s.counters()
        u, _ = s.download_state()
        return ms, c, u

    def newton(c):
        return {"solves": int(c["imp_solves"]), "mean_iterations_per_solve": c["imp_iters"] / max(1, c["imp_solves"]),
                "mean_evaluations_per_solve": c["imp_evals"] / max(1, c["imp_solves"]),
                "mean_nested_inversion_iterations_per_solve": c["imp_inner"] / max(1, c["imp_solves"]),
                "failed_solves": int(c["radimp_failed"]), "fallbacks": int(c["imp_fallbacks"]),
                "evaluations_handed_to_a_warp": int(c["imp_cooperative"]),
                "radiation_corrections": int(c["rad_corrected"])}

    # warm-up from the initial torus (graph capture included), then every leg
    # times the same K steps from the state reached
    s.set_implicit_solver(main_mode, mlp)
    s.rk2imex_steps(max(1, args.warmup), graph=True)
    # launch shapes and solver settings chosen by the autotuner on the state
    # reached (same arithmetic whatever it picks; every leg uses the choice)
    t_tune = time.perf_counter()
    tuned, tune_ms = s.autotune(steps=2)
    tune_s = time.perf_counter() - t_tune
    u_start, p_start = s.download_state()
    tsd_start = s.tstepdenmax
    launches0 = s.launches
    with ClockSampler(local_rank) as clk:
        ms, c_main, u_main = leg(main_mode, mlp, args.steps)
    launches = s.launches - launches0
    value = cells * args.steps * world / (ms / 1e3)
    # the same steps without the network, with the other queued solver and
    # with one thread per cell (the cost per step falls by several times over
    # the first tens of steps, so every leg times the same steps)
    ms_n, c_n, u_n = leg(main_mode, None, args.steps)
    ms_o, c_o, u_o = leg(other_mode, mlp, args.steps)
    ms_p, c_p, u_p = leg(k.RAD_PLAIN, None, args.steps)
    g = s.cfg.ng

    def l1(a, b):
        a, b = a[g:-g, g:-g, g:-g], b[g:-g, g:-g, g:-g]
        return [float(np.abs(a[..., v] - b[..., v]).sum() / (np.abs(b[..., v]).sum() + 1e-300)) for v in range(13)]

    # the flow's own sensitivity: the steps without the network again, from
    # the same state with the gas energy of the densest cell moved by one
    # unit in the last place; the L1 between the two runs is what any
    # last-place change grows to over these steps
    s.set_implicit_solver(main_mode, None)
    u_nudge0 = u_start.copy()
    dom_u = u_nudge0[g:-g, g:-g, g:-g]
    iz, iy, ix = np.unravel_index(np.argmax(p_start[g:-g, g:-g, g:-g, 0]), dom_u.shape[:3])
    dom_u[iz, iy, ix, 1] = np.nextafter(dom_u[iz, iy, ix, 1], np.inf)
    s.upload_state(u_nudge0, p_start.copy())
    s.tstepdenmax = tsd_start
    s.reset_counters()
    barrier()
    timed_steps(args.steps)
    u_nudge, _ = s.download_state()

    def density_l1_by_region(a, b):
        """Shares of the density L1 difference by radius and near the axes
        (MKS2 with R0 = 0: r = exp(x1), x1 uniform in [ln 1.8, ln 1000])."""
        d = np.abs(a[g:-g, g:-g, g:-g, 0] - b[g:-g, g:-g, g:-g, 0])
        tot = d.sum() or 1.
        r = np.exp(np.log(1.8) + (np.arange(nx) + 0.5) * (np.log(1000.) - np.log(1.8)) / nx)
        rh = 1. + np.sqrt(1. - 0.9 * 0.9)
        out = {}
        for lo, hi, tag in ((0., 2. * rh, "r < 2 r_h"), (2. * rh, 10., "2 r_h <= r < 10"), (10., 50., "10 <= r < 50"),
                            (50., 1e9, "r >= 50")):
            m = (r >= lo) & (r < hi)
            out[tag] = float(d[:, :, m].sum() / tot)
        out["within 8 rows of an axis"] = float((d[:, :8].sum() + d[:, -8:].sum()) / tot)
        return out

    # per-kernel device times (events around each launch, stream replay) and
    # the solver's counters over the same steps
    s.set_implicit_solver(main_mode, mlp)
    restart()
    kprof = min(args.steps, 5)
    timed_steps(kprof, profile=True)
    prof = s.profile_read()
    c_prof = s.counters()
    total = sum(v[0] for v in prof.values())
    top = max(prof.items(), key=lambda kv: kv[1][0])

    # e2e through the C-ABI with pinned host buffers
    shape = s.shape
    hu = torch.empty(shape, dtype=torch.float64, pin_memory=True)
    hp = torch.empty(shape, dtype=torch.float64, pin_memory=True)
    hu.numpy()[...] = u_start
    hp.numpy()[...] = p_start
    L = k.lib()
    dp = ctypes.POINTER(ctypes.c_double)
    pu = ctypes.cast(hu.data_ptr(), dp)
    pp = ctypes.cast(hp.data_ptr(), dp)
    ke = args.steps   # the same steps as the device-timed legs
    s.tstepdenmax = tsd_start
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(ext):
        e0.record(ext)
    for _ in range(ke):
        k._check(L.kgpu_upload_state(s.h, pu, pp), "upload")
        k._check(L.kgpu_rk2imex_steps(s.h, 1), "step")
        k._check(L.kgpu_download_state(s.h, pu, pp), "download")
    with torch.cuda.stream(ext):
        e1.record(ext)
    torch.cuda.synchronize(dev)
    e2e_value = cells * ke * world / (dmax(e0.elapsed_time(e1)) / 1e3)
    state_bytes = 2 * int(np.prod(shape)) * 8
    if rank != 0:
        return
    fp64_peak = fp64_peak_tflops(k)
    solve_ms = prof["k_imp_solve"][0]
    roof = {"kernel": "k_imp_solve (" + MAIN_SOLVER + " implicit source solve)", "bound": "fp64",
            "peak": fp64_peak, "unit": "TFLOP/s", "peak_source": "measured live (DMUL+DADD chains, no FMA)",
            "traffic": None, "evaluations": int(c_prof["imp_evals"]), "solve_ms": solve_ms,
            "share_of_step": solve_ms / total if total else None}
    if IMP_FP64_PER_EVAL and solve_ms > 0:
        tf = IMP_FP64_PER_EVAL * c_prof["imp_evals"] / (solve_ms / 1e3) / 1e12
        roof.update(achieved=tf, frac=tf / fp64_peak, flop_per_evaluation=IMP_FP64_PER_EVAL)
    else:
        roof.update(achieved=None, frac=None)
    it_main = c_main["imp_iters"] / max(1, c_main["imp_solves"])
    it_n = c_n["imp_iters"] / max(1, c_n["imp_solves"])
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl["desc"], "cells_per_gpu": cells, "l2": "flushed (256 MB write) before every step",
                   "parallelism": "replicas" if world > 1 else "single subdomain",
                   "graph": "one CUDA graph per RK2IMEX step", "solver": MAIN_SOLVER,
                   "warm_start_weights": mlp_name, "warm_attempts": WARM_ATTEMPTS_RADTORUS,
                   "warm_start_skip": SKIP_RADTORUS,
                   "tuning": {"chosen": tuned.as_dict(), "seconds": tune_s, "ms_per_step_before": tune_ms[0],
                              "ms_per_step_after": tune_ms[1], "by": "kgpu_autotune on the warmed-up state"},
                   "timed_steps": f"{args.warmup + 1}..{args.warmup + args.steps} from the initial torus"},
        "newton": {"learned": newton(c_main), "no_network": newton(c_n),
                   "iteration_ratio_no_network_over_learned": it_n / it_main if it_main > 0 else None},
        "no_network": {"value": cells * args.steps * world / (ms_n / 1e3), "unit": UNIT,
                       "ms_per_step": ms_n / args.steps, "end_state_l1_vs_learned": l1(u_main, u_n),
                       "end_state_l1_one_ulp_nudge": l1(u_nudge, u_n),
                       "one_ulp_nudge": "gas energy of the densest cell moved by one unit in the last place at "
                                        "the start of the timed steps, the same steps without the network",
                       "density_l1_vs_learned_by_region": density_l1_by_region(u_main, u_n),
                       "density_l1_one_ulp_nudge_by_region": density_l1_by_region(u_nudge, u_n)},
        other_name: {"value": cells * args.steps * world / (ms_o / 1e3), "unit": UNIT,
                     "ms_per_step": ms_o / args.steps, "with_network": mlp_name is not None,
                     "same_state_as_main": bool(np.array_equal(u_o, u_main)), "newton": newton(c_o)},
        "plain": {"value": cells * args.steps * world / (ms_p / 1e3), "unit": UNIT,
                  "ms_per_step": ms_p / args.steps, "newton": newton(c_p)},
        "roofline": roof,
        "flux_roofline": flux_roofline(prof, nx, ny, nz, *hbm_peak_of(), fp64_peak),
        "kernels": {kk: {"ms_per_launch": v[0] / max(1, v[1]), "share": v[0] / total if total else 0.}
                    for kk, v in prof.items() if v[1]},
        "top_kernel": top[0],
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "setup": setup_record(s),
    }
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sample = wl.get("ref_sample_desc", "the whole grid")
        nz_s = 8 + 2 * g
        us, ps = u_start[:nz_s].copy(), p_start[:nz_s].copy()
        val, err = cpu_baseline_from_state(wl, us, ps, tsd_start, 2, threads)
        val1, err1 = cpu_baseline_from_state(wl, us, ps, tsd_start, 1, 1)
        line["cpu_baseline"] = {"value": val, "unit": UNIT, "cores": threads, "kind": "reference",
                                "cpu": cpu_model(), "value_1_thread": val1,
                                "sample": (f"2 time steps (and 1 on one thread) of {sample}, from the state the "
                                           f"GPU run reached after {args.warmup} steps: the reference sources "
                                           f"(gcc -O3 -fopenmp) on the host cores"
                                           if val is not None else f"unavailable: {err}")}
    print(json.dumps(line))


def hbm_peak_of():
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    return peaks.get("hbm_gbs", 6650.0), ("measured" if "hbm_gbs" in peaks else "fallback")


# ---------------------------------------------------------------------------
# our arm, batched implicit solve
# ---------------------------------------------------------------------------
def learned_leg(k, rp, d_in, work, stream, n, st_plain, it_plain, all_plain, args, dev):
    """The same solve with the learned warm start (features, network on the
    tensor cores, warm batched solve), timed as a whole, against the plain
    batched solve's iterations on the same cells."""
    import numpy as np
    import torch
    from koral_b200 import train_warmstart
    path = train_warmstart.DEFAULT_OUT
    if not os.path.exists(path):
        return {"unavailable": "no trained weights (python -m koral_b200.train_warmstart)"}
    mlp = train_warmstart.load(k, path)
    uu, pp, g, G, dt = d_in

    def run():
        X = k.rad_features_device(rp, pp, g, G, dt)
        Y = mlp.forward(X)
        return k.rad_solve_device(rp, uu, pp, g, G, dt, ypred=Y, work=work), X, Y

    run()
    torch.cuda.synchronize(dev)
    steps = max(1, min(3, args.steps))
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        out, X, Y = run()
    b.record(stream)
    torch.cuda.synchronize(dev)
    ms = a.elapsed_time(b) / steps
    # the network alone (tensor-core roofline: 2 (16 128 + 128 128 + 128 5) flop per sample)
    a.record(stream)
    for _ in range(10):
        mlp.forward(X)
    b.record(stream)
    torch.cuda.synchronize(dev)
    ms_mlp = a.elapsed_time(b) / 10
    flop = 2 * (16 * 128 + 128 * 128 + 128 * 5) * n
    po, uo, st, at, it, stats = out
    st, it = st.cpu().numpy(), it.cpu().numpy()
    ok = (st == 0) & (st_plain == 0)
    # error of the BF16 prediction against the converged FP64 state
    pred = torch.exp(Y[:, :2].double()).cpu().numpy()
    true = (po[:, [1, 9]] / pp[:, [1, 9]]).cpu().numpy()
    gerr = np.abs(pred - true) / np.abs(true)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    bf16_peak = peaks.get("bf16_tflops", 1590.0)
    at = out[3].cpu().numpy()
    return {"value": n / (ms / 1e3), "unit": RAD_UNIT, "ms_per_step": ms,
            "mean_iterations_all_attempts": stats[0] / n, "plain_mean_iterations_all_attempts": all_plain / n,
            "iteration_ratio": all_plain / max(1, stats[0]),
            "iteration_ratio_note": "Newton iterations per implicit solve over every attempt (failed attempts "
                                    "and the fallback to the reference cascade included), plain over learned",
            "mean_iterations_successful_attempt": float(it[ok].mean()),
            "plain_mean_iterations_successful_attempt": float(it_plain[ok].mean()),
            "iteration_ratio_successful_attempt": float(it_plain[ok].mean() / it[ok].mean()),
            "succeeding_attempt_histogram": {int(a): int((at == a).sum()) for a in np.unique(at)},
            "fallback_rate": stats[2] / n,
            "status_agreement": float(np.mean(st == st_plain)),
            "guess_error_median": {"u_gas": float(np.median(gerr[ok, 0])), "E_rad": float(np.median(gerr[ok, 1]))},
            "mlp": {"ms": ms_mlp, "achieved_tflops": flop / (ms_mlp / 1e3) / 1e12, "peak_tflops": bf16_peak,
                    "frac": flop / (ms_mlp / 1e3) / 1e12 / bf16_peak, "bound": "tensor"}}


def u2p_leg(k, rp, n, stream, dev):
    """The MHD inversion with and without its learned warm start on n
    held-out cells of the warm start's distribution (the batched-solve cells
    with a magnetic field, B^2/rho log-uniform in [1e-3, 1e3], seed 2026):
    the gas state after the plain implicit solve, inverted from the
    primitives before it (calc_u2p's situation after a step that moved the
    gas energy); device time and Newton iterations over all solves of each
    inversion."""
    import numpy as np
    import torch
    from koral_b200 import train_warmstart
    path = train_warmstart.DEFAULT_OUT_U2P
    if not os.path.exists(path):
        return {"unavailable": "no trained weights (python -m koral_b200.train_warmstart --source u2p)"}
    mlp = train_warmstart.load(k, path)
    U, P0, gg, GG = train_warmstart.u2p_cells(k, rp, n, 2026)
    m = U.shape[0]
    cfg = k.u2p_config(rp.gamma)

    def plain():
        return k.u2p_cells_device(cfg, U, P0, gg, GG)

    def learned():
        Y = mlp.forward(k.u2p_features_device(cfg, U, P0, gg, GG))
        return k.u2p_cells_device(cfg, U, P0, gg, GG, ypred=Y)

    res = {}
    for tag, fn in (("plain", plain), ("learned", learned)):
        fn()
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        out = fn()
        b.record(stream)
        torch.cuda.synchronize(dev)
        res[tag] = (a.elapsed_time(b), out)
    (ms_p, op), (ms_l, ol) = res["plain"], res["learned"]
    sp, sl = op[1].cpu().numpy(), ol[1].cpu().numpy()
    return {"inversions": m, "cells": "2^22 batched-solve cells with a magnetic field (sigma 1e-3..1e3, seed 2026) "
                                      "whose plain implicit solve succeeded",
            "plain": {"value": m / (ms_p / 1e3), "unit": "inversions/s",
                                       "mean_iterations": op[4][0] / m, "w_evaluations": op[4][2] / m,
                                       "entropy_rate": float(np.mean(sp == -1))},
            "learned": {"value": m / (ms_l / 1e3), "unit": "inversions/s", "mean_iterations": ol[4][0] / m,
                        "w_evaluations": ol[4][2] / m, "fallback_rate": ol[4][1] / m,
                        "status_agreement": float(np.mean(sp == sl)), "wgate": k.U2P_WGATE, "sgate": k.U2P_SGATE},
            "iteration_ratio": op[4][0] / max(1, ol[4][0]),
            "note": "Newton iterations per inversion over all its solves (energy, entropy, fallback), plain over "
                    "learned; the learned time includes features and network"}


def our_arm_radcells(args, wl, rank, world, local_rank):
    import numpy as np
    import torch
    import koral_b200 as k

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    from koral_b200 import build
    build.build()
    L = k.lib()
    n = wl["ncells"]
    rp = k.rad_params()
    uu, pp, g, G, dt = k.rad_cells(n, 2026 + rank, rp)
    # inputs resident in HBM (2.2 GB, larger than L2)
    d_in = [torch.from_numpy(a).to(dev) for a in (uu, pp, g, G, dt)]
    d_po = torch.empty((n, 13), dtype=torch.float64, device=dev)
    d_uo = torch.empty((n, 13), dtype=torch.float64, device=dev)
    d_st, d_at, d_it = (torch.empty(n, dtype=torch.int32, device=dev) for _ in range(3))
    work = torch.empty(int(L.kgpu_rad_work_bytes(n)), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    vp = ctypes.c_void_p

    def solve(mode, stats=None):
        ptrs = [vp(t.data_ptr()) for t in d_in] + [vp(d_po.data_ptr()), vp(d_uo.data_ptr()), vp(d_st.data_ptr()),
                                                   vp(d_at.data_ptr()), vp(d_it.data_ptr())]
        k._check(L.kgpu_rad_implicit_cells_device(n, ctypes.byref(rp), *ptrs, mode, vp(work.data_ptr()),
                                                  vp(stream.cuda_stream), stats), "kgpu_rad_implicit_cells_device")

    dist = None
    if world > 1:
        import torch.distributed as dist_
        dist = dist_

    def timed(mode, steps):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for a, b in ev:
            a.record(stream)
            solve(mode)
            b.record(stream)
        torch.cuda.synchronize(dev)
        ms = sum(a.elapsed_time(b) for a, b in ev)
        return max_over_ranks(ms, dist, dev)

    for _ in range(args.warmup):
        solve(k.RAD_BATCHED)
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    with ClockSampler(local_rank) as clk:
        ms = timed(k.RAD_BATCHED, args.steps)
    value = n * args.steps * world / (ms / 1e3)
    # the plain one-thread-per-cell form on the same cells, for comparison
    steps_plain = max(1, min(3, args.steps))
    ms_plain = timed(k.RAD_PLAIN, steps_plain)
    plain_value = n * steps_plain * world / (ms_plain / 1e3)
    # iteration statistics of one batched solve, with its residual evaluations
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    sout = k.rad_solve_device(rp, *d_in, mode=k.RAD_BATCHED, work=work, nstats=4)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    ms_one = ev0.elapsed_time(ev1)
    stats = sout[5]
    d_po.copy_(sout[0]), d_uo.copy_(sout[1]), d_st.copy_(sout[2]), d_at.copy_(sout[3]), d_it.copy_(sout[4])
    st = d_st.cpu().numpy()
    it = d_it.cpu().numpy()
    at = d_at.cpu().numpy()
    peak = ctypes.c_double()
    k._check(L.kgpu_fp64_peak(ctypes.byref(peak)), "kgpu_fp64_peak")
    learned = learned_leg(k, rp, d_in, work, stream, n, st, it, stats[0], args, dev)
    u2p = u2p_leg(k, rp, n, stream, dev)
    fp64_peak = peak.value / 1e12
    tf = IMP_FP64_PER_EVAL_CELLS * stats[3] / (ms_one / 1e3) / 1e12 if IMP_FP64_PER_EVAL_CELLS else None

    # e2e: the host-pointer entry point with pinned buffers, copies included
    hin = []
    for a in (uu, pp, g, G, dt):
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[...] = a
        hin.append(t)
    hpo = torch.empty((n, 13), dtype=torch.float64, pin_memory=True)
    huo = torch.empty((n, 13), dtype=torch.float64, pin_memory=True)
    hst, hat, hit = (torch.empty(n, dtype=torch.int32, pin_memory=True) for _ in range(3))
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    ke = max(1, min(2, args.steps))
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(ke):
        k._check(L.kgpu_rad_implicit_cells(n, ctypes.byref(rp), *[ctypes.cast(t.data_ptr(), dp) for t in hin],
                                           ctypes.cast(hpo.data_ptr(), dp), ctypes.cast(huo.data_ptr(), dp),
                                           ctypes.cast(hst.data_ptr(), ip), ctypes.cast(hat.data_ptr(), ip),
                                           ctypes.cast(hit.data_ptr(), ip), k.RAD_BATCHED), "kgpu_rad_implicit_cells")
    torch.cuda.synchronize(dev)
    e2e_s = time.perf_counter() - t0
    e2e_value = whole_job_rate(n, ke, world, 1e3 * max_over_ranks(e2e_s, dist, dev))
    if rank != 0:
        return
    ok = st == 0
    passes = (6 * 51 + 7) // 8 + 1   # pass launches of one batched solve at 8 iterations per pass
    line = {
        "metric": RAD_METRIC, "value": value, "unit": RAD_UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl["desc"], "cells_per_gpu": n, "l2": "inputs 2.2 GB > L2, no flush",
                   "parallelism": "replicas" if world > 1 else "one batch", "solver": "batched work queue"},
        "plain": {"value": plain_value, "unit": RAD_UNIT, "ms_per_step": ms_plain / steps_plain},
        "learned": learned,
        "u2p_warm_start": u2p,
        "newton": {"mean_iterations_successful_attempt": float(it[ok].mean()),
                   "mean_iterations_all_attempts": stats[0] / n, "passes_with_work": int(stats[1]),
                   "success_rate": float(ok.mean()),
                   "attempt_histogram": {int(a): int((at == a).sum()) for a in np.unique(at)}},
        "roofline": {"kernel": "k_rad_pass + k_rad_slow + k_rad_tail (batched implicit solve)", "bound": "fp64",
                     "peak": fp64_peak, "unit": "TFLOP/s",
                     "peak_source": "measured live (DMUL+DADD chains, no FMA)", "achieved": tf,
                     "frac": tf / fp64_peak if tf else None, "traffic": None, "evaluations": int(stats[3]),
                     "solve_ms": ms_one,
                     "flop_per_evaluation": IMP_FP64_PER_EVAL_CELLS},
        "e2e": {"value": e2e_value, "unit": RAD_UNIT, "h2d_bytes_per_step": n * (13 + 13 + 20 + 20 + 1) * 8,
                "d2h_bytes_per_step": n * (26 * 8 + 12)},
        "gpu_launches": passes * args.steps,
        "clocks": clk.summary(),
    }
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        val, err = run_reference_radcells(wl, wl["ref_sample_cells"], threads)
        line["cpu_baseline"] = {"value": val, "unit": RAD_UNIT, "cores": threads, "kind": "reference",
                                "sample": (f"{wl['ref_sample_cells']} cells of the same distribution"
                                           if val is not None else f"unavailable: {err}")}
    print(json.dumps(line))


def main():
    args = parse()
    wl = WORKLOADS[args.workload]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        reference_arm(args, wl, rank)
        return
    if args.profile_solve:
        profile_solve(args)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if "ncells" in wl:
            our_arm_radcells(args, wl, rank, world, local_rank)
        elif wl.get("radiation"):
            our_arm_radtorus(args, wl, rank, world, local_rank)
        else:
            our_arm(args, wl, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
