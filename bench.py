#!/usr/bin/env python
"""Benchmark: ms/timestep of the MHIT36 NS+ACDI step at 512^3 on one B200.

Workload (the headline metric's configuration): 512^3 periodic box, NS + ACDI phase field,
64 drops of radius 0.3 (eps = dx) at seeded uniform centres (seed 1), seeded solenoidal
velocity (seed 2, unit rms), nu = 0.003, rho = 1, sigma from We = 1, dt = 2e-4 (the reference's
input.inp value; 5e-4 exceeds the explicit ACDI diffusion limit dx/(6 gamma) at 512^3), ABC forcing
f = 1 at k0 = 2.  ``value`` is the mixed-precision step at matched divergence: the incremental FP32
Poisson solve with the discrete Laplacian (FP64 state, one FP32 solve per step for the pressure
increment over the previous step, its right-hand side the FP64 residual), which keeps
max |div u| <= 1e-6; ``fp64_ms_per_step`` is the FP64 step with the same divide (divergence at
round-off).  The line also carries both steps' divergence, kinetic energy and dissipation, and
the reference's own divide (exact k^2, FP32 as its branch and FP64) under ``reference_divide``.
Fields are 1.07 GB each, larger than L2, so no flush is needed between steps.

Timing: W warm-up steps, then K steps between two CUDA events on the library's stream
(mhit_time_steps), max over ranks.  ``e2e`` repeats the mixed run through the public API with
pinned host buffers: upload u,v,w,phi -> K x mhit_step(1) (each reads back the step
scalars) -> download u,v,w,p,phi, all inside the timed region.  ``gpu_launches`` is K times the
kernel nodes of the library's captured step graph.  ``configs`` carries the other scope-table
configurations at N = 1: 1024^3 NS (FP32 and FP64 Poisson), 512^3 NS+ACDI with 1e6 tracers, and
the 32-box ensemble (fields built on the device from the same seeds).

--impl reference times the reference loop on the host cores.  The reference is Fortran + OpenACC +
cuDecomp and no Fortran compiler exists on this image, so its CPU implementation is the C/OpenMP
restatement in oracle/ (kind "port"), run on the bench workload itself at the same size and
Poisson precision; the line reports the warm-up and timed steps it actually ran.  ``cpu_baseline``
in the GPU arm's line is a bounded sample of the same run (one Euler step, then a few AB2 steps).
With torchrun (N > 1) every rank advances its own box (replicas; the step does not shard).
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
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ms/timestep 512^3 NS+ACDI, 1 B200: mixed-prec Poisson vs FP64, at matched div err"

# algorithmic HBM bytes per grid point and launch (compulsory traffic of each kernel)
BYTES_PER_POINT = {
    "fp32": {"k_phase": 56, "k_mom": 104, "k_div_fftx": 28, "k_fft_cols_yfwd": 8, "k_fft_cols_zsolve": 8,
             "k_fft_cols_yinv": 8, "k_fftx_inv": 8, "k_correct+k_finalize": 52, "k_xinv_correct+k_finalize": 52},
    "fp64": {"k_phase": 56, "k_mom": 104, "k_div_fftx": 32, "k_fft_cols_yfwd": 16, "k_fft_cols_zsolve": 16,
             "k_fft_cols_yinv": 16, "k_fftx_inv": 16, "k_correct+k_finalize": 56, "k_xinv_correct+k_finalize": 56},
}
# DRAM bytes per grid point and launch measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum
# of one launch / cells): k_phase and k_mom from a 256^3 capture, the Poisson and projection kernels
# from a 512x512x256 capture.  Traffic scales with the cell count for these streaming kernels, so
# the line reports these per-cell figures times the bench's cell count and says so.
TRAFFIC_PER_POINT = {"k_phase": 55.1, "k_mom": 104.4, "k_div_fftx": 28.4, "k_fft_cols_yfwd": 7.5,
                     "k_fft_cols_zsolve": 7.5, "k_fft_cols_yinv": 7.5, "k_fftx_inv": 7.5,
                     "k_correct+k_finalize": 51.2}
TRAFFIC_SOURCE = {"k_phase": "256^3", "k_mom": "256^3"}
BYTES_PER_POINT["fp32_incremental"] = dict(BYTES_PER_POINT["fp32"], k_div_fftx=32, k_fftx_inv=20,
                                           **{"k_correct+k_finalize": 56, "k_xinv_correct+k_finalize": 60})
# the step-level model (the x-inverse fused with the projection, the y/z passes as two spectrum
# round trips): NS+ACDI 256 B/pt (FP32 Poisson), 280 B/pt (FP64); the incremental FP32 solve adds
# the predictor's read in the x pass (4) and its read and write in the fused projection (8): 268
STEP_BYTES = {"fp32": 256, "fp64": 280, "fp32_incremental": 268}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or not self.path:
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                sm.append(float(f[1]))
                mx = float(f[2])
                for nm, val in zip(names, f[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(nm)
        except Exception:
            return None
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def workload(n, seed_drops=1, seed_vel=2):
    from mhit36_mixedp_b200 import synth
    radius, we, rho = 0.3, 1.0, 1.0
    eps = 2 * math.pi / n
    u, v, w = synth.solenoidal_velocity(n, seed_vel)
    phi = synth.drops_phi(n, synth.drop_centres(64, seed_drops), radius, eps)
    sigma = synth.sigma_from_weber(rho, 1.0, radius, we)
    prm = dict(nx=n, dt=2e-4, mu=0.003, rho=rho, f1=1.0, f2=1.0, f3=1.0, k0=2.0, radius=radius, sigma=sigma,
               epsr=1.0, phiflag=1, partflag=0, acdi_clamp=1)
    return prm, u, v, w, phi


def max_over_ranks(values, dist, device):
    """Element-wise maximum of per-rank timings over the process group (every rank gets it)."""
    import torch
    t = torch.tensor([float(x) for x in values], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def measure_mode(prm, fields, dev, poisson, laplacian, steps, warmup, profile=True):
    """Time `steps` graph-replayed steps of one Poisson mode on the workload after `warmup`
    steps; with `profile`, also per-stage event timings (3 profiled steps), clocks during the
    timed region and the kernels one step launches.  Returns a dict; the solver stays open for
    `extra(s)` callbacks via the 'solver' hook of the caller."""
    from mhit36_mixedp_b200 import Params, Solver
    _, u, v, w, phi = fields
    out = {}
    with Solver(Params(device=dev, poisson=poisson, laplacian=laplacian, **prm)) as s:
        s.upload(u, v, w, phi)
        s.step(max(warmup, 3))
        with Clocks(dev) as clk:
            ms = s.time_steps(steps)
        s.step(0)  # flag check of the timed steps
        out["ms"] = ms / steps
        out["diag"] = s.diagnostics()
        if profile:
            out["clocks"] = clk.summary()
            out["kernels_per_step"] = s.kernels_per_step()
            prof = [s.profile_step() for _ in range(3)]
            out["stages"] = {k: statistics.mean(p[k] for p in prof) for k in prof[0]}
            out["diag"] = s.diagnostics()
        if poisson == "fp32" and laplacian == "exact":
            # droplet labelling of the current state (post/unionfind_periodic): host call,
            # wall clock including its host<->device copies of the per-drop sums
            s.label_drops(0.5, 6)
            t0 = time.perf_counter()
            drops = s.label_drops(0.5, 6)
            out["drops"] = {"ms_per_call": (time.perf_counter() - t0) * 1e3, "ndrops": len(drops["cells"]),
                            "connectivity": 6, "cells_in_drops": int(drops["cells"].sum())}
        if poisson == "fp64" and laplacian == "exact":
            # energy spectrum of the current state through the FP64 transform passes: host call,
            # wall clock; Parseval against the diagnostics' kinetic energy
            try:
                s.energy_spectrum()
                t0 = time.perf_counter()
                E = s.energy_spectrum()
                out["spectrum"] = {"ms_per_call": (time.perf_counter() - t0) * 1e3, "nbins": int(E.size),
                                   "parseval_relerr": abs(float(E.sum()) - out["diag"]["ke"]) / out["diag"]["ke"]}
            except Exception as ex:  # pragma: no cover - reported, not hidden
                out["spectrum"] = {"error": str(ex)}
    return out


# the headline pair: the mixed-precision step that keeps max |div u| <= 1e-6 (incremental FP32
# solve) and the FP64 step, both with the discrete Laplacian (divergence at round-off for FP64)
HEADLINE = {"mixed": ("fp32_incremental", "modified"), "fp64": ("fp64", "modified")}


def run_ours(args, rank, world, dev, fields):
    prm = fields[0]
    res = {m: measure_mode(prm, fields, dev, pm, lap, args.steps, args.warmup) for m, (pm, lap) in HEADLINE.items()}
    # the reference's own divide (exact k^2, O(dx^2) divergence), FP32 as its branch and FP64
    res["exact"] = {pm: measure_mode(prm, fields, dev, pm, "exact", args.steps, args.warmup)
                    for pm in ("fp32", "fp64")}
    # the other discrete-Laplacian modes: plain FP32 and FP32 + one FP64 residual sweep
    res["modified_others"] = {pm: measure_mode(prm, fields, dev, pm, "modified", max(args.steps // 2, 3),
                                               args.warmup, profile=False) for pm in ("fp32", "fp32_refined")}
    # e2e through the public API with pinned host buffers (the headline mixed mode)
    e2e = None
    n = args.n
    try:
        import torch
        from mhit36_mixedp_b200 import Params, Solver
        from mhit36_mixedp_b200.api import _dptr
        _, u, v, w, phi = fields
        shp = (n, n, n)
        host = {f: torch.empty(shp, dtype=torch.float64, pin_memory=True).numpy() for f in ("u", "v", "w", "phi")}
        outs = {f: torch.empty(shp, dtype=torch.float64, pin_memory=True).numpy() for f in ("u", "v", "w", "p", "phi")}
        host["u"][...] = u
        host["v"][...] = v
        host["w"][...] = w
        host["phi"][...] = phi
        pm, lap = HEADLINE["mixed"]
        with Solver(Params(device=dev, poisson=pm, laplacian=lap, **prm)) as s:
            s.upload(host["u"], host["v"], host["w"], host["phi"])
            s.step(max(args.warmup, 3))
            lib, ctx = s._lib, s._ctx
            t0 = time.perf_counter()
            s.upload(host["u"], host["v"], host["w"], host["phi"])
            for _ in range(args.steps):
                s.step(1)
            rc = lib.mhit_download_fields(ctx, *[_dptr(outs[f]) for f in ("u", "v", "w", "p", "phi")])
            t1 = time.perf_counter()
            assert rc == 0
        h2d = 4 * n ** 3 * 8
        d2h = 5 * n ** 3 * 8 + args.steps * 160
        e2e = {"value": (t1 - t0) * 1e3 / args.steps, "unit": "ms/timestep",
               "h2d_bytes_per_step": h2d // args.steps, "d2h_bytes_per_step": d2h // args.steps,
               "how": "pinned host u,v,w,phi -> mhit_upload_fields -> K x mhit_step(1) -> mhit_download_fields"}
    except Exception as ex:  # pragma: no cover - reported, not hidden
        e2e = {"value": None, "error": str(ex)}
    return res, e2e


def headline_config(n, world):
    return {"workload": f"NS+ACDI {n}^3, 64 drops R=0.3 eps=dx, We=1, nu=0.003, dt=2e-4, "
                        f"seeds drops=1 vel=2; value: mixed step with max|div u| <= 1e-6 (incremental FP32 "
                        f"Poisson, discrete Laplacian) against the FP64 step",
            "parallelism": "replicas" if world > 1 else "single", "l2": "inputs larger than L2"}


def cpu_reference(fields, warmup, steps, budget_s):
    """The C/OpenMP restatement of the reference loop (oracle/mhit_oracle.c, multi/main.f90:456-1007
    pass by pass) on the bench workload itself (same size, same inputs, FP32 Poisson), on all host
    threads: `warmup` untimed steps (the first is the Euler step), then up to `steps` timed steps,
    fewer when the first step's time says the run would not end within `budget_s` seconds.
    Returns (ms per timed step, warm-up steps run, timed steps run, threads)."""
    from oracle.coracle import COracle, threads
    prm, u, v, w, phi = fields
    c = COracle(poisson="fp32", **prm)
    try:
        c.set_fields(u, v, w, phi)
        t0 = time.perf_counter()
        c.step(1)
        t_step = time.perf_counter() - t0
        nwarm = max(1, min(int(warmup), int(0.25 * budget_s / max(t_step, 1e-9))))
        for _ in range(nwarm - 1):
            c.step(1)
        ntimed = max(1, min(int(steps), int((budget_s - nwarm * t_step) / max(t_step, 1e-9))))
        t0 = time.perf_counter()
        c.step(ntimed)
        ms = (time.perf_counter() - t0) * 1e3 / ntimed
    finally:
        c.close()
    return ms, nwarm, ntimed, threads()


def cpu_baseline_line(fields, warmup, steps, budget_s):
    ms, nwarm, ntimed, cores = cpu_reference(fields, warmup, steps, budget_s)
    n = fields[0]["nx"]
    return {"value": ms, "unit": "ms/timestep", "cores": cores, "kind": "port",
            "sample": f"C/OpenMP restatement of multi/main.f90:456-1007 on the bench workload itself "
                      f"({n}^3 NS+ACDI, FP32 Poisson): {nwarm} untimed step(s) including the Euler step, "
                      f"then {ntimed} timed AB2 step(s), mean"}


def ensemble_workload(indices=None):
    """32 NS+ACDI boxes: 16 x 64^3, 10 x 128^3, 6 x 192^3; per-box seeds 100+b; nu ~ U[0.002,0.01],
    We ~ U[0.5,5], 32-256 drops of radius 0.3 (eps = dx), FP32 Poisson, dt = 2e-4.  Returns the
    parameters of every box (from one seeded stream) and, per box, the seed and drop centres the
    fields are built from on the device (seeded solenoidal velocity of unit rms, drops at seeded
    uniform centres); with indices, only those boxes."""
    from mhit36_mixedp_b200 import Params, synth
    rng = np.random.default_rng(99)
    boxes = []
    for b, n in enumerate(ENSEMBLE_SIZES):
        nu = float(rng.uniform(0.002, 0.01))
        we = float(rng.uniform(0.5, 5.0))
        ndrops = int(rng.integers(32, 257))
        if indices is not None and b not in indices:
            continue
        prm = Params(nx=n, dt=2e-4, mu=nu, rho=1.0, radius=0.3, sigma=synth.sigma_from_weber(1.0, 1.0, 0.3, we),
                     phiflag=1, poisson="fp32", acdi_clamp=1)
        boxes.append((prm, 100 + b, synth.drop_centres(ndrops, 100 + b)))
    return boxes


ENSEMBLE_SIZES = [64] * 16 + [128] * 10 + [192] * 6


def partition_boxes(sizes, nranks):
    """Boxes onto ranks by greedy longest-first bin packing on the cell count (the step cost is
    proportional to it): the box indices of each rank, sorted."""
    order = sorted(range(len(sizes)), key=lambda b: (-sizes[b] ** 3, b))
    load = [0] * nranks
    parts = [[] for _ in range(nranks)]
    for b in order:
        r = min(range(nranks), key=lambda q: (load[q], q))
        parts[r].append(b)
        load[r] += sizes[b] ** 3
    return [sorted(p) for p in parts]


def ensemble_measure(indices, device, steps, warmup):
    """Advance the given boxes of the 32-box ensemble as one ensemble on `device` and time `steps`
    graph-launched ensemble steps.  Returns (ms per step, tuning, clocks)."""
    from mhit36_mixedp_b200 import Ensemble
    boxes = ensemble_workload(set(indices))
    for b in boxes:
        b[0].device = device
    with Ensemble([b[0] for b in boxes]) as ens:
        tuning = ens.autotune(trials=2)
        for box, (prm, seed, centres) in zip(ens.boxes, boxes):
            box.init_solenoidal(seed=seed, kmax=4)
            box.init_drops(centres, prm.radius)
        ens.step(max(warmup, 3))
        with Clocks(device) as clk:
            ms = ens.time_steps(steps)
        ens.step(0)
    return ms / steps, tuning, clk.summary()


def run_ensemble(args):
    """The 32-box ensemble; under torchrun the boxes are shared out over the ranks (strong
    scaling: the same 32 boxes whatever N), each rank steps its share as one ensemble, and the
    step time is the max over ranks."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    mine = partition_boxes(ENSEMBLE_SIZES, world)[rank]
    ms, tuning, clocks = 0.0, None, None
    if dist:
        dist.barrier()
    if mine:
        ms, tuning, clocks = ensemble_measure(mine, local, args.steps, args.warmup)
    if dist:
        ms = max_over_ranks([ms], dist, f"cuda:{local}")[0]
        dist.barrier()
    if rank == 0:
        npts = sum(n ** 3 for n in ENSEMBLE_SIZES)
        peak, kind = peaks()
        frac = STEP_BYTES["fp32"] * npts / (ms * 1e-3) / 1e9 / peak / world
        line = {"metric": "ms per ensemble step, 32 NS+ACDI boxes (16x64^3, 10x128^3, 6x192^3), FP32 Poisson",
                "value": ms, "unit": "ms/timestep", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "higher_is_better": False, "scaling": "strong", "data": "synthetic",
                "dtype": "f64+f32",
                "config": {"workload": "ensemble", "boxes": len(ENSEMBLE_SIZES), "points": npts,
                           "one_graph_launch_per_step": True, "boxes_per_rank": [len(p) for p in partition_boxes(ENSEMBLE_SIZES, world)]},
                "tuning_rank0": tuning, "step_roofline_frac": frac, "peak_kind": kind, "clocks": clocks}
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def large_ns_measure(n, device, steps, warmup):
    """n^3 NS (no phase field), FP32 and FP64 Poisson, nu = 8e-4: the seeded random solenoidal
    velocity (seed 4, 0 < |k| <= 4, unit rms) synthesised on the device (its host version would
    need tens of GB of host memory at 1024^3), ABC forcing on."""
    from mhit36_mixedp_b200 import Params, Solver
    prm = dict(nx=n, dt=2e-4, mu=8e-4, rho=1.0, f1=1.0, f2=1.0, f3=1.0, k0=2.0)
    res = {}
    peak, _ = peaks()
    ns_bytes = {"fp32": 192, "fp64": 216}  # NS step model: 192 / 216 B per point
    for mode in ("fp32", "fp64"):
        with Solver(Params(device=device, poisson=mode, **prm)) as s:
            s.init_solenoidal(seed=4, kmax=4)
            s.step(max(warmup, 3))
            with Clocks(device) as clk:
                ms = s.time_steps(steps)
            s.step(0)
            prof = s.profile_step()
            dg = s.diagnostics()
        res[mode] = {"ms_per_step": ms / steps, "stages_ms": prof, "maxdiv": dg["maxdiv"], "ke": dg["ke"],
                     "step_roofline_frac": ns_bytes[mode] * n ** 3 / (ms / steps * 1e-3) / 1e9 / peak,
                     "clocks": clk.summary()}
    return res


def run_large_ns(args):
    n = 1024 if args.n == 512 else args.n
    res = large_ns_measure(n, 0, args.steps, args.warmup)
    line = {"metric": f"ms/timestep {n}^3 NS, 1 B200, FP32 vs FP64 Poisson", "value": res["fp32"]["ms_per_step"],
            "unit": "ms/timestep", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
            "data": "synthetic (seeded solenoidal modes 0<|k|<=4, seed 4, built on the device)", "dtype": "f64+f32",
            "config": {"workload": f"NS {n}^3, nu=8e-4, dt=2e-4", "l2": "inputs larger than L2"},
            "fp64_ms_per_step": res["fp64"]["ms_per_step"], "detail": res, "peak_kind": peaks()[1]}
    print(json.dumps(line), flush=True)
    return 0


def tracers_measure(fields, device, steps, warmup, npart=1_000_000):
    """512^3 NS+ACDI with 1e6 uniform tracers (seed 3): FP64 Poisson with both interpolation modes,
    FP32 Poisson with trilinear interpolation, and the configuration's own Poisson: the
    tensor-core DFT z solve (BF16x3 split, FP32 accumulation) inside the incremental FP32 solve,
    whose right-hand side is the FP64 residual (discrete Laplacian)."""
    from mhit36_mixedp_b200 import Params, Solver, synth
    prm, u, v, w, phi = fields
    part = synth.uniform_particles(npart, 3)
    prm = dict(prm, partflag=1, npart=npart)
    res = {}
    for poisson, interp, lap, tc in (("fp64", "linear1d", "exact", 0), ("fp64", "trilinear", "exact", 0),
                                     ("fp32", "trilinear", "exact", 0),
                                     ("fp32_incremental", "trilinear", "modified", 0),
                                     ("fp32_incremental", "trilinear", "modified", 1)):
        with Solver(Params(device=device, poisson=poisson, interp=interp, laplacian=lap, zsolve_tc=tc, **prm)) as s:
            s.upload(u, v, w, phi)
            s.upload_particles(part)
            s.step(max(warmup, 3))
            with Clocks(device) as clk:
                ms = s.time_steps(steps)
            s.step(0)
            prof = [s.profile_step() for _ in range(3)]
            dg = s.diagnostics()
        tr = statistics.mean(p["k_tracer"] for p in prof)
        zs = statistics.mean(p["k_fft_cols_zsolve"] for p in prof)
        key = f"{poisson}_{interp}" + ("_tensorcore_zsolve" if tc else "") + ("_modified" if lap == "modified" else "")
        res[key] = {"ms_per_step": ms / steps, "tracer_stage_ms": tr, "zsolve_stage_ms": zs, "maxdiv": dg["maxdiv"],
                    "clocks": clk.summary()}
    return res


def run_tracers(args):
    fields = workload(args.n)
    res = tracers_measure(fields, 0, args.steps, args.warmup)
    line = {"metric": f"ms/timestep {args.n}^3 NS+ACDI + 1e6 tracers, 1 B200",
            "value": res["fp64_linear1d"]["ms_per_step"], "unit": "ms/timestep", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": False, "data": "synthetic", "dtype": "f64",
            "config": {"workload": f"NS+ACDI {args.n}^3 + 1e6 uniform tracers (seed 3)"}, "detail": res}
    print(json.dumps(line), flush=True)
    return 0


def run_reference(args):
    """--impl reference: the reference's loop on the host cores.  The reference itself is Fortran
    + OpenACC + cuDecomp with no Fortran compiler on this image, so its CPU implementation is the C
    restatement (kind "port") on the bench workload at the same size and Poisson precision as the
    GPU arm's value, timed on all host threads.  Under torchrun only rank 0 runs."""
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    world = int(os.environ.get("WORLD_SIZE", "1"))
    fields = workload(args.n)
    ms, nwarm, ntimed, cores = cpu_reference(fields, args.warmup, args.steps, REFERENCE_BUDGET_S)
    cb = {"value": ms, "unit": "ms/timestep", "cores": cores, "kind": "port",
          "sample": f"the whole bench workload ({args.n}^3 NS+ACDI, FP32 Poisson), {nwarm} untimed step(s) "
                    f"including the Euler step, {ntimed} timed AB2 step(s), mean; C/OpenMP restatement of "
                    f"multi/main.f90:456-1007"}
    line = {"impl": "reference", "metric": METRIC, "value": ms, "unit": "ms/timestep", "n_gpus": args.gpus,
            "steps": ntimed, "warmup": nwarm, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic", "config": headline_config(args.n, world),
            "requested": {"steps": args.steps, "warmup": args.warmup}, "cpu_baseline": cb,
            "reference_algorithm": "the reference's FP32 branch (exact k^2 divide, FP32 transforms); its loop has "
                                   "no incremental solve",
            "e2e": {"value": ms, "unit": "ms/timestep", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# wall-clock budget of the reference arm's steps (about a minute on a 16-core host at 512^3)
REFERENCE_BUDGET_S = 120.0
# the GPU arm's CPU-baseline sample: one Euler + a few AB2 steps of the same workload
CPU_SAMPLE_BUDGET_S = 15.0


def measure_configs(args, dev, fields):
    """The other scope-table configurations, compact: 1024^3 NS (FP32 / FP64 Poisson), 512^3
    NS+ACDI + 1e6 tracers, the 32-box ensemble.  A failure is reported in its entry."""
    out = {}
    jobs = (("ns_1024", large_ns_measure, (1024, dev, min(args.steps, 5), 3)),
            ("tracers_1e6", tracers_measure, (fields, dev, min(args.steps, 10), 3)),
            ("ensemble_32", ensemble_measure, (range(len(ENSEMBLE_SIZES)), dev, args.steps, args.warmup)))
    for name, fn, fargs in jobs:
        try:
            out[name] = fn(*fargs)
        except Exception as ex:  # pragma: no cover - reported, not hidden
            out[name] = {"error": str(ex)}
    e = out["ensemble_32"]
    if isinstance(e, tuple):
        ms, tuning, clocks = e
        npts = sum(m ** 3 for m in ENSEMBLE_SIZES)
        out["ensemble_32"] = {"ms_per_step": ms, "tuning": tuning, "clocks": clocks,
                              "step_roofline_frac": STEP_BYTES["fp32"] * npts / (ms * 1e-3) / 1e9 / peaks()[0]}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="only the headline configuration")
    ap.add_argument("--ensemble", action="store_true", help="time the 32-box ensemble instead")
    ap.add_argument("--workload", choices=["acdi", "ns-large", "tracers"], default="acdi",
                    help="acdi: the headline NS+ACDI step; ns-large: 1024^3 NS; tracers: + 1e6 tracers")
    args = ap.parse_args()
    if args.ensemble:
        return run_ensemble(args)
    if args.workload == "ns-large":
        return run_large_ns(args)
    if args.workload == "tracers":
        return run_tracers(args)
    if args.impl == "reference":
        return run_reference(args)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    dev = local
    fields = workload(args.n)
    if dist:
        dist.barrier()
    res, e2e = run_ours(args, rank, world, dev, fields)
    msmix, ms64 = res["mixed"]["ms"], res["fp64"]["ms"]
    if dist:
        msmix, ms64 = max_over_ranks([msmix, ms64], dist, f"cuda:{local}")
        dist.barrier()
    extras = measure_configs(args, dev, fields) if world == 1 and not args.no_extras else None
    if rank == 0:
        n = args.n
        npts = n ** 3
        peak, peak_kind = peaks()
        mix_mode = HEADLINE["mixed"][0]
        st = res["mixed"]["stages"]
        dom = max(st, key=st.get)
        dom_bytes = BYTES_PER_POINT[mix_mode][dom] * npts
        achieved = dom_bytes / (st[dom] * 1e-3) / 1e9
        traffic = None
        if dom in TRAFFIC_PER_POINT:
            traffic = TRAFFIC_PER_POINT[dom] * npts
        roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                "traffic_how": f"ncu DRAM bytes per cell of a {TRAFFIC_SOURCE.get(dom, '512x512x256')} capture of "
                               f"{dom} x the {n}^3 cells (scaled, not measured in this run)",
                "algorithmic_bytes_per_launch": dom_bytes, "launch_ms": st[dom]}
        step_roof = {"mixed": STEP_BYTES[mix_mode] * npts / (msmix * 1e-3) / 1e9 / peak,
                     "fp64": STEP_BYTES["fp64"] * npts / (ms64 * 1e-3) / 1e9 / peak}
        cb = None
        if not args.no_cpu_baseline and world == 1:
            try:
                cb = cpu_baseline_line(fields, 1, 3, CPU_SAMPLE_BUDGET_S)
            except Exception as ex:
                cb = {"value": None, "error": str(ex)}
        ex = res["exact"]
        mo = res["modified_others"]
        line = {
            "metric": METRIC, "value": msmix, "unit": "ms/timestep", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": msmix, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic", "config": headline_config(n, world),
            "fp64_ms_per_step": ms64, "mixed_speedup_vs_fp64": ms64 / msmix,
            "divergence": {
                "definition": "max over cells of |div u| of the staggered operator of multi/main.f90:841-843 "
                              "(without rho/dt), absolute, after the timed steps; bound 1e-6",
                "mixed": res["mixed"]["diag"]["maxdiv"], "fp64": res["fp64"]["diag"]["maxdiv"],
                "mixed_le_1e-6": res["mixed"]["diag"]["maxdiv"] <= 1e-6},
            "dissipation": {"mixed": res["mixed"]["diag"]["dissipation"], "fp64": res["fp64"]["diag"]["dissipation"],
                            "relerr": abs(res["mixed"]["diag"]["dissipation"] / res["fp64"]["diag"]["dissipation"] - 1)},
            "kinetic_energy_relerr": abs(res["mixed"]["diag"]["ke"] / res["fp64"]["diag"]["ke"] - 1),
            "step_roofline_frac": step_roof, "stages_ms": {m: res[m]["stages"] for m in ("mixed", "fp64")},
            "roofline": roof, "cpu_baseline": cb, "e2e": e2e,
            "gpu_launches": res["mixed"]["kernels_per_step"] * args.steps,
            "kernels_per_step": {m: res[m]["kernels_per_step"] for m in ("mixed", "fp64")},
            "clocks": res["mixed"]["clocks"], "clocks_fp64": res["fp64"]["clocks"],
            "reference_divide": {
                "what": "exact k^2 divide of multi/main.f90:889 (O(dx^2) divergence), FP32 as the reference's "
                        "branch and FP64",
                "fp32_ms_per_step": ex["fp32"]["ms"], "fp64_ms_per_step": ex["fp64"]["ms"],
                "fp32_speedup_vs_fp64": ex["fp64"]["ms"] / ex["fp32"]["ms"],
                "maxdiv": {"fp32": ex["fp32"]["diag"]["maxdiv"], "fp64": ex["fp64"]["diag"]["maxdiv"]},
                "dissipation": {"fp32": ex["fp32"]["diag"]["dissipation"], "fp64": ex["fp64"]["diag"]["dissipation"]},
                "stages_ms": {m: ex[m]["stages"] for m in ("fp32", "fp64")},
                "step_roofline_frac": {m: STEP_BYTES[m] * npts / (ex[m]["ms"] * 1e-3) / 1e9 / peak
                                       for m in ("fp32", "fp64")}},
            "modified_laplacian_other_modes": {m: {"ms_per_step": mo[m]["ms"], "maxdiv": mo[m]["diag"]["maxdiv"],
                                                   "dissipation": mo[m]["diag"]["dissipation"]} for m in mo},
            "drop_labelling": ex["fp32"].get("drops"), "energy_spectrum": ex["fp64"].get("spectrum"),
            "configs": extras,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
