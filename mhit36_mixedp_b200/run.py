"""Command-line driver: the run control of the reference's ``program main`` on one GPU.

Reads ``input.inp`` (multi/readinput.f90) when given, builds the initial condition (Taylor-Green
``inflow=0`` / fields from files ``inflow=1``, as multi/main.f90:322-350; or the seeded
synthetic fields of ``synth``), advances ``tfin - tstart`` steps, writes field files every
``dump`` steps (multi/main.f90:1023-1034) and prints the step scalars.

Examples::

    python -m mhit36_mixedp_b200.run --input multi/input.inp --n 128 --outdir output
    python -m mhit36_mixedp_b200.run --n 256 --synthetic --phiflag 1 --steps 4
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from . import api, synth


def taylor_green(n, yz_shift=1, ny=None, nz=None):
    """multi/main.f90:324-337 with the accumulated grid x(i) = x(i-1) + dx (one spacing 2 pi/n
    on every axis, y and z read yz_shift entries on)."""
    ny = ny or n
    nz = nz or n
    dx = 8.0 * math.atan(1.0) / n
    m = max(n, ny, nz)
    xs = np.zeros(m + 1)
    acc = 0.0
    for i in range(1, m + 1):
        acc = acc + dx
        xs[i] = acc
    X, Y, Z = xs[:n], xs[yz_shift:yz_shift + ny], xs[yz_shift:yz_shift + nz]
    u = np.sin(X - dx / 2)[None, None, :] * np.cos(Y)[None, :, None] * np.cos(Z)[:, None, None]
    v = -np.cos(X)[None, None, :] * np.sin(Y - dx / 2)[None, :, None] * np.cos(Z)[:, None, None]
    return u, v, np.zeros_like(u)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--input", help="input.inp to read (multi/readinput.f90 format)")
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--ny", type=int, help="grid points in y (default n)")
    ap.add_argument("--nz", type=int, help="grid points in z (default n)")
    ap.add_argument("--steps", type=int, help="steps to run (default tfin - tstart)")
    ap.add_argument("--phiflag", type=int, default=0)
    ap.add_argument("--poisson", default="fp64", choices=["fp64", "fp32", "fp32_refined", "fp32_incremental"])
    ap.add_argument("--laplacian", default="exact", choices=["exact", "modified"])
    ap.add_argument("--synthetic", action="store_true", help="seeded solenoidal velocity (+ 64 drops)")
    ap.add_argument("--indir", default="input", help="directory of u.dat, v.dat, w.dat, phi.dat")
    ap.add_argument("--outdir", default=None, help="write field files here every dump steps")
    ap.add_argument("--dt", type=float)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--zsolve-tc", action="store_true", help="512-point z solve on the tensor cores (FP32 modes)")
    args = ap.parse_args(argv)

    run = {"restart": 0, "tstart": 0, "tfin": 10, "dump": 10 ** 9, "inflow": 0, "inphi": 0}
    kw = dict(nx=args.n, ny=args.ny or args.n, nz=args.nz or args.n, phiflag=args.phiflag, poisson=args.poisson,
              laplacian=args.laplacian, device=args.device, zsolve_tc=int(args.zsolve_tc))
    if args.input:
        prm, run = api.read_input(args.input, **kw)
    else:
        prm = api.Params(**kw)
    if args.dt:
        prm.dt = args.dt
    n = args.n
    phi = None
    if args.synthetic:
        u, v, w = synth.solenoidal_velocity(n, 2, ny=prm.ny, nz=prm.nz)
        if prm.phiflag:
            prm.radius, prm.sigma = 0.3, synth.sigma_from_weber(prm.rho, 1.0, 0.3, 1.0)
            phi = synth.drops_phi(n, synth.drop_centres(64, 1), prm.radius, prm.epsr * 2 * math.pi / n)
    elif run.get("inflow", 0) == 1:
        u, v, w = (np.fromfile(os.path.join(args.indir, f"{c}.dat"), dtype=np.float64).reshape(prm.shape)
                   for c in "uvw")
    else:
        u, v, w = taylor_green(n, prm.yz_shift, prm.ny, prm.nz)
    if prm.phiflag and phi is None:
        if run.get("inphi", 0) == 1:
            phi = np.fromfile(os.path.join(args.indir, "phi.dat"), dtype=np.float64).reshape(prm.shape)
        else:  # centred drop, multi/main.f90:370-382
            dx = 8.0 * math.atan(1.0) / n
            x = np.arange(n) * dx
            y = (np.arange(prm.ny) + prm.yz_shift) * dx
            z = (np.arange(prm.nz) + prm.yz_shift) * dx
            lx = 8.0 * math.atan(1.0)
            pos = ((x - lx / 2) ** 2)[None, None, :] + ((y - lx / 2) ** 2)[None, :, None] + ((z - lx / 2) ** 2)[:, None, None]
            phi = 0.5 * (1.0 - np.tanh((np.sqrt(pos) - prm.radius) / 2 / (prm.epsr * dx)))
    steps = args.steps if args.steps is not None else run["tfin"] - run["tstart"]
    with api.Solver(prm) as s:
        s.upload(u, v, w, phi)
        if args.outdir:
            os.makedirs(args.outdir, exist_ok=True)
            for f in (1, 2, 3, 4) + ((5,) if prm.phiflag else ()):
                s.writefield(args.outdir, run["tstart"], f)
        t0 = time.perf_counter()
        for t in range(run["tstart"] + 1, run["tstart"] + steps + 1):
            s.step(1)
            if args.outdir and t % run["dump"] == 0:
                for f in (1, 2, 3, 4) + ((5,) if prm.phiflag else ()):
                    s.writefield(args.outdir, t, f)
        el = time.perf_counter() - t0
        d = s.diagnostics()
        print(json.dumps({"steps": steps, "wall_s": el, "ms_per_step": 1e3 * el / max(steps, 1), **d}))


if __name__ == "__main__":
    main()
