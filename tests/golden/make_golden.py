"""Generate the golden fixtures under tests/golden (run in a checkout that has the reference).

1. tg128_d2z.json, tg512_d2z.json -- the reference's own published Taylor-Green Re=1600
   dissipation curves at 128^3 and 512^3 (val/cudec_128_d2z.txt and val/cudec_512_d2z.txt of
   aroccon/MHIT36_mixedp: t, epsilon; nu = 6.25e-4, dt = 2e-4,
   val/comparison_diss.m:5,10), plus how epsilon was computed by the reference's
   post-processor (post/compute_diss/main.f90:7-11,72-117: central differences with
   dx = lx/(nx-1), lx = 2*pi where pi=3.14159265358979 is a default-REAL literal, i.e. the
   float32 value of pi, post/compute_diss/module.f90:5).
2. oracle_16.npz -- oracle outputs on 16^3 seeded inputs (NS FP64; NS+ACDI+tracers FP64;
   NS FP32 Poisson; 10 steps each) so the GPU path and the oracle can both be checked
   against stored numbers.

Usage: python tests/golden/make_golden.py /path/to/reference
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def tg_curve(ref, n):
    rows = []
    with open(os.path.join(ref, "val", f"cudec_{n}_d2z.txt")) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 2:
                rows.append([float(parts[0]), float(parts[1])])
    out = {
        "source": f"val/cudec_{n}_d2z.txt (aroccon/MHIT36_mixedp)",
        "nx": n, "nu": 6.25e-4, "dt": 2e-4, "forcing": 0.0,
        "postproc_dx": "lx/(nx-1) with lx = 2*float32(pi)",
        "t_eps": rows,
    }
    with open(os.path.join(HERE, f"tg{n}_d2z.json"), "w") as f:
        json.dump(out, f, indent=1)


def case_inputs(name):
    from mhit36_mixedp_b200 import synth
    n = 16
    prm = dict(nx=n, dt=5e-4, mu=0.006, rho=1.0, f1=1.0, f2=1.0, f3=1.0, k0=2.0, radius=0.6, sigma=0.5,
               epsr=1.0, phiflag=0, partflag=0)
    u, v, w = synth.solenoidal_velocity(n, 0)
    phi = part = None
    if name == "acdi_tracers":
        prm.update(phiflag=1, partflag=1)
        phi = synth.drops_phi(n, synth.drop_centres(4, 1), 0.6, 2 * np.pi / n)
        part = synth.uniform_particles(64, 3)
    if name == "ns_fp32":
        prm["poisson"] = "fp32"
    return prm, u, v, w, phi, part


CASES = ["ns_fp64", "acdi_tracers", "ns_fp32"]
NSTEPS = 10


def oracle_fixtures():
    from oracle import mhit_oracle as orc
    arrays = {}
    for name in CASES:
        prm, u, v, w, phi, part = case_inputs(name)
        op = orc.Params(**prm)
        st = orc.new_state(op, u, v, w, phi=phi, part=part)
        orc.run(op, st, NSTEPS)
        for f in ("u", "v", "w", "p"):
            arrays[f"{name}/{f}"] = getattr(st, f)
        if phi is not None:
            arrays[f"{name}/phi"] = st.phi
        if part is not None:
            arrays[f"{name}/part"] = st.part
        arrays[f"{name}/gumax"] = np.array(st.gumax)
    np.savez_compressed(os.path.join(HERE, "oracle_16.npz"), **arrays)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the reference checkout>")
    ref = sys.argv[1]
    tg_curve(ref, 128)
    tg_curve(ref, 512)
    oracle_fixtures()
    print("written", os.listdir(HERE))
