"""Generate the golden fixtures of the MHM solver from the reference itself.

Runs GAMER's own CPU_FluidSolver (compiled unmodified from the reference sources by
oracle/build_ref.sh into oracle/_ref/) on small seeded inputs and stores input + outputs as
compressed npz files next to this script.  Re-run only when the case list changes:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

import pyoracle as po  # noqa: E402
from gamer_b200 import ic  # noqa: E402

GAMMA = 5.0 / 3.0

# name, ic, lr, rsolver, dual, precision, nxt, limiter, minmod_maxiter, dt factor
# (+ optional: CHAR_RECONSTRUCTION, scheme "mhm" / "mhm_rp")
CASES = [
    ("mhm_plm_hllc_fp32_lognormal", "lognormal", "plm", "hllc", False, "fp32", 20, "gminmod", 0, 1.0),
    ("mhm_plm_hllc_fp64_lognormal", "lognormal", "plm", "hllc", False, "fp64", 20, "gminmod", 0, 1.0),
    ("mhm_ppm_roe_fp32_kh", "kh", "ppm", "roe", False, "fp32", 22, "gminmod", 0, 1.0),
    ("mhm_plm_hllc_de_fp64_blast", "blast", "plm", "hllc", True, "fp64", 20, "vl_gminmod", 3, 2.0),
    ("mhm_plm_exact_fp32_kh", "kh", "plm", "exact", False, "fp32", 20, "gminmod", 0, 1.0),
    ("mhm_plm_hllc_char_fp64_lognormal", "lognormal", "plm", "hllc", False, "fp64", 20, "vanleer", 0, 1.0, True),
    ("mhmrp_plm_hllc_fp32_kh", "kh", "plm", "hllc", False, "fp32", 22, "gminmod", 0, 1.0, False, "mhm_rp"),
]


def make_case(kind, dual, nxt, seed=2024):
    if kind == "lognormal":
        box = ic.lognormal_box(2, seed=seed, gamma=GAMMA, dual=dual)
    elif kind == "kh":
        box = ic.kelvin_helmholtz_box(2, seed=seed, gamma=GAMMA, dual=dual)
    else:
        box = ic.blast_box(2, seed=seed, gamma=GAMMA, dual=dual)
    dh = 1.0 / 32
    dt = ic.cfl_dt(box, GAMMA, dh, cfl=0.5)
    return ic.cut_patch_groups(box, nxt), dt, dh


def main():
    for case in CASES:
        name, kind, lr, rs, dual, prec, nxt, lim, maxit, dtf = case[:10]
        char = case[10] if len(case) > 10 else False
        scheme = case[11] if len(case) > 11 else "mhm"
        x, dt, dh = make_case(kind, dual, nxt)
        pg = ( [0, 5] if prec == "fp32" else [5] ) if kind != "blast" else [3]
        if len(case) > 10:
            pg = [5]
        x = x[pg]
        ref = po.RefSolver(po.ref_variant_name(scheme.replace("_", ""), lr, rs, dual=dual, char=char), prec)
        x = x.astype(ref.dtype)
        r = ref.solve(x, dt * dtf, dh, limiter=lim, minmod_maxiter=maxit)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), flu_in=x, flu_out=r["out"], flux=r["flux"],
                            de=r["de"], dt=dt * dtf, dh=dh, lr=lr, rsolver=rs, dual=dual, precision=prec,
                            limiter=lim, minmod_maxiter=maxit, gamma=GAMMA, char=char, scheme=scheme)
        print("wrote", name)


if __name__ == "__main__":
    main()
