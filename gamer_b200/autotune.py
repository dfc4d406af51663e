"""Autotuner of the solver's launch shape.

For one solver configuration it times every candidate launch shape on a seeded batch of patch
groups with CUDA events and records the fastest in ``gamer_b200/tuned.json`` (keyed by GPU name and
configuration).  ``FluidSolver(block_size="auto")`` reads that table.

    python -m gamer_b200.autotune --precision mixed --lr plm --rsolver hllc
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CACHE = os.path.join(HERE, "tuned.json")
BLOCKS = (256, 288, 320, 352, 384, 416, 448, 480, 512)


def config_key(gpu_name, scheme, lr, rsolver, precision, dual, flu_nxt):
    return f"{gpu_name}|{scheme}|{lr}|{rsolver}|{precision}|{'de' if dual else 'nde'}|{flu_nxt}"


def load_cache():
    if os.path.exists(CACHE):
        with open(CACHE) as f:
            return json.load(f)
    return {}


def lookup(gpu_name, scheme, lr, rsolver, precision, dual, flu_nxt):
    e = load_cache().get(config_key(gpu_name, scheme, lr, rsolver, precision, dual, flu_nxt))
    return None if e is None else int(e["block"])


def tune(scheme="mhm", lr="plm", rsolver="hllc", precision="mixed", dual=False, flu_nxt=None, npd=10,
         reps=5, blocks=BLOCKS, write=True, verbose=True):
    import torch
    from gamer_b200 import ic
    from gamer_b200.fluid import FluidSolver, SolverParams

    if flu_nxt is None:
        flu_nxt = 22 if lr == "ppm" else 20
    gamma = 5.0 / 3.0
    box = ic.kelvin_helmholtz_box(npd, seed=77, gamma=gamma, dual=dual)
    dh = 1.0 / (npd * 16)
    dt = ic.cfl_dt(box, gamma, dh)
    x = ic.cut_patch_groups(box, flu_nxt)
    s = FluidSolver(scheme=scheme, lr=lr, rsolver=rsolver, precision=precision, dual_energy=dual, flu_nxt=flu_nxt)
    dev = torch.device("cuda", torch.cuda.current_device())
    t_in = torch.from_numpy(x.astype(s.np_dtype)).to(dev)
    npg = x.shape[0]
    t_out = torch.empty((npg, s.ncomp, 16, 16, 16), dtype=s.torch_dtype, device=dev)
    t_flx = torch.empty((npg, 9, s.ncomp, 16, 16), dtype=s.torch_dtype, device=dev)
    t_de = torch.zeros((npg, 16, 16, 16), dtype=torch.int8, device=dev) if dual else None
    prm = SolverParams(dt=dt, dh=dh)
    results = {}
    for b in blocks:
        s.set_block_size(b)
        s.solve_device(t_in, t_out, prm, flux=t_flx, de_out=t_de)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            s.solve_device(t_in, t_out, prm, flux=t_flx, de_out=t_de)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        results[b] = ms
        if verbose:
            print(f"block {b:4d}: {ms:.3f} ms  {npg * 4096 / ms / 1e6:.3f} Gcell/s")
    best = min(results, key=results.get)
    if write:
        cache = load_cache()
        name = torch.cuda.get_device_name(dev)
        cache[config_key(name, scheme, lr, rsolver, precision, dual, flu_nxt)] = {
            "block": best, "ms": results[best], "npg": npg, "all_ms": {str(k): v for k, v in results.items()}}
        with open(CACHE, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    s.close()
    return best, results


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scheme", default="mhm")
    ap.add_argument("--lr", default="plm")
    ap.add_argument("--rsolver", default="hllc")
    ap.add_argument("--precision", default="mixed")
    ap.add_argument("--dual", action="store_true")
    ap.add_argument("--npd", type=int, default=10)
    ap.add_argument("--all", action="store_true", help="tune every configuration the benchmarks use")
    a = ap.parse_args()
    if a.all:
        for prec in ("fp32", "mixed", "fp64"):
            for lr, rs in (("plm", "hllc"), ("ppm", "roe"), ("plm", "roe"), ("ppm", "hllc")):
                if prec == "fp64" and lr == "ppm":
                    continue
                print(f"== {prec} {lr} {rs}")
                tune(lr=lr, rsolver=rs, precision=prec, npd=a.npd)
        print("== mixed plm hllc dual")
        tune(lr="plm", rsolver="hllc", precision="mixed", dual=True, npd=a.npd)
    else:
        tune(a.scheme, a.lr, a.rsolver, a.precision, a.dual, npd=a.npd)


if __name__ == "__main__":
    main()
