"""Autotuner of the solver's launch.

For one solver configuration it times every candidate launch of the MHM kernel — threads per CTA,
a cap on CTAs per SM, and (for the headline configuration, which has them) the register-capped
instantiations — on seeded batches of several sizes with CUDA events, and records the fastest per
batch size in ``gamer_b200/tuned.json`` (keyed by GPU name and configuration).
``FluidSolver(block_size="auto")`` applies, at each call, the entry of the batch size nearest to the
call's (in log scale).

    python -m gamer_b200.autotune --precision fp32 --lr plm --rsolver hllc
"""
from __future__ import annotations

import argparse
import json
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))
CACHE = os.path.join(HERE, "tuned.json")
BLOCKS = (256, 288, 320, 352, 384, 416, 448, 480, 512)
CTAS = (0, 1)                  # 0: as many CTAs per SM as fit
NPGS = (216, 1000, 4096)       # batch sizes: 6^3, 10^3, 16^3 patch groups
# register variants of the headline kernel (0 = the default instantiation, 96 per thread in float):
# with 64 / 72 / 80 registers two CTAs of 512 / 448 / 384 threads, or three of 320 / 288 / 256, fit
# an SM's 64K registers; every thread count is tried with each
REG_BLOCKS = {0: BLOCKS, 64: BLOCKS, 72: BLOCKS, 80: BLOCKS, 128: BLOCKS}


def config_key(gpu_name, scheme, lr, rsolver, precision, dual, flu_nxt):
    return f"{gpu_name}|{scheme}|{lr}|{rsolver}|{precision}|{'de' if dual else 'nde'}|{flu_nxt}"


def has_reg_variants(scheme, lr, rsolver, precision, dual, flu_nxt):
    """The register-capped instantiations exist for the float policies' MHM + PLM + HLLC, 5
    variables, FLU_NXT = 20 (the library's gb_fluid_set_launch)."""
    return (scheme, lr, rsolver, dual, flu_nxt) == ("mhm", "plm", "hllc", False, 20) and precision != "fp64"


def load_cache(path=None):
    path = path or CACHE
    if not os.path.exists(path) and path != CACHE:
        path = CACHE                  # a new output file starts from the shipped table
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def lookup_launch(gpu_name, scheme, lr, rsolver, precision, dual, flu_nxt, npg=None):
    """(threads, ctas_per_sm, max_registers) recorded for this configuration and the batch size
    nearest to npg; None if the configuration was not tuned."""
    e = load_cache().get(config_key(gpu_name, scheme, lr, rsolver, precision, dual, flu_nxt))
    if e is None:
        return None
    by = e.get("by_npg")
    if not by:
        return (int(e["block"]), 0, 0)
    sizes = sorted(int(k) for k in by)
    n = max(1, int(npg or sizes[-1]))
    best = min(sizes, key=lambda k: abs(math.log(k) - math.log(n)))
    t = by[str(best)]
    return (int(t["block"]), int(t["ctas"]), int(t["reg"]))


def lookup(gpu_name, scheme, lr, rsolver, precision, dual, flu_nxt):
    """Threads per CTA of the largest tuned batch (None if not tuned)."""
    t = lookup_launch(gpu_name, scheme, lr, rsolver, precision, dual, flu_nxt)
    return None if t is None else t[0]


def candidates(scheme, lr, rsolver, precision, dual, flu_nxt, blocks=BLOCKS):
    regs = REG_BLOCKS if has_reg_variants(scheme, lr, rsolver, precision, dual, flu_nxt) else {0: BLOCKS}
    out = []
    for reg, bl in regs.items():
        for b in bl:
            if reg == 0 and b not in blocks:
                continue
            for c in CTAS:
                out.append((b, c, reg))
    return out


def tune(scheme="mhm", lr="plm", rsolver="hllc", precision="fp32", dual=False, flu_nxt=None, npgs=NPGS,
         reps=5, blocks=BLOCKS, write=True, verbose=True, out=None):
    """Time every candidate launch on each batch size; returns {npg: (best, {launch: ms})}."""
    import torch
    from gamer_b200 import ic
    from gamer_b200.fluid import FluidSolver, SolverParams

    if flu_nxt is None:
        flu_nxt = 22 if lr == "ppm" else 20
    gamma = 5.0 / 3.0
    s = FluidSolver(scheme=scheme, lr=lr, rsolver=rsolver, precision=precision, dual_energy=dual, flu_nxt=flu_nxt)
    dev = torch.device("cuda", torch.cuda.current_device())
    cands = candidates(scheme, lr, rsolver, precision, dual, flu_nxt, blocks)
    found = {}
    for npg in npgs:
        npd = round(npg ** (1.0 / 3.0))
        box = ic.kelvin_helmholtz_box(npd, seed=77, gamma=gamma, dual=dual)
        dh = 1.0 / (npd * 16)
        dt = ic.cfl_dt(box, gamma, dh)
        x = ic.cut_patch_groups(box, flu_nxt)
        n = x.shape[0]
        t_in = torch.from_numpy(x.astype(s.np_dtype)).to(dev)
        t_out = torch.empty((n, s.ncomp, 16, 16, 16), dtype=s.torch_dtype, device=dev)
        t_flx = torch.empty((n, 9, s.ncomp, 16, 16), dtype=s.torch_dtype, device=dev)
        t_de = torch.zeros((n, 16, 16, 16), dtype=torch.int8, device=dev) if dual else None
        prm = SolverParams(dt=dt, dh=dh)
        res = {}
        for (b, c, reg) in cands:
            s.set_launch(b, c, reg)
            try:
                s.solve_device(t_in, t_out, prm, flux=t_flx, de_out=t_de)
                torch.cuda.synchronize()
            except Exception as e:  # noqa: BLE001  (a launch that does not fit an SM is skipped)
                if verbose:
                    print(f"npg {n:5d} block {b:3d} ctas {c} reg {reg:3d}: skipped ({e})")
                continue
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                s.solve_device(t_in, t_out, prm, flux=t_flx, de_out=t_de)
            e1.record()
            torch.cuda.synchronize()
            res[(b, c, reg)] = e0.elapsed_time(e1) / reps
            if verbose:
                ms = res[(b, c, reg)]
                print(f"npg {n:5d} block {b:3d} ctas {c} reg {reg:3d}: {ms:.4f} ms  {n * 4096 / ms / 1e6:.3f} Gcell/s")
        best = min(res, key=res.get)
        found[n] = (best, res)
        del t_in, t_out, t_flx, t_de
    s.close()
    if write:
        cache = load_cache(out)
        name = torch.cuda.get_device_name(dev)
        by = {}
        for n, (best, res) in found.items():
            dflt = res.get((256 if precision == "fp64" else 320, 0, 0))     # the library's default launch
            by[str(n)] = {"block": best[0], "ctas": best[1], "reg": best[2], "ms": res[best],
                          "default_ms": dflt,
                          "all_ms": {f"{b}/{c}/{r}": v for (b, c, r), v in sorted(res.items())}}
        big = str(max(found))
        cache[config_key(name, scheme, lr, rsolver, precision, dual, flu_nxt)] = {
            "block": by[big]["block"], "by_npg": by}
        with open(out or CACHE, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    return found


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scheme", default="mhm")
    ap.add_argument("--lr", default="plm")
    ap.add_argument("--rsolver", default="hllc")
    ap.add_argument("--precision", default="fp32")
    ap.add_argument("--dual", action="store_true")
    ap.add_argument("--npgs", default=",".join(str(n) for n in NPGS), help="batch sizes (patch groups)")
    ap.add_argument("--all", action="store_true", help="tune every configuration the benchmarks use")
    ap.add_argument("--out", default=None, help="table to update (default: gamer_b200/tuned.json)")
    a = ap.parse_args()
    npgs = tuple(int(v) for v in a.npgs.split(","))
    if a.all:
        for prec in ("fp32", "mixed", "fp64"):
            for lr, rs in (("plm", "hllc"), ("ppm", "roe")):
                print(f"== {prec} {lr} {rs}")
                tune(lr=lr, rsolver=rs, precision=prec, npgs=npgs, out=a.out)
        print("== mixed plm hllc dual")
        tune(lr="plm", rsolver="hllc", precision="mixed", dual=True, npgs=npgs, out=a.out)
    else:
        tune(a.scheme, a.lr, a.rsolver, a.precision, a.dual, npgs=npgs, out=a.out)


if __name__ == "__main__":
    main()
