"""Benchmark of the B200 patch-group fluid solver (one JSON line on rank 0).

Workload: 4096 patch groups (16^3 PG grid = 256^3 cells, ~16.7M cell updates per step), hydro
MHM + PLM (generalized MinMod, theta = 1.5) + HLLC, ideal gas gamma = 5/3, seeded Kelvin-Helmholtz
shear layer, FP32 (float arrays and arithmetic; `--precision mixed` keeps the internal-energy
recovery, dual-energy selection and flux-difference accumulation in double, `fp64` is the FLOAT8
build), coarse-fine flux planes stored.  FP32 is the headline policy: against analytic solutions
(`--workload accuracy`) FP32, mixed and FP64 reach the same L1 error where the truncation error
dominates, and the mixed policy is nowhere measurably more accurate than FP32 -- float storage
bounds both -- while FP32 is ~11% faster.  A step is one solver call over all 4096 patch groups;
inputs (655 MB) exceed the 126 MB L2, so no flush is needed between steps.

  value  : cell updates/s with the arrays resident in HBM (device entry point)
  e2e    : the same through the asynchronous host entry point (pinned host arrays, H2D of the input
           and D2H of output + flux inside the timed region)
  roofline: algorithmic HBM bytes per launch / launch time vs the measured copy bandwidth
  cpu_baseline: GAMER's own CPU_FluidSolver (compiled from source, OpenMP on all host cores) on the
           whole workload

--impl reference times the reference CPU solver alone (rank 0 only).
--gpus N (under torchrun): N independent replicas, each solving its own 4096 patch groups (weak
scaling, no data-path collective; the patch groups are independent once ghost zones are filled).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from gamer_b200 import ic  # noqa: E402

GAMMA = 5.0 / 3.0
NPD = 16                       # patch groups per dimension -> 4096 PGs
CELLS_PER_PG = 16 ** 3


# DRAM bytes per patch group of one mhm_kernel launch, from ncu captures of 1000 patch groups
# (FP32: read 160.04 MB + write 90.31 MB; mixed: read 160.05 MB + write 90.43 MB); traffic grows in
# proportion to the patch groups of a launch
DRAM_BYTES_PER_PG = {("fp32", "plm", "hllc"): (160.04e6 + 90.31e6) / 1000,
                     ("mixed", "plm", "hllc"): (160.05e6 + 90.43e6) / 1000}


# CTU+MHD, FP32 arrays, per patch group: Flu_In 5*22^3 + Mag_In 3*23*22^2 + Flu_Out 5*16^3 +
# Mag_Out 3*17*16^2 + flux 9*5*16^2 + Ele 9*2*17*16 reals
MHD_ALG_BYTES_PER_PG = 4 * (5 * 22 ** 3 + 3 * 23 * 22 ** 2 + 5 * 16 ** 3 + 3 * 17 * 16 ** 2 + 9 * 5 * 16 ** 2 + 9 * 2 * 17 * 16)


def algorithmic_bytes_per_pg(nxt, ncomp, rsize, store_flux=True):
    """Input read once + output written once (+ 9 flux planes): the per-PG figures of the
    measurement plan (59.06 B/cell for 20^3 FP32 without fluxes, 70.31 with)."""
    b = ncomp * nxt ** 3 * rsize + ncomp * CELLS_PER_PG * rsize
    if store_flux:
        b += 9 * ncomp * 16 * 16 * rsize
    return b


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.path is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
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
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_inputs(nxt, dual=False, seed=2025):
    box = ic.kelvin_helmholtz_box(NPD, seed=seed, gamma=GAMMA, dual=dual)
    dh = 1.0 / (NPD * 16)
    dt = ic.cfl_dt(box, GAMMA, dh, cfl=0.5)
    return ic.cut_patch_groups(box, nxt), dt, dh


def run_reference_cpu(x, dt, dh, variant, precision, steps, warmup, sample_pg, threads):
    """Reference CPU_FluidSolver (oracle/_ref) on the first sample_pg patch groups (the whole
    workload when sample_pg = npg), median of `steps` timed calls after `warmup`; returns
    (cell-updates/s, seconds per call)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    ref = po.RefSolver(variant, precision)
    xs = np.ascontiguousarray(x[:sample_pg], dtype=ref.dtype)
    for _ in range(warmup):
        ref.solve(xs, dt, dh, nthreads=threads)
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        ref.solve(xs, dt, dh, nthreads=threads)
        ts.append(time.perf_counter() - t0)
    t = statistics.median(ts)
    return sample_pg * CELLS_PER_PG / t, t


def run_reference_close_cpu(x, dt, dh, steps, sample_pg, threads):
    """Reference CorrectUnphysical (src/Fluid/Flu_Close.cpp:542, oracle/_ref) on the host over the
    output of a bounded sample of the workload's patch groups; returns cells screened per second."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    ref = po.RefSolver("mhm_plm_hllc", "fp32")
    xs = np.ascontiguousarray(x[:sample_pg], dtype=ref.dtype)
    r = ref.solve(xs, dt, dh, nthreads=threads)
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        ref.correct_unphysical(xs, r["out"], dt, dh, flux=r["flux"], corr="3d", scheme="hlle", nthreads=threads)
        ts.append(time.perf_counter() - t0)
    t = statistics.median(ts)
    return sample_pg * CELLS_PER_PG / t, t


def fixup_patches(x, dh, seed):
    """The 8 patches of every patch group of a FLU_NXT = 20 input ([8*npg][5][8][8][8]) and a flux
    difference of the size one coarse step leaves on each of their six faces."""
    npg = x.shape[0]
    pu = np.ascontiguousarray(x[:, :, 2:18, 2:18, 2:18].reshape(npg, 5, 2, 8, 2, 8, 2, 8)
                              .transpose(0, 2, 4, 6, 1, 3, 5, 7).reshape(8 * npg, 5, 8, 8, 8), dtype=np.float32)
    rng = np.random.default_rng(seed)
    pf = (1e-3 * dh * rng.standard_normal((8 * npg, 6, 5, 8, 8))).astype(np.float32)
    return pu, pf


def run_reference_fixup_cpu(x, dh, steps, sample_pg, threads):
    """Reference Flu_FixUp_Flux (src/Fluid/Flu_FixUp_Flux.cpp:23, oracle/_ref) on the host over the
    patches of a bounded sample of patch groups, all six faces carrying a flux difference; the time
    is that of the reference routine alone.  Returns patches per second."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    ref = po.RefSolver("mhm_plm_hllc", "fp32")
    pu, pf = fixup_patches(x[:sample_pg], dh, 5)
    has = np.ones((pu.shape[0], 6), np.uint8)
    ts = []
    for _ in range(steps):
        ref.fixup_flux(pu, pf, has, dh, nthreads=threads, timing=ts)
    t = statistics.median(ts)
    return pu.shape[0] / t, t


def time_reference_gpu(dev, x, dt, dh, variant, precision, steps, warmup, barrier, max_over_ranks):
    """The reference's own GPU kernel CUFLU_FluidSolver_MHM (oracle/_ref/libgrefgpu_*: built
    unmodified from the reference sources for sm_100a by oracle/build_ref_gpu.sh, with the launch of
    CUAPI_Asyn_FluidSolver and its global-memory scratch) on the same device-resident input: one
    launch over all patch groups per step, CUDA events on the launching stream.  Returns
    (ms per step, output array)."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    r = po.RefGpuSolver(variant, precision)
    dtype = torch.float64 if precision == "fp64" else torch.float32
    npg = x.shape[0]
    t_in = torch.from_numpy(np.ascontiguousarray(x)).to(dev, dtype)
    t_out = torch.empty((npg, 5, 16, 16, 16), dtype=dtype, device=dev)
    t_flx = torch.empty((npg, 9, 5, 16, 16), dtype=dtype, device=dev)
    st = torch.cuda.current_stream(dev)
    for _ in range(warmup):
        r.solve_device(t_in, t_out, dt, dh, t_flx, stream=st)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        r.solve_device(t_in, t_out, dt, dh, t_flx, stream=st)
    e1.record(st)
    torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1)) / steps
    out = t_out.cpu().numpy()
    del t_in, t_out, t_flx
    torch.cuda.empty_cache()
    return ms, out, r.scratch_bytes_per_pg


def time_ghost_fill(dev, npg, nxt, steps, barrier, max_over_ranks):
    """Ghost-zone fill of npg patch-group windows (FLU_NXT = nxt) whose 26 sides all come from the
    coarser level: gb_interpolate_device over each window's parents (conservative quadratic,
    Interpolate_Iterate with OPT__INT_PRIM, MONO_MAX_ITER = 10; smooth seeded coarse data) and
    gb_assemble_windows_device.  Returns the times per step and the bytes each kernel moves."""
    import torch
    from gamer_b200.fluid import assemble_windows_device, interpolate_device
    nw = nxt // 2
    n = nw + 2
    rng = np.random.default_rng(41)
    x = np.arange(n)
    ph = rng.random((npg, 3)) * 2.0 * np.pi
    base = (np.sin(0.5 * x[None, :, None, None] + ph[:, 0, None, None, None]) +
            np.sin(0.4 * x[None, None, :, None] + ph[:, 1, None, None, None]) +
            np.sin(0.3 * x[None, None, None, :] + ph[:, 2, None, None, None]))
    creg = np.empty((npg, 5, n, n, n), np.float32)
    creg[:, 0] = 1.0 + 0.2 * base
    creg[:, 1] = 0.3 * base
    creg[:, 2] = -0.2 * base
    creg[:, 3] = 0.1
    creg[:, 4] = 2.0 + 0.3 * base
    tc = torch.from_numpy(creg).to(dev)
    cint = torch.empty((npg, 5, nxt, nxt, nxt), dtype=torch.float32, device=dev)
    fine = torch.ones((npg, 5, 16, 16, 16), dtype=torch.float32, device=dev)
    nbr = torch.full((npg, 27), -1, dtype=torch.int32, device=dev)
    win = torch.empty_like(cint)
    st = torch.zeros(1, dtype=torch.int32, device=dev)
    kw = dict(iterate=True, int_prim=True, mono_max_iter=10, status=st)
    for _ in range(2):
        interpolate_device(tc, cint, "cquad", (1, 1, 1), (nw, nw, nw), **kw)
        assemble_windows_device(fine, nbr, cint, win)
    torch.cuda.synchronize()
    barrier()
    s = torch.cuda.current_stream(dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record(s)
    for _ in range(steps):
        interpolate_device(tc, cint, "cquad", (1, 1, 1), (nw, nw, nw), **kw)
    ev[1].record(s)
    for _ in range(steps):
        assemble_windows_device(fine, nbr, cint, win)
    ev[2].record(s)
    torch.cuda.synchronize()
    barrier()
    ti = max_over_ranks(ev[0].elapsed_time(ev[1])) / steps
    ta = max_over_ranks(ev[1].elapsed_time(ev[2])) / steps
    bi = npg * 5 * 4 * (n ** 3 + nxt ** 3)
    ba = npg * 5 * 4 * (2 * nxt ** 3 + 16 ** 3)
    return {"ghost_fill_ms": ti + ta, "ghost_fill_interpolate_ms": ti, "ghost_fill_assemble_ms": ta,
            "ghost_fill_interpolate_gbs": bi / (ti * 1e-3) / 1e9, "ghost_fill_assemble_gbs": ba / (ta * 1e-3) / 1e9,
            "ghost_fill_failed": int(st.item()),
            "ghost_fill_workload": f"{npg} windows of {nxt}^3, all 26 sides from the coarse level, CQuad + "
                                   f"Interpolate_Iterate, FP32"}


def frac_within_rel(dev, args, xs, dt, dh, variant, threads, tol=1e-5):
    """Fraction of output values (all variables, all cells) whose relative difference from the
    reference FP32 CPU solver is at most tol, for this run's policy: the first patch groups of the
    headline input, and 8 patch groups of a Mach-10 blast (a 1e3 density and pressure jump) at the
    same limiter; the blast's shocks are where float round-off is amplified."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    from gamer_b200.fluid import FluidSolver, SolverParams
    nxt = xs.shape[-1]
    s = FluidSolver(lr=args.lr, rsolver=args.rsolver, precision=args.precision, flu_nxt=nxt)
    res = {}
    bx = ic.blast_box(2, seed=13, gamma=GAMMA, dual=False)
    bdh = 1.0 / 32
    cases = {"kh": (xs, dt, dh), "blast": (ic.cut_patch_groups(bx, nxt), ic.cfl_dt(bx, GAMMA, bdh, cfl=0.5), bdh)}
    for name, (xx, tdt, tdh) in cases.items():
        xx = np.ascontiguousarray(xx, dtype=np.float32)
        ref = po.RefSolver(variant, "fp32").solve(xx, tdt, tdh, nthreads=threads)["out"].astype(np.float64)
        t_in = torch.from_numpy(xx).to(dev)
        t_out = torch.empty((xx.shape[0], 5, 16, 16, 16), dtype=torch.float32, device=dev)
        s.solve_device(t_in, t_out, SolverParams(dt=tdt, dh=tdh, StoreFlux=False))
        g = t_out.cpu().numpy().astype(np.float64)
        res[f"frac_within_1e-5_rel_{name}"] = float(np.mean(np.abs(g - ref) <= tol * np.abs(ref)))
        # momenta that pass through zero make a pure relative test meaningless there: the same
        # fraction over density and energy alone
        res[f"frac_within_1e-5_rel_{name}_dens_engy"] = float(np.mean(
            (np.abs(g - ref) <= tol * np.abs(ref))[:, [0, 4]]))
    res["frac_within_sample"] = (f"{xs.shape[0]} headline patch groups and 8 blast patch groups, this run's "
                                 f"policy against the reference FP32 CPU solver")
    s.close()
    return res


LEVEL_NPG = (512, 1536, 3072, 1024)


class Replicas:
    """One process per GPU (launched by torchrun), each solving its own patch groups: the process
    group, the barrier around every timed region and the maximum of a time over the ranks, so that
    a value is all ranks' cell updates over the slowest rank's time.  No data-path collective: the
    patch groups of the ranks are independent."""

    def __init__(self, world, rank, backend="nccl", timeout_s=120):
        self.world, self.rank, self.backend = world, rank, backend
        self.dist = None
        self.owner = False
        if world > 1:
            import datetime
            import torch.distributed as dist
            if not dist.is_initialized():
                dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
                self.owner = True
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, v):
        """The maximum of a float (or of every value of a dict of floats) over the ranks."""
        if self.dist is None:
            return v
        import torch
        dev = torch.device("cuda", torch.cuda.current_device()) if self.backend == "nccl" else torch.device("cpu")
        keys = sorted(v) if isinstance(v, dict) else None
        vals = [v[k] for k in keys] if keys is not None else [v]
        t = torch.tensor(vals, dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        out = [float(x) for x in t.cpu()]
        return dict(zip(keys, out)) if keys is not None else out[0]

    def close(self):
        if self.dist is not None and self.owner:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def run_levels(args, world, rank, local, rep):
    """Batched AMR sub-step: levels 0-3 with 512/1536/3072/1024 patch groups, MHM+PLM+HLLC with dual
    energy (mixed), Mach-10 blast with a 1e3 density/pressure jump on a lognormal background,
    dh_l = dh_0/2^l, dt_l = dt_0/2^l.  Times (a) one launch per level, (b) one multi-level launch,
    (c) the multi-level launch replayed from a captured CUDA graph."""
    import torch
    from gamer_b200.fluid import FluidSolver, SolverParams
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    box = ic.blast_box(16, seed=31 + rank, gamma=GAMMA, dual=True)
    dh0 = 1.0 / 256
    dt0 = ic.cfl_dt(box, GAMMA, dh0, cfl=0.5)
    base = ic.cut_patch_groups(box, 20)
    total = sum(LEVEL_NPG)
    x = base[np.arange(total) % base.shape[0]]
    dts = [dt0 / 2 ** l for l in range(4)]
    dhs = [dh0 / 2 ** l for l in range(4)]
    s = FluidSolver(lr="plm", rsolver="hllc", precision=args.precision, dual_energy=True, flu_nxt=20,
                    block_size=args.block or None)
    t_in = torch.from_numpy(x.astype(s.np_dtype)).to(dev)
    t_out = torch.empty((total, 6, 16, 16, 16), dtype=s.torch_dtype, device=dev)
    t_flx = torch.empty((total, 9, 6, 16, 16), dtype=s.torch_dtype, device=dev)
    t_de = torch.zeros((total, 16, 16, 16), dtype=torch.int8, device=dev)
    prm = SolverParams(dt=dt0, dh=dh0, StoreFlux=True)
    offs = np.concatenate([[0], np.cumsum(LEVEL_NPG)])
    st = torch.cuda.current_stream(dev)

    def per_level():
        for l in range(4):
            a, b = int(offs[l]), int(offs[l + 1])
            s.solve_device(t_in[a:b], t_out[a:b], SolverParams(dt=dts[l], dh=dhs[l], StoreFlux=True),
                           flux=t_flx[a:b], de_out=t_de[a:b], stream=st)

    def one_launch():
        s.solve_levels_device(t_in, t_out, LEVEL_NPG, dts, dhs, prm, flux=t_flx, de_out=t_de, stream=st)

    g = s.capture_levels(t_in, t_out, LEVEL_NPG, dts, dhs, prm, flux=t_flx, de_out=t_de)

    def graph():
        g.launch(st)

    def timeit(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    rep.barrier()
    with ClockSampler(local) as clk:
        ms = {"per_level": timeit(per_level, args.steps, args.warmup),
              "one_launch": timeit(one_launch, args.steps, args.warmup),
              "graph": timeit(graph, args.steps, args.warmup)}
    ms = rep.max(ms)
    ref_out = t_out.clone()
    per_level()
    torch.cuda.synchronize()
    same = bool(torch.equal(ref_out, t_out))
    g.close()
    cells = total * CELLS_PER_PG
    line = {"metric": "cell-updates/s (batched AMR sub-step, MHM+PLM+HLLC+dual energy, levels 0-3)",
            "value": world * cells / (ms["graph"] * 1e-3), "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms["graph"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": {"mixed": "f32+f64", "fp32": "f32", "fp64": "f64"}[args.precision],
            "data": "synthetic (seeded Mach-10 blast, 1e3 jump, lognormal background)",
            "config": {"workload": f"levels 0-3 with {'/'.join(map(str, LEVEL_NPG))} patch groups, dual energy",
                       "block": s.block_size()},
            "modes_ms": ms, "graph_equals_per_level": same,
            "speedup_graph_vs_per_level": ms["per_level"] / ms["graph"],
            "gpu_launches": args.steps, "clocks": clk.summary()}
    s.close()
    if rank == 0:
        print(json.dumps(line))
    return 0


def run_adjoint(args, world, rank, local, rep):
    """K = 8 MHM+PLM+HLLC steps of a periodic box of 1024 patch groups (8x8x16) and the hand-written
    adjoint of all 8 steps (per-step checkpoints), FP32 with double accumulation; loss = sum w*rho_K.
    Reports forward, backward and total time and the cell updates/s of forward + backward."""
    import torch
    from gamer_b200.adjoint import mhm_steps
    from gamer_b200.fluid import FluidSolver, SolverParams
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    K = 8
    prec = "fp64" if args.precision == "fp64" else "fp32"
    b = ic.supersonic_separable_box(8, gamma=GAMMA, seed=rank)
    dh = 1.0 / 128
    dt = ic.cfl_dt(b, GAMMA, dh, cfl=0.5)
    box = np.concatenate([ic.to_device_layout(b)] * 2, axis=1)          # [5][Z=256][Y=128][X=128]
    s = FluidSolver(precision=prec)
    prm = SolverParams(dt=dt, dh=dh)
    x0 = torch.from_numpy(box).to(device=dev, dtype=s.torch_dtype)
    w = torch.from_numpy(np.random.default_rng(7).standard_normal(box.shape[1:])).to(dev)
    st = torch.cuda.current_stream(dev)

    def run():
        x = x0.clone().requires_grad_(True)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(st)
        y = mhm_steps(x, K, s, prm)
        loss = (y[0].double() * w).sum()
        e[1].record(st)
        loss.backward()
        e[2].record(st)
        torch.cuda.synchronize()
        return e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2]), x.grad

    for _ in range(max(1, args.warmup)):
        run()
    rep.barrier()
    fw, bw = [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            f, bk, g = run()
            fw.append(f)
            bw.append(bk)
    f, bk = statistics.median(fw), statistics.median(bw)
    mx = rep.max({"f": f, "bk": bk})
    f, bk = mx["f"], mx["bk"]
    cells = K * 1024 * CELLS_PER_PG
    line = {"metric": "cell-updates/s (K=8 MHM+PLM+HLLC steps forward + hand-written adjoint, 1024 patch groups)",
            "value": world * cells / ((f + bk) * 1e-3), "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": f + bk, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64acc" if prec == "fp32" else "f64",
            "data": "synthetic (supersonic diagonal flow + separable sinusoids, periodic 128x128x256)",
            "config": {"workload": "K=8 steps, 1024 patch groups, checkpoint per step, loss = sum w*rho_K"},
            "forward_ms": f, "backward_ms": bk, "backward_over_forward": bk / f,
            "grad_norm": float(g.double().norm()),
            # per step: forward gather + solve + scatter; backward gather + scatter adjoint + the 4
            # adjoint kernels (one chunk of 1024 patch groups) + gather adjoint
            "gpu_launches": args.steps * K * ( 3 + 7 ), "clocks": clk.summary()}
    s.close()
    if rank == 0:
        print(json.dumps(line))
    return 0


def mag_window_20(b):
    """The face-centred B of the central 20^3 window of 22^3 MHD windows [npg][3][23*22*22] ->
    [npg][3][21*20*20] (component d keeps its faces 1..21 along d, cells 1..20 across)."""
    npg = b.shape[0]
    out = []
    for d in range(3):
        shp = [22, 22, 22]
        shp[2 - d] = 23                      # arrays are [k][j][i], the extent along d is one more
        a = b[:, d].reshape(npg, *shp)
        sl = [slice(None)] + [slice(1, 21)] * 3
        sl[3 - d] = slice(1, 22)
        out.append(a[tuple(sl)].reshape(npg, -1))
    return np.ascontiguousarray(np.stack(out, axis=1))


def run_mhd(args, world, rank, local, rep):
    """CTU + MHD (PLM, HLLD, constrained transport) on 2048 patch groups (divergence-free lognormal-like
    magnetised state, beta ~ 1), device arrays; sweeps the chunk size of the multi-kernel pipeline and
    reports mixed (headline) / FP32 / FP64 throughput and the reference CPU solver on a sample."""
    import torch
    from gamer_b200.fluid import FluidSolver, SolverParams
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from parity import mhd_case
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # 2048 patch groups: four seeded 8^3-PG periodic boxes (each 128^3 cells); --no-extras (profiling
    # runs): one box of --npd^3 patch groups (at most 8^3), mixed precision only
    if args.no_extras:
        parts = [mhd_case(npd=min(args.npd, 8), seed=11 + rank)]
    else:
        parts = [mhd_case(npd=8, seed=11 + 4 * rank + q) for q in range(4)]
    dt = min(p[2] for p in parts)
    dh = parts[0][3]
    # every precision and the reference see the same float-rounded state
    x = np.concatenate([p[0] for p in parts]).astype(np.float32).astype(np.float64)
    b = np.concatenate([p[1] for p in parts]).astype(np.float32).astype(np.float64)
    del parts
    npg = x.shape[0]
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True)
    st = torch.cuda.current_stream(dev)

    def time_prec(prec, chunk, steps, warmup, scheme="ctu", xb=None):
        s = FluidSolver(scheme=scheme, lr="plm", rsolver="hlld", precision=prec)
        s.set_mhd_chunk(chunk)
        dt_ = s.torch_dtype
        xi, bi = (x, b) if xb is None else xb
        t_in = torch.from_numpy(xi.astype(s.np_dtype)).to(dev)
        t_b = torch.from_numpy(bi.astype(s.np_dtype)).to(dev)
        t_out = torch.empty((npg, 5, 16, 16, 16), dtype=dt_, device=dev)
        t_bo = torch.empty((npg, 3, 17 * 256), dtype=dt_, device=dev)
        t_f = torch.empty((npg, 9, 5, 16, 16), dtype=dt_, device=dev)
        t_e = torch.empty((npg, 9, 2, 17 * 16), dtype=dt_, device=dev)

        def step():
            s.solve_device(t_in, t_out, prm, flux=t_f, mag_in=t_b, mag_out=t_bo, ele=t_e, stream=st)
        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            step()
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out = t_out.cpu().numpy()
        s.close()
        return ms, out

    sweep = {}
    ms = {}
    outs = {}
    rep.barrier()
    with ClockSampler(local) as clk:
        if not args.no_extras:
            for chunk in (16, 32, 64, 128, 256, 512, 1024, 2048):
                sweep[chunk], _ = time_prec("fp32", chunk, max(3, args.steps // 2), args.warmup)
        for prec in (("mixed",) if args.no_extras else ("mixed", "fp32", "fp64")):
            ms[prec], outs[prec] = time_prec(prec, 0, args.steps, args.warmup)
        # MHM_RP with MHD (first-order Riemann predictor + its own CT half step) on the same state
        ms_rp, ms_mm = {}, {}
        if not args.no_extras:
            for prec in ("fp32", "fp64"):
                ms_rp[prec], _ = time_prec(prec, 0, args.steps, args.warmup, scheme="mhm_rp")
            # MHM with MHD reads 20^3 windows: the central window of the same state
            xb20 = (np.ascontiguousarray(x[:, :, 1:21, 1:21, 1:21]), mag_window_20(b))
            for prec in ("fp32", "fp64"):
                ms_mm[prec], _ = time_prec(prec, 0, args.steps, args.warmup, scheme="mhm", xb=xb20)
    ms = rep.max(ms)
    ms_rp = rep.max(ms_rp) if ms_rp else ms_rp
    ms_mm = rep.max(ms_mm) if ms_mm else ms_mm
    sweep = {int(k): v for k, v in rep.max({str(k): v for k, v in sweep.items()}).items()} if sweep else sweep
    best = min(sweep, key=sweep.get) if sweep else None
    cells = npg * CELLS_PER_PG
    extras = {"chunk_sweep_fp32_ms": sweep, "best_chunk": best}
    for prec, v in ms_rp.items():
        extras[f"mhmrp_mhd_{prec}_ms"] = v
        extras[f"mhmrp_mhd_{prec}_cell_updates_per_s"] = world * cells / (v * 1e-3)
    for prec, v in ms_mm.items():
        extras[f"mhm_mhd_{prec}_ms"] = v
        extras[f"mhm_mhd_{prec}_cell_updates_per_s"] = world * cells / (v * 1e-3)
    cpu = None
    if rank == 0 and not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as po
        threads = os.cpu_count() or 1
        samp = min(64, npg)
        ref = po.RefSolver("ctu_plm_hlld_mhd", "fp32")
        xs, bs = x[:samp].astype(np.float32), b[:samp].astype(np.float32)
        ref.solve(xs, dt, dh, mag_in=bs, store_ele=True, nthreads=threads)
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            ref.solve(xs, dt, dh, mag_in=bs, store_ele=True, nthreads=threads)
            ts.append(time.perf_counter() - t0)
        v = samp * CELLS_PER_PG / statistics.median(ts)
        cpu = {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "reference",
               "sample": f"{samp} of {npg} patch groups, median of 3, reference CPU_FluidSolver_CTU (MHD, FP32) "
                         f"from source, OpenMP {threads} threads"}
        r64 = po.RefSolver("ctu_plm_hlld_mhd", "fp64").solve(xs.astype(np.float64), dt, dh, mag_in=bs.astype(np.float64),
                                                             nthreads=threads)["out"]
        for prec in ms:
            o = outs[prec][:samp].astype(np.float64)
            extras[f"l1_vs_fp64_reference_{prec}"] = float(np.abs(o - r64).sum() / np.abs(r64).sum())
        if ms_rp and po.ref_available("mhmrp_plm_hlld_mhd", "fp32"):
            rrp = po.RefSolver("mhmrp_plm_hlld_mhd", "fp32")
            rrp.solve(xs, dt, dh, mag_in=bs, store_ele=True, nthreads=threads)
            t0 = time.perf_counter()
            rrp.solve(xs, dt, dh, mag_in=bs, store_ele=True, nthreads=threads)
            extras["mhmrp_mhd_reference_cpu_cell_updates_per_s"] = samp * CELLS_PER_PG / (time.perf_counter() - t0)
    line = {"metric": f"cell-updates/s (CTU+PLM+HLLD+CT MHD, {npg} patch groups)",
            "value": world * cells / (ms["mixed"] * 1e-3), "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms["mixed"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (lognormal-like gas, beta ~ 1, uniform + curl of a random |k|<=4 vector potential)",
            "config": {"workload": f"CTU+MHD mixed, {npg} patch groups, FLU_NXT=22, StoreFlux, StoreElectric"},
            "fp32_cell_updates_per_s": world * cells / (ms["fp32"] * 1e-3) if "fp32" in ms else None,
            "fp64_cell_updates_per_s": world * cells / (ms["fp64"] * 1e-3) if "fp64" in ms else None,
            "roofline": {"bound": "hbm", "achieved": MHD_ALG_BYTES_PER_PG * npg / (ms["mixed"] * 1e-3) / 1e9,
                         "peak": load_peaks()[0], "unit": "GB/s",
                         "frac": MHD_ALG_BYTES_PER_PG * npg / (ms["mixed"] * 1e-3) / 1e9 / load_peaks()[0],
                         "traffic": None, "note": "achieved over the whole 11-kernel step (algorithmic bytes: "
                                                  "fluid + magnetic in/out, flux and Ele planes)"},
            "ms": ms, "cpu_baseline": cpu, "extras": extras, "gpu_launches": 11 * -(-npg // 512) * args.steps,
            "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(line))
    return 0


def measure_copy_pipeline(dev, h_in, h_out, h_flx, chunk=256, nstream=3):
    """The host entry point's copies alone: per chunk of patch groups an upload of the input and a
    download of output and fluxes, round-robin over the same number of streams, no kernels.
    Returns the ms of one pass (best of 3): the copy bound of the e2e leg."""
    import torch
    npg = h_in.shape[0]
    src, outs = torch.from_numpy(h_in), [torch.from_numpy(h_out), torch.from_numpy(h_flx)]
    streams = [torch.cuda.Stream(dev) for _ in range(nstream)]
    d_in = [torch.empty((chunk,) + tuple(h_in.shape[1:]), dtype=src.dtype, device=dev) for _ in range(nstream)]
    d_out = [[torch.empty((chunk,) + tuple(o.shape[1:]), dtype=o.dtype, device=dev) for o in outs] for _ in range(nstream)]
    best = None
    for _ in range(3):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for s in streams:
            s.wait_event(e0)
        for k, p0 in enumerate(range(0, npg, chunk)):
            n = min(chunk, npg - p0)
            q = k % nstream
            with torch.cuda.stream(streams[q]):
                d_in[q][:n].copy_(src[p0:p0 + n], non_blocking=True)
                for o, d in zip(outs, d_out[q]):
                    o[p0:p0 + n].copy_(d[:n], non_blocking=True)
        for s in streams:
            torch.cuda.current_stream(dev).wait_stream(s)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del d_in, d_out
    torch.cuda.empty_cache()
    return best


def measure_pcie(dev, h_src, h_dst):
    """Pinned host<->device copy rates (GB/s) of the host arrays of the e2e leg: one large
    cudaMemcpyAsync each way, best of 3, CUDA events."""
    import torch
    src = torch.from_numpy(h_src.reshape(-1))
    dst = torch.from_numpy(h_dst.reshape(-1))
    d_src = torch.empty_like(src, device=dev)
    d_dst = torch.empty_like(dst, device=dev)
    out = {}
    for name, (a, b, nbytes) in {"h2d_gbs": (d_src, src, src.numel() * src.element_size()),
                                 "d2h_gbs": (dst, d_dst, dst.numel() * dst.element_size())}.items():
        best = None
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            a.copy_(b, non_blocking=True)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        out[name] = nbytes / (best * 1e-3) / 1e9
    del d_src, d_dst
    torch.cuda.empty_cache()
    return out


def headline_metric(args):
    """The metric string both arms print (this solver and the reference CPU solver)."""
    return f"cell-updates/s (MHM+{args.lr.upper()}+{args.rsolver.upper()}, {NPD ** 3} patch groups)"


def headline_config(args, npg, nxt, world):
    return {"workload": f"MHM+{args.lr.upper()}+{args.rsolver.upper()} {args.precision}, {npg} patch groups "
                        f"({NPD * 16}^3 cells) per GPU, FLU_NXT={nxt}, StoreFlux",
            "l2": "inputs (>600 MB) larger than L2, no flush", "parallelism": f"replicas x{world}",
            "block": args.block or "default"}


def accuracy_cases(npd):
    """Problems with an analytic solution for the accuracy study, on an (npd*16)^3 periodic box:
    (name, box [v][x][y][z] (x, y, z), end time, perturbation amplitude, rho0, p0).  The end time
    is one period, after which the exact solution is the initial state."""
    g = GAMMA
    cases = []
    # linear acoustic wave along x (src/TestProblem/Hydro/AcousticWave: rho0 = 1, c_s = 1), GAMER's
    # default amplitude 1e-6 (example/test_problem/Hydro/AcousticWave/Input__TestProb) and 1e-3
    for amp in (1e-6, 1e-3):
        cases.append((f"acoustic_wave_amp{amp:g}", ic.acoustic_wave_box(npd, amp=amp, gamma=g), 1.0, amp, 1.0, 1.0 / g))
    # a density wave advected at Mach 30 in pressure balance: the kinetic energy is ~500x the
    # internal energy, so every pressure recovery E - 1/2 m^2/rho cancels ~3 digits
    n = npd * 16
    x = (np.arange(n) + 0.5) / n
    X = np.meshgrid(x, x, x, indexing="ij")[0]
    amp, rho0, p0 = 0.1, 1.0, 1.0 / g
    rho = rho0 * (1.0 + amp * np.sin(2.0 * np.pi * X))
    v0 = 30.0 * np.sqrt(g * p0 / rho0)
    zero = np.zeros_like(rho)
    cases.append(("cold_advection_mach30", ic.prim2cons(rho, zero + v0, zero, zero, zero + p0, g), 1.0 / v0, amp,
                  rho0, p0))
    return cases


def run_accuracy(args, world, rank, local, rep):
    """Accuracy of the three precision policies against analytic solutions (multi-step runs of the
    MHM+PLM+HLLC solver on a periodic box: ghost zones gathered on the device, all patch groups
    solved, interiors scattered back, every step).  L1 of the density perturbation (relative to its
    amplitude) and of the pressure (relative to p0) after one period, for FP32, mixed and FP64;
    the same fixed dt sequence (CFL 0.5 of the initial state) for every policy."""
    import torch
    from gamer_b200 import adjoint
    from gamer_b200.fluid import FluidSolver, SolverParams
    dev = torch.device("cuda", local)
    table = []
    t0 = time.perf_counter()
    for npd in (2, 4):
        dh = 1.0 / (npd * 16)
        for name, box, t_end, amp, rho0, p0 in accuracy_cases(npd):
            dt_cfl = ic.cfl_dt(box, GAMMA, dh, cfl=0.5)
            nstep = int(np.ceil(t_end / dt_cfl))
            dt = t_end / nstep
            exact = box
            row = {"case": name, "cells": (npd * 16) ** 3, "steps": nstep}
            for prec in ("fp32", "mixed", "fp64"):
                s = FluidSolver(lr="plm", rsolver="hllc", precision=prec)
                tb = torch.from_numpy(ic.to_device_layout(box)).to(dev, s.torch_dtype)
                prm = SolverParams(dt=dt, dh=dh)
                for _ in range(nstep):
                    tb = adjoint.step(s, tb, prm)
                torch.cuda.synchronize()
                res = ic.from_device_layout(tb.double().cpu().numpy())
                rho = res[0]
                ek = 0.5 * (res[1] ** 2 + res[2] ** 2 + res[3] ** 2) / rho
                pres = (GAMMA - 1.0) * (res[4] - ek)
                ek0 = 0.5 * (exact[1] ** 2 + exact[2] ** 2 + exact[3] ** 2) / exact[0]
                pres0 = (GAMMA - 1.0) * (exact[4] - ek0)
                row[f"l1_rho_{prec}"] = float(np.mean(np.abs(rho - exact[0])) / (rho0 * amp))
                row[f"l1_pres_{prec}"] = float(np.mean(np.abs(pres - pres0)) / p0)
                s.close()
            row["rho_mixed_over_fp64"] = row["l1_rho_mixed"] / row["l1_rho_fp64"]
            row["rho_fp32_over_fp64"] = row["l1_rho_fp32"] / row["l1_rho_fp64"]
            row["pres_mixed_over_fp32"] = row["l1_pres_mixed"] / row["l1_pres_fp32"]
            table.append(row)
    wall = time.perf_counter() - t0
    if rank == 0:
        big = [r for r in table if r["case"] == "acoustic_wave_amp0.001"][-1]
        line = {"metric": "L1 error ratio mixed/FP64 vs analytic (acoustic wave A=1e-3, 64^3, one period)",
                "value": big["rho_mixed_over_fp64"], "unit": "ratio", "n_gpus": world, "steps": big["steps"],
                "warmup": 0, "ms_per_step": None, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32+f64", "data": "synthetic (analytic acoustic wave and Mach-30 density advection)",
                "config": {"workload": "accuracy of FP32 / mixed / FP64 MHM+PLM+HLLC against analytic solutions, "
                                       "32^3 and 64^3 periodic boxes, one period", "parallelism": f"replicas x{world}"},
                "accuracy": table, "wall_s": wall}
        print(json.dumps(line))
    return 0


def run_ctu(args, world, rank, local, rep):
    """Hydro CTU (PLM with characteristic tracing, HLLC) on the headline's 4096 patch groups of the
    Kelvin-Helmholtz layer (FLU_NXT = 20): mixed (headline of this line), FP32 and FP64, device
    arrays, and the reference CTU CPU solver on a sample."""
    import torch
    from gamer_b200.fluid import FluidSolver, SolverParams
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    x, dt, dh = make_inputs(20, seed=2025 + rank)
    npg = x.shape[0]
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=True)
    st = torch.cuda.current_stream(dev)

    def time_prec(prec, steps, warmup):
        s = FluidSolver(scheme="ctu", lr="plm", rsolver="hllc", precision=prec)
        t_in = torch.from_numpy(x.astype(s.np_dtype)).to(dev)
        t_out = torch.empty((npg, 5, 16, 16, 16), dtype=s.torch_dtype, device=dev)
        t_f = torch.empty((npg, 9, 5, 16, 16), dtype=s.torch_dtype, device=dev)
        for _ in range(warmup):
            s.solve_device(t_in, t_out, prm, flux=t_f, stream=st)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            s.solve_device(t_in, t_out, prm, flux=t_f, stream=st)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        s.close()
        return ms

    rep.barrier()
    with ClockSampler(local) as clk:
        ms = {p: time_prec(p, args.steps, args.warmup) for p in ("mixed", "fp32", "fp64")}
    ms = rep.max(ms)
    cells = npg * CELLS_PER_PG
    cpu = None
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        v, _ = run_reference_cpu(x, dt, dh, "ctu_plm_hllc", "fp32", 3, 1, 128, threads)
        cpu = {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "reference",
               "sample": f"128 of {npg} patch groups, median of 3, reference CPU_FluidSolver_CTU (hydro, FP32) "
                         f"from source, OpenMP {threads} threads"}
    line = {"metric": f"cell-updates/s (CTU+PLM+HLLC hydro, {npg} patch groups)",
            "value": world * cells / (ms["mixed"] * 1e-3), "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms["mixed"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded Kelvin-Helmholtz shear layer)",
            "config": {"workload": f"CTU hydro mixed, {npg} patch groups, FLU_NXT=20, StoreFlux"},
            "fp32_cell_updates_per_s": world * cells / (ms["fp32"] * 1e-3),
            "fp64_cell_updates_per_s": world * cells / (ms["fp64"] * 1e-3),
            "ms": ms, "cpu_baseline": cpu, "gpu_launches": 6 * -(-npg // 512) * args.steps,
            "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(line))
    return 0


def run_close(args, world, rank, local, rep):
    """Flu_Close's CorrectUnphysical on the device (gb_fluid_correct_unphysical_device) over the
    headline's output (4096 patch groups of the Kelvin-Helmholtz layer after one MHM+PLM+HLLC step,
    every cell physical): the pass GAMER runs after every solve, a screen of every output cell.
    Mixed (this line's value) and FP32.  Algorithmic bytes: the output read once."""
    import torch
    from gamer_b200.fluid import FluidSolver, SolverParams
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    x, dt, dh = make_inputs(20, seed=2025 + rank)
    npg = x.shape[0]
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=True)
    st = torch.cuda.current_stream(dev)

    def time_prec(prec, steps, warmup):
        s = FluidSolver(precision=prec)
        t_in = torch.from_numpy(x.astype(s.np_dtype)).to(dev)
        t_out = torch.empty((npg, 5, 16, 16, 16), dtype=s.torch_dtype, device=dev)
        t_f = torch.empty((npg, 9, 5, 16, 16), dtype=s.torch_dtype, device=dev)
        counts = torch.zeros(2, dtype=torch.int32, device=dev)
        s.solve_device(t_in, t_out, prm, flux=t_f, stream=st)
        for _ in range(warmup):
            s.correct_unphysical_device(t_in, t_out, prm, flux=t_f, counts=counts, stream=st)
        torch.cuda.synchronize()
        rep.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            s.correct_unphysical_device(t_in, t_out, prm, flux=t_f, counts=counts, stream=st)
        e1.record(st)
        torch.cuda.synchronize()
        rep.barrier()
        ms = e0.elapsed_time(e1) / steps
        n = counts.tolist()
        s.close()
        return ms, n

    def time_fixup(steps, warmup):
        # Flu_FixUp_Flux over the 8 patches of every patch group (32768 patches), all six faces
        # carrying a flux difference of the size one coarse step leaves: the bound case
        s = FluidSolver(precision="mixed")
        npatch = 8 * npg
        pu, pf = fixup_patches(x, dh, 5 + rank)
        t_u = torch.from_numpy(pu).to(dev)
        t_f = torch.from_numpy(pf).to(dev)
        t_h = torch.ones((npatch, 6), dtype=torch.uint8, device=dev)
        fprm = SolverParams(dt=dt, dh=dh)
        for _ in range(warmup):
            s.flux_fixup_device(t_u, t_f, t_h, fprm, stream=st)
        torch.cuda.synchronize()
        rep.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            s.flux_fixup_device(t_u, t_f, t_h, fprm, stream=st)
        e1.record(st)
        torch.cuda.synchronize()
        rep.barrier()
        s.close()
        # algorithmic bytes: the 296 surface cells of each patch read and written, the flux read
        byt = npatch * (2 * 296 * 5 * 4 + 6 * 5 * 64 * 4 + 6)
        # the least DRAM traffic at 32-byte sectors: every row of 8 cells holds a surface cell, so
        # the whole fluid of a patch is read and written
        sec = npatch * (2 * 512 * 5 * 4 + 6 * 5 * 64 * 4 + 6)
        return e0.elapsed_time(e1) / steps, byt, sec

    def time_mhd_close(steps, warmup):
        # MHD_FixUp_Electric and Flu_FixUp_Flux with the magnetic energy over 32768 patches, every
        # side on a coarse-fine boundary and every sibling a leaf (the bound case), FP32
        s = FluidSolver(scheme="ctu", rsolver="hlld", precision="fp32")
        npatch = 8 * npg
        rng = np.random.default_rng(11 + rank)
        from gamer_b200.fluid import ELE_PER_PATCH
        mag = (0.5 * rng.standard_normal((npatch, 3, 576))).astype(np.float32)
        t_b = torch.from_numpy(mag).to(dev)
        t_e = torch.from_numpy((1e-3 * rng.standard_normal((npatch, ELE_PER_PATCH))).astype(np.float32)).to(dev)
        t_eb = torch.zeros_like(t_e)
        t_he = torch.ones((npatch, 18), dtype=torch.uint8, device=dev)
        t_sl = torch.ones((npatch, 6), dtype=torch.uint8, device=dev)
        pu, pf = fixup_patches(x, dh, 7 + rank)
        bx, by, bz = mag[:, 0].reshape(-1, 8, 8, 9), mag[:, 1].reshape(-1, 8, 9, 8), mag[:, 2].reshape(-1, 9, 8, 8)
        pu[:, 4] += 0.5 * ((0.5 * (bx[..., 1:] + bx[..., :-1])) ** 2 + (0.5 * (by[:, :, 1:] + by[:, :, :-1])) ** 2 +
                           (0.5 * (bz[:, 1:] + bz[:, :-1])) ** 2)      # the cells' magnetic energy
        t_u = torch.from_numpy(pu).to(dev)
        t_f = torch.from_numpy(pf).to(dev)
        t_h = torch.ones((npatch, 6), dtype=torch.uint8, device=dev)
        fprm = SolverParams(dt=dt, dh=dh)
        out = {}
        for name, fn in (("fixup_electric", lambda: s.fixup_electric_device(t_b, t_e, t_eb, t_he, t_sl, dh, stream=st)),
                         ("flux_fixup_mhd", lambda: s.flux_fixup_device(t_u, t_f, t_h, fprm, stream=st, magnetic=t_b))):
            for _ in range(warmup):
                fn()
            torch.cuda.synchronize()
            rep.barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(steps):
                fn()
            e1.record(st)
            torch.cuda.synchronize()
            rep.barrier()
            out[name] = e0.elapsed_time(e1) / steps
        s.close()
        # algorithmic bytes per patch: electric fix-up: both E arrays read and zeroed, the 756 B
        # components on the sides read and written; MHD flux fix-up: as the hydro one plus the
        # patch's face-centred field read
        ele_b = npatch * (4 * ELE_PER_PATCH * 4 + 2 * 756 * 4)
        fx_b = npatch * (2 * 296 * 5 * 4 + 6 * 5 * 64 * 4 + 6 + 3 * 576 * 4)
        return out, ele_b, fx_b

    with ClockSampler(local) as clk:
        res = {p: time_prec(p, args.steps, args.warmup) for p in ("mixed", "fp32")}
        fx_ms, fx_bytes, fx_sec = time_fixup(args.steps, args.warmup)
        mhd_ms, ele_bytes, fxm_bytes = time_mhd_close(args.steps, args.warmup)
    ms = rep.max({p: v[0] for p, v in res.items()})
    fx_ms = rep.max(fx_ms)
    mhd_ms = rep.max(mhd_ms)
    cells = npg * CELLS_PER_PG
    alg = cells * 5 * 4
    hbm_peak, peak_kind = load_peaks()
    achieved = alg / (ms["mixed"] * 1e-3) / 1e9
    cpu = None
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        try:
            v, _ = run_reference_close_cpu(x, dt, dh, 5, 512, threads)
            cpu = {"value": v, "unit": "cells/s", "cores": threads, "kind": "reference",
                   "sample": f"512 of {npg} patch groups, median of 5, reference CorrectUnphysical (FP32 build) "
                             f"from source on the output of one step, OpenMP {threads} threads"}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": "cells/s", "cores": threads, "kind": "reference",
                   "sample": f"unavailable: {e}"}
        try:
            v, _ = run_reference_fixup_cpu(x, dh, 5, 512, threads)
            fx_cpu = {"value": v, "unit": "patches/s", "cores": threads, "kind": "reference",
                      "sample": f"4096 patches (512 patch groups), median of 5, reference Flu_FixUp_Flux (FP32 "
                                f"build) alone, OpenMP {threads} threads"}
        except Exception as e:  # noqa: BLE001
            fx_cpu = {"value": None, "unit": "patches/s", "sample": f"unavailable: {e}"}
    else:
        fx_cpu = None
    line = {"metric": f"cells screened/s (Flu_Close CorrectUnphysical, {npg} patch groups)",
            "value": world * cells / (ms["mixed"] * 1e-3), "unit": "cells/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms["mixed"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded Kelvin-Helmholtz shear layer, one MHM step)",
            "config": {"workload": f"CorrectUnphysical after MHM+PLM+HLLC mixed, {npg} patch groups, 3D, HLLE"},
            "fp32_cells_per_s": world * cells / (ms["fp32"] * 1e-3), "ms": ms, "cpu_baseline": cpu,
            "cells_corrected": {p: v[1] for p, v in res.items()},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "algorithmic_bytes_per_launch": alg,
                         "peak_source": f"{peak_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)"},
            "flux_fixup": {"workload": f"Flu_FixUp_Flux, {8 * npg} patches, all 6 faces, mixed",
                           "ms": fx_ms, "algorithmic_bytes": fx_bytes,
                           "patches_per_s": world * 8 * npg / (fx_ms * 1e-3), "cpu_baseline": fx_cpu,
                           "gbs": fx_bytes / (fx_ms * 1e-3) / 1e9,
                           "frac_of_hbm": fx_bytes / (fx_ms * 1e-3) / 1e9 / hbm_peak,
                           "sector_min_bytes": fx_sec,
                           "sector_min_gbs": fx_sec / (fx_ms * 1e-3) / 1e9,
                           "frac_of_hbm_at_sector_min": fx_sec / (fx_ms * 1e-3) / 1e9 / hbm_peak},
            "mhd_fixup_electric": {"workload": f"MHD_FixUp_Electric, {8 * npg} patches, all 18 sides, FP32",
                                   "ms": mhd_ms["fixup_electric"], "algorithmic_bytes": ele_bytes,
                                   "gbs": ele_bytes / (mhd_ms["fixup_electric"] * 1e-3) / 1e9,
                                   "frac_of_hbm": ele_bytes / (mhd_ms["fixup_electric"] * 1e-3) / 1e9 / hbm_peak},
            "mhd_flux_fixup": {"workload": f"Flu_FixUp_Flux with MHD, {8 * npg} patches, all 6 faces, FP32",
                               "ms": mhd_ms["flux_fixup_mhd"], "algorithmic_bytes": fxm_bytes,
                               "gbs": fxm_bytes / (mhd_ms["flux_fixup_mhd"] * 1e-3) / 1e9,
                               "frac_of_hbm": fxm_bytes / (mhd_ms["flux_fixup_mhd"] * 1e-3) / 1e9 / hbm_peak},
            "gpu_launches": 5 * args.steps, "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--lr", default="plm")
    ap.add_argument("--rsolver", default="hllc")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "mixed", "fp64"])
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--no-extras", action="store_true", help="skip the FP32/FP64/PPM comparison legs")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-array leg (profiling runs)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline and accuracy legs (profiling runs)")
    ap.add_argument("--npd", type=int, default=16, help="patch groups per dimension (default 16 -> 4096)")
    ap.add_argument("--workload", default="kh", choices=["kh", "levels", "adjoint", "mhd", "ctu", "close", "accuracy"],
                    help="kh: 4096 patch groups (headline); levels: batched AMR sub-step; adjoint: K=8 steps + adjoint")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    global NPD
    NPD = args.npd

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    nxt = 22 if args.lr == "ppm" else 20
    variant = f"mhm_{args.lr}_{args.rsolver}"
    threads = os.cpu_count() or 1

    if args.impl == "ours" and args.workload != "kh":
        import torch
        torch.cuda.set_device(local)
        rep = Replicas(world, rank)
        fn = {"levels": run_levels, "adjoint": run_adjoint, "mhd": run_mhd, "ctu": run_ctu,
              "close": run_close, "accuracy": run_accuracy}[args.workload]
        rc = fn(args, world, rank, local, rep)
        rep.close()
        return rc

    if args.impl == "reference":
        if rank != 0:
            return 0
        x, dt, dh = make_inputs(nxt)
        npg_full = x.shape[0]
        # every step is the whole workload (all patch groups), as in this solver's arm
        v, t = run_reference_cpu(x, dt, dh, variant, "fp64" if args.precision == "fp64" else "fp32",
                                 args.steps, args.warmup, npg_full, threads)
        line = {"impl": "reference", "metric": headline_metric(args),
                "value": v, "unit": "cell-updates/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "f32",
                "data": "synthetic (seeded Kelvin-Helmholtz shear layer)",
                "config": headline_config(args, npg_full, nxt, args.gpus),
                "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "reference",
                                 "sample": f"all {npg_full} patch groups per step (median of {args.steps}), "
                                           f"reference CPU_FluidSolver built from source, OpenMP {threads} threads"},
                "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import torch
    from gamer_b200.fluid import FluidSolver, PinnedArray, SolverParams

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    rep = Replicas(world, rank)
    barrier, max_over_ranks = rep.barrier, rep.max

    x, dt, dh = make_inputs(nxt, seed=2025 + rank)
    npg = x.shape[0]

    def time_device(precision, lr, rsolver, steps, warmup, block=0, scheme="mhm"):
        nx = 22 if (lr == "ppm" or scheme == "mhm_rp") else 20
        xx = x if nx == nxt else make_inputs(nx, seed=2025 + rank)[0]
        s = FluidSolver(scheme=scheme, lr=lr, rsolver=rsolver, precision=precision, flu_nxt=nx,
                        block_size=block or None)
        t_in = torch.from_numpy(np.ascontiguousarray(xx, dtype=s.np_dtype)).to(dev)
        t_out = torch.empty((npg, 5, 16, 16, 16), dtype=s.torch_dtype, device=dev)
        t_flx = torch.empty((npg, 9, 5, 16, 16), dtype=s.torch_dtype, device=dev)
        prm = SolverParams(dt=dt, dh=dh, StoreFlux=True)
        st = torch.cuda.current_stream(dev)
        for _ in range(warmup):
            s.solve_device(t_in, t_out, prm, flux=t_flx, stream=st)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        ev[0].record(st)
        for k in range(steps):
            s.solve_device(t_in, t_out, prm, flux=t_flx, stream=st)
            ev[k + 1].record(st)
        torch.cuda.synchronize()
        barrier()
        per = [ev[k].elapsed_time(ev[k + 1]) for k in range(steps)]
        total_ms = ev[0].elapsed_time(ev[steps])
        status = s.status()
        out = t_out.cpu().numpy()
        s.close()
        del t_in, t_out, t_flx
        torch.cuda.empty_cache()
        return total_ms, per, status, out, s.np_dtype

    # ---- headline: device-resident ------------------------------------------------------------
    with ClockSampler(local) as clk:
        total_ms, per, status, out_main, _ = time_device(args.precision, args.lr, args.rsolver, args.steps,
                                                         args.warmup, args.block)
    clocks = clk.summary()
    total_ms = max_over_ranks(total_ms)
    ms_step = total_ms / args.steps
    value = world * npg * CELLS_PER_PG / (ms_step * 1e-3)

    rsize = 8 if args.precision == "fp64" else 4
    alg_bytes = npg * algorithmic_bytes_per_pg(nxt, 5, rsize)
    mean_launch_ms = statistics.mean(per)
    hbm_peak, peak_kind = load_peaks()
    achieved = alg_bytes / (mean_launch_ms * 1e-3) / 1e9

    # ---- e2e: host arrays through the C ABI -----------------------------------------------------
    # GAMER's pattern (src/Main/InvokeSolver.cpp:214-245): two pinned buffer sets; the asynchronous
    # host-array call of batch k (H2D, solve, D2H inside) runs while the host prepares batch k+1 in
    # the other set.  `value` of e2e: back-to-back asynchronous calls, ended by gb_fluid_synchronize
    # (host wall clock, every copy inside); `prepare_overlap`: how much of a host-side fill of the
    # next batch's input (a copy of the 655 MB input array) the call hides.
    e2e = None
    if not args.no_e2e:
        s = FluidSolver(lr=args.lr, rsolver=args.rsolver, precision=args.precision, flu_nxt=nxt,
                        block_size=args.block or None)
        dtype = s.np_dtype
        sets = [dict(inp=PinnedArray(x.shape, dtype), out=PinnedArray((npg, 5, 16, 16, 16), dtype),
                     flx=PinnedArray((npg, 9, 5, 16, 16), dtype)) for _ in range(2)]
        for b in sets:
            b["inp"].array[...] = x
        prm = SolverParams(dt=dt, dh=dh, StoreFlux=True)
        e2e_steps = max(4, args.steps // 4)

        def call(k):
            b = sets[k % 2]
            s.solve_host_async(b["inp"].array, b["out"].array, prm, flux=b["flx"].array)

        def fill(k):
            np.copyto(sets[k % 2]["inp"].array, x)

        for k in range(2):
            call(k)
        s.synchronize()
        barrier()
        t0 = time.perf_counter()
        for k in range(e2e_steps):
            call(k)
        s.synchronize()
        e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3) / e2e_steps
        # the host-side fill alone, then fill and call overlapped (call k, fill k+1, synchronise)
        t0 = time.perf_counter()
        for k in range(e2e_steps):
            fill(k)
        fill_ms = max_over_ranks((time.perf_counter() - t0) * 1e3) / e2e_steps
        barrier()
        t0 = time.perf_counter()
        for k in range(e2e_steps):
            call(k)
            fill(k + 1)
            s.synchronize()
        pipe_ms = max_over_ranks((time.perf_counter() - t0) * 1e3) / e2e_steps
        h2d = x.size * np.dtype(dtype).itemsize
        d2h = (sets[0]["out"].array.size + sets[0]["flx"].array.size) * np.dtype(dtype).itemsize
        matches = bool(np.array_equal(sets[0]["out"].array, out_main) and np.array_equal(sets[1]["out"].array, out_main))
        pcie = measure_pcie(dev, sets[0]["inp"].array, sets[0]["out"].array)      # overwrites out
        # copy bound of a step: the same chunked uploads and downloads without the kernels
        bound_ms = measure_copy_pipeline(dev, sets[0]["inp"].array, sets[0]["out"].array, sets[0]["flx"].array)
        hidden = (e2e_ms + fill_ms - pipe_ms) / min(e2e_ms, fill_ms)
        e2e = {"value": world * npg * CELLS_PER_PG / (e2e_ms * 1e-3), "unit": "cell-updates/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": e2e_ms, "launches_per_step": -(-npg // 256),
               "entry_point": "gb_fluid_solve_host_async + gb_fluid_synchronize, two pinned buffer sets",
               "pcie": pcie, "copy_bound_ms": bound_ms, "copy_bound_frac": bound_ms / e2e_ms,
               "prepare_overlap": {"call_ms": e2e_ms, "host_fill_ms": fill_ms, "call_then_fill_ms": pipe_ms,
                                   "hidden_frac": hidden,
                                   "fill": "np.copyto of the next batch's input into the other pinned set"},
               "matches_device_result": matches}
        s.close()
        for b in sets:
            for a in b.values():
                a.free()

    extras = {}
    cpu_base = None
    if rank == 0 and not args.no_cpu:
        # ---- accuracy of this run against the reference FP64 solver on a sample ------------------
        try:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import pyoracle as po
            samp = 64
            ref64 = po.RefSolver(variant, "fp64").solve(x[:samp].astype(np.float32).astype(np.float64), dt, dh,
                                                        nthreads=threads)["out"]
            extras["l1_vs_fp64_reference"] = float(np.abs(out_main[:samp].astype(np.float64) - ref64).sum()
                                                   / np.abs(ref64).sum())
            extras["l1_sample"] = f"first {samp} patch groups, FP64 reference on the float-rounded input"
        except Exception as e:  # noqa: BLE001
            extras["l1_vs_fp64_reference"] = f"unavailable: {e}"
        # ---- per-cell parity gate: fraction of output values within a pure relative 1e-5 of the
        # reference FP32 solver, on the headline input and on a Mach-10 blast (shocks) ----------
        if args.precision != "fp64":
            try:
                extras.update(frac_within_rel(dev, args, x[:64], dt, dh, variant, threads))
            except Exception as e:  # noqa: BLE001
                extras["frac_within_1e-5"] = f"unavailable: {e}"
        # ---- CPU baseline: the reference solver on the host cores ------------------------------
        try:
            v, t = run_reference_cpu(x, dt, dh, variant, "fp64" if args.precision == "fp64" else "fp32",
                                     5, 3, npg, threads)
            cpu_base = {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "reference",
                        "ms_per_step": t * 1e3,
                        "sample": f"all {npg} patch groups per step, median of 5 after 3 warm-up calls, "
                                  f"reference CPU_FluidSolver "
                                  f"({'FLOAT8' if args.precision == 'fp64' else 'FP32'} build) from source, "
                                  f"OpenMP {threads} threads"}
        except Exception as e:  # noqa: BLE001
            cpu_base = {"value": None, "unit": "cell-updates/s", "cores": threads, "kind": "reference",
                        "sample": f"unavailable: {e}"}

    # ---- Flu_Close: the first-order-flux correction pass over this workload's output ----------
    # (every cell is physical here, so this is the cost GAMER pays on every step: one test of
    # every output cell; algorithmic bytes = the output read once)
    if not args.no_extras:
        s = FluidSolver(lr=args.lr, rsolver=args.rsolver, precision=args.precision, flu_nxt=nxt,
                        block_size=args.block or None)
        t_in = torch.from_numpy(np.ascontiguousarray(x, dtype=s.np_dtype)).to(dev)
        t_out = torch.empty((npg, 5, 16, 16, 16), dtype=s.torch_dtype, device=dev)
        t_flx = torch.empty((npg, 9, 5, 16, 16), dtype=s.torch_dtype, device=dev)
        counts = torch.zeros(2, dtype=torch.int32, device=dev)
        prm = SolverParams(dt=dt, dh=dh, StoreFlux=True)
        st = torch.cuda.current_stream(dev)
        s.solve_device(t_in, t_out, prm, flux=t_flx, stream=st)
        n = max(5, args.steps)
        for _ in range(3):
            s.correct_unphysical_device(t_in, t_out, prm, flux=t_flx, counts=counts, stream=st)
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(n):
            s.correct_unphysical_device(t_in, t_out, prm, flux=t_flx, counts=counts, stream=st)
        e1.record(st)
        torch.cuda.synchronize()
        barrier()
        cms = max_over_ranks(e0.elapsed_time(e1) / n)
        rb = npg * 5 * CELLS_PER_PG * (8 if args.precision == "fp64" else 4)
        extras["close_correct_unphysical_ms"] = cms
        extras["close_correct_unphysical_gbs"] = rb / (cms * 1e-3) / 1e9
        extras["close_correct_unphysical_frac_of_step"] = cms / ms_step
        extras["close_cells_corrected"] = int(counts[0].item())
        s.close()
        del t_in, t_out, t_flx
        torch.cuda.empty_cache()

    # ---- comparison legs: the same solver in plain FP32 and plain FP64, PPM+Roe, and the exact
    # Riemann solver ----------------------------------------------------------------------------
    # (with the L1 error of each leg against the reference FLOAT8 solver on its first 64 patch groups)
    if not args.no_extras:
        legs = [("fp64", "plm", "hllc", "mhm"), ("fp32", "plm", "hllc", "mhm"), ("mixed", "plm", "hllc", "mhm"),
                ("mixed", "ppm", "roe", "mhm"),
                ("fp64", "ppm", "roe", "mhm"), ("mixed", "plm", "exact", "mhm"), ("mixed", "plm", "hllc", "mhm_rp"),
                ("fp64", "plm", "hllc", "mhm_rp")]
        for prec, lr, rs, sch in legs:
            if (prec, lr, rs, sch) == (args.precision, args.lr, args.rsolver, "mhm"):
                continue
            key = f"{prec}_{lr}_{rs}" + ("_mhm_rp" if sch == "mhm_rp" else "")
            n = max(3, args.steps // 4)
            try:
                tm, pr, st_, o, _ = time_device(prec, lr, rs, n, 3, scheme=sch)
            except Exception as e:  # noqa: BLE001  (a leg that cannot run is reported, the line stands)
                extras[f"{key}_cell_updates_per_s"] = f"unavailable: {e}"
                continue
            tm = max_over_ranks(tm)
            extras[f"{key}_cell_updates_per_s"] = world * npg * CELLS_PER_PG / (tm / n * 1e-3)
            if rank == 0 and not args.no_cpu:
                try:
                    nx = 22 if (lr == "ppm" or sch == "mhm_rp") else 20
                    xs = (x if nx == nxt else make_inputs(nx, seed=2025 + rank)[0])[:64]
                    xs = xs if prec == "fp64" else xs.astype(np.float32).astype(np.float64)
                    leg_variant = ("mhmrp" if sch == "mhm_rp" else "mhm") + f"_{lr}_{rs}"
                    r64 = po.RefSolver(leg_variant, "fp64").solve(xs, dt, dh, nthreads=threads)["out"]
                    extras[f"l1_vs_fp64_reference_{key}"] = float(
                        np.abs(o[:64].astype(np.float64) - r64).sum() / np.abs(r64).sum())
                except Exception as e:  # noqa: BLE001
                    extras[f"l1_vs_fp64_reference_{key}"] = f"unavailable: {e}"

    # ---- ghost-zone fill of the same patch groups from a coarser level (every side coarse, the worst
    # case): the windows interpolated from their parents with the reference's default hydro path
    # (conservative quadratic, Interpolate_Iterate with OPT__INT_PRIM and MONO_MAX_ITER = 10), then
    # assembled; timed beside the solve -------------------------------------------------------
    if not args.no_extras:
        try:
            extras.update(time_ghost_fill(dev, npg, nxt, max(3, args.steps // 4), barrier, max_over_ranks))
            extras["ghost_fill_frac_of_step"] = extras["ghost_fill_ms"] / ms_step
        except Exception as e:  # noqa: BLE001
            extras["ghost_fill_ms"] = f"unavailable: {e}"

    # ---- the reference's own GPU kernel on this GPU (same input, device resident): FP32 and FLOAT8
    # builds, against this solver's mixed / FP32 and FP64 policies -----------------------------
    if not args.no_extras:
        ours = {p: extras.get(f"{p}_{args.lr}_{args.rsolver}_cell_updates_per_s") for p in ("mixed", "fp32", "fp64")}
        ours[args.precision] = value
        for rprec in ("fp32", "fp64"):
            key = f"reference_gpu_{rprec}_{args.lr}_{args.rsolver}"
            try:
                n = max(3, args.steps // 4)
                rms, rout, sbytes = time_reference_gpu(dev, x, dt, dh, variant, rprec, n, 3, barrier, max_over_ranks)
                rv = world * npg * CELLS_PER_PG / (rms * 1e-3)
                extras[f"{key}_cell_updates_per_s"] = rv
                extras[f"{key}_ms"] = rms
                extras[f"{key}_scratch_bytes_per_pg"] = sbytes
                for pol in (("fp32", "mixed") if rprec == "fp32" else ("fp64",)):
                    if isinstance(ours.get(pol), float):
                        extras[f"ratio_{pol}_vs_{key}"] = ours[pol] / rv
                if rprec == "fp32" and args.precision != "fp64":
                    extras[f"{key}_max_scaled_diff_vs_this_run"] = float(
                        np.max(np.abs(rout.astype(np.float64) - out_main) /
                               (np.abs(rout.astype(np.float64)) + np.sqrt(np.mean(rout.astype(np.float64) ** 2)))))
            except Exception as e:  # noqa: BLE001  (a leg that cannot run is reported, the line stands)
                extras[f"{key}_cell_updates_per_s"] = f"unavailable: {e}"
        extras["reference_gpu_build"] = ("CUFLU_FluidSolver_MHM from the reference sources, unmodified, nvcc "
                                         "sm_100a -O3 -Xptxas -dlcm=ca -prec-div=false -ftz=true, maxrregcount "
                                         "128 (FP32) / 192 (FLOAT8), 512 / 256 threads, one CTA per patch group")

    if rank == 0:
        line = {
            "metric": headline_metric(args),
            "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": {"mixed": "f32+f64", "fp32": "f32", "fp64": "f64"}[args.precision],
            "data": "synthetic (seeded Kelvin-Helmholtz shear layer)",
            "config": dict(headline_config(args, npg, nxt, world), block=args.block or "default"),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak,
                         "traffic": (DRAM_BYTES_PER_PG[(args.precision, args.lr, args.rsolver)] * npg
                                     if (args.precision, args.lr, args.rsolver) in DRAM_BYTES_PER_PG else None),
                         "traffic_kind": "constant from an ncu capture, not measured by this run",
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one 1000-patch-group "
                                           "launch of this kernel, scaled by patch groups",
                         "peak_source": f"{peak_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)",
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "mean_launch_ms": mean_launch_ms},
            "cpu_baseline": cpu_base,
            "e2e": e2e,
            "gpu_launches": args.steps,
            "clocks": clocks,
            "status": status,
            "extras": extras,
        }
        print(json.dumps(line))
    rep.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
