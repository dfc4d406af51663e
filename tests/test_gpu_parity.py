"""GPU parity of the MHM solver (hydro) against the reference CPU solver, through the C ABI.

The reference is GAMER's own CPU_FluidSolver built from source (oracle/_ref); the C restatement
(oracle/gamer_oracle.c) is pinned bit-for-bit against it by tests/test_oracle.py.
"""
import numpy as np
import pytest

import pyoracle as po
from gamer_b200.fluid import FluidSolver, FluidSolverError, SolverParams, STATUS_UNPHYSICAL
from parity import (GAMMA, RTOL32, RTOL64, blast_case, frac_rel_within, gpu_solve, kh_case, l1_rel,
                    lognormal_case, scaled_err)

pytestmark = pytest.mark.gpu

VARIANTS = [("plm", "hllc", False), ("plm", "roe", False), ("plm", "hlle", False),
            ("ppm", "roe", False), ("ppm", "hllc", False), ("plm", "hllc", True)]


def _ref(lr, rs, dual, prec):
    return po.RefSolver(po.ref_variant_name("mhm", lr, rs, dual=dual), prec)


@pytest.mark.parametrize("lr,rs,dual", VARIANTS)
def test_fp32_matches_reference_fp32(cuda_device, lr, rs, dual):
    nxt = 22 if lr == "ppm" else 20
    x, dt, dh = lognormal_case(npd=4, seed=11, nxt=nxt, dual=dual)
    ref = _ref(lr, rs, dual, "fp32").solve(x, dt, dh, limiter="gminmod", minmod_coeff=1.5)
    s = FluidSolver(lr=lr, rsolver=rs, precision="fp32", dual_energy=dual, flu_nxt=nxt)
    g = gpu_solve(s, x, SolverParams(dt=dt, dh=dh))
    e_out = scaled_err(g["out"], ref["out"])
    e_flx = scaled_err(g["flux"], ref["flux"], axis_var=2)
    assert e_out <= RTOL32, e_out
    assert e_flx <= RTOL32, e_flx
    # most cells also pass a pure relative 1e-5 test (momenta near zero excepted)
    assert frac_rel_within(g["out"], ref["out"], RTOL32) > 0.99
    if dual:
        assert np.array_equal(g["de"], ref["de"])
    assert s.status() == 0


@pytest.mark.parametrize("lr,rs,dual", VARIANTS)
def test_fp64_matches_reference_fp64(cuda_device, lr, rs, dual):
    nxt = 22 if lr == "ppm" else 20
    x, dt, dh = lognormal_case(npd=2, seed=5, nxt=nxt, dual=dual)
    s = FluidSolver(lr=lr, rsolver=rs, precision="fp64", dual_energy=dual, flu_nxt=nxt)
    ref = _ref(lr, rs, dual, "fp64").solve(x, dt, dh)
    g = gpu_solve(s, x, SolverParams(dt=dt, dh=dh))
    assert scaled_err(g["out"], ref["out"]) <= RTOL64
    assert scaled_err(g["flux"], ref["flux"], axis_var=2) <= RTOL64
    if dual:
        assert np.array_equal(g["de"], ref["de"])


@pytest.mark.parametrize("dual,nxt", [(True, 22), (False, 24)])
def test_fp64_ppm_dual_energy_and_wide_window(cuda_device, dual, nxt):
    """FP64 PPM (slopes formed in place) with dual energy (6 variables, 219 KB of shared memory), or
    with a 24^3 input of which the central 22^3 window is used (200 KB)."""
    x, dt, dh = lognormal_case(npd=1, seed=5, nxt=nxt, dual=dual)
    ref = _ref("ppm", "roe", dual, "fp64").solve(x, dt, dh)
    s = FluidSolver(lr="ppm", rsolver="roe", precision="fp64", dual_energy=dual, flu_nxt=nxt)
    g = gpu_solve(s, x, SolverParams(dt=dt, dh=dh))
    assert scaled_err(g["out"], ref["out"]) <= RTOL64
    assert scaled_err(g["flux"], ref["flux"], axis_var=2) <= RTOL64
    if dual:
        assert np.array_equal(g["de"], ref["de"])


def test_fp64_ppm_dual_energy_24_cubed_input_matches_reference(cuda_device):
    """FP64 PPM with dual energy and a 24^3 input: the largest configuration, 219 KB of shared memory
    per CTA with single-buffered flux planes; the reference reads the central 22^3 window."""
    x, dt, dh = lognormal_case(npd=2, seed=5, nxt=24, dual=True)
    ref = _ref("ppm", "roe", True, "fp64").solve(x, dt, dh)
    s = FluidSolver(lr="ppm", rsolver="roe", precision="fp64", dual_energy=True, flu_nxt=24)
    g = gpu_solve(s, x, SolverParams(dt=dt, dh=dh))
    assert scaled_err(g["out"], ref["out"]) <= RTOL64
    assert scaled_err(g["flux"], ref["flux"], axis_var=2) <= RTOL64
    assert np.array_equal(g["de"], ref["de"])


def test_fp64_ppm_blast_with_retries(cuda_device):
    """FP64 PPM (slopes formed in place) on the Mach-10 blast with MinMod retries."""
    x, dt, dh = blast_case(npd=2, seed=13, nxt=22, dual=False)
    prm = SolverParams(dt=2.0 * dt, dh=dh, MinMod_MaxIter=3)
    ref = _ref("ppm", "roe", False, "fp64").solve(x, 2.0 * dt, dh, minmod_maxiter=3)
    g = gpu_solve(FluidSolver(lr="ppm", rsolver="roe", precision="fp64", flu_nxt=22), x, prm, pg_fail=True)
    # FMA contraction differences (~1e-16) grow through the 1e3 shock and PPM's steeper stencil
    # (1.2e-9 observed; the PLM blast stays within 1e-9)
    assert scaled_err(g["out"], ref["out"]) <= 1e-8


@pytest.mark.parametrize("lr,rs", [("plm", "hllc"), ("ppm", "roe")])
def test_mixed_is_closer_to_fp64_oracle_than_its_fp32_inputs_allow(cuda_device, lr, rs):
    """Mixed precision vs the FP64 oracle run on the same (float-rounded) input: its error must not
    exceed the FP32 path's error."""
    nxt = 22 if lr == "ppm" else 20
    x, dt, dh = kh_case(npd=2, seed=9, nxt=nxt)
    x32 = x.astype(np.float32)
    ref64 = _ref(lr, rs, False, "fp64").solve(x32.astype(np.float64), dt, dh)
    g32 = gpu_solve(FluidSolver(lr=lr, rsolver=rs, precision="fp32", flu_nxt=nxt), x32, SolverParams(dt=dt, dh=dh))
    gmx = gpu_solve(FluidSolver(lr=lr, rsolver=rs, precision="mixed", flu_nxt=nxt), x32, SolverParams(dt=dt, dh=dh))
    e32, emx = l1_rel(g32["out"], ref64["out"]), l1_rel(gmx["out"], ref64["out"])
    assert emx <= e32 * 1.1 + 1e-12, (emx, e32)
    assert scaled_err(gmx["out"], ref64["out"]) <= 1e-5


def test_plm_reads_central_window_of_wider_input(cuda_device):
    """BASELINE's 22^3 input for MHM+PLM: the solver reads the central 20^3 window."""
    x22, dt, dh = lognormal_case(npd=2, seed=21, nxt=22)
    ref = _ref("plm", "hllc", False, "fp32").solve(x22, dt, dh)
    g = gpu_solve(FluidSolver(lr="plm", rsolver="hllc", flu_nxt=22), x22, SolverParams(dt=dt, dh=dh))
    assert scaled_err(g["out"], ref["out"]) <= RTOL32


@pytest.mark.parametrize("limiter", ["vanleer", "albada", "vl_gminmod", "central"])
def test_limiters(cuda_device, limiter):
    x, dt, dh = lognormal_case(npd=2, seed=4)
    ref = _ref("plm", "hllc", False, "fp32").solve(x, dt, dh, limiter=limiter)
    g = gpu_solve(FluidSolver(), x, SolverParams(dt=dt, dh=dh, LR_Limiter=limiter))
    assert scaled_err(g["out"], ref["out"]) <= RTOL32


@pytest.mark.parametrize("lr,rs", [("plm", "hllc"), ("plm", "roe"), ("plm", "hlle"), ("ppm", "roe"), ("ppm", "hllc")])
def test_two_dimensional_flow_keeps_zero_momentum_exactly(cuda_device, lr, rs):
    """A z-independent Kelvin-Helmholtz layer with m_z = 0: the reference keeps m_z exactly zero, and
    so must every GPU variant (a contracted multiply-add could leave round-off there)."""
    from gamer_b200 import ic
    nxt = 22 if lr == "ppm" else 20
    box = ic.kelvin_helmholtz_box(2, seed=9, gamma=GAMMA)
    box = np.repeat(box[:, :, :, :1], box.shape[3], axis=3)      # [v][x][y][z]: no z dependence
    box[3] = 0.0
    dh = 1.0 / 32
    dt = ic.cfl_dt(box, GAMMA, dh, cfl=0.5)
    x = ic.cut_patch_groups(box, nxt)
    ref = _ref(lr, rs, False, "fp32").solve(x, dt, dh)
    assert not np.any(ref["out"][:, 3])
    for prec in ("fp32", "mixed", "fp64"):
        g = gpu_solve(FluidSolver(lr=lr, rsolver=rs, precision=prec, flu_nxt=nxt), x, SolverParams(dt=dt, dh=dh))
        assert not np.any(g["out"][:, 3]), prec


def test_gminmod_theta_2_takes_the_clamped_path(cuda_device):
    """Generalized MinMod with theta = 2 runs the run-time-limiter instantiation, whose PLM clamps
    can act (theta < 2 runs the built-in GMinMod instantiation without them)."""
    x, dt, dh = lognormal_case(npd=2, seed=4)
    ref = _ref("plm", "hllc", False, "fp32").solve(x, dt, dh, limiter="gminmod", minmod_coeff=2.0)
    g = gpu_solve(FluidSolver(), x, SolverParams(dt=dt, dh=dh, MinMod_Coeff=2.0))
    assert scaled_err(g["out"], ref["out"]) <= RTOL32


@pytest.mark.parametrize("lr,rs", [("plm", "hllc"), ("ppm", "roe")])
def test_blast_with_minmod_retries(cuda_device, lr, rs):
    """Mach-10 blast with a 1e3 jump: exercises the Hancock reset, the Riemann rescue and the
    MinMod-coefficient retry loop (MinMod_MaxIter = 3)."""
    nxt = 22 if lr == "ppm" else 20
    x, dt, dh = blast_case(npd=2, seed=13, nxt=nxt, dual=True)
    # FP64 where it fits one SM (PLM); PPM runs the mixed policy against the FP64 reference
    # (FP32 round-off amplified through the 1e3 shock: ~4e-4 observed)
    prec, tol = ("fp64", 1e-9) if lr == "plm" else ("mixed", 2e-3)
    ref = _ref(lr, rs, True, "fp64").solve(x, 2.0 * dt, dh, minmod_maxiter=3)
    s = FluidSolver(lr=lr, rsolver=rs, precision=prec, dual_energy=True, flu_nxt=nxt)
    g = gpu_solve(s, x, SolverParams(dt=2.0 * dt, dh=dh, MinMod_MaxIter=3), pg_fail=True)
    assert scaled_err(g["out"], ref["out"]) <= tol
    if prec == "fp64":
        assert np.array_equal(g["de"], ref["de"])
    else:
        assert np.mean(g["de"] == ref["de"]) > 0.999


def test_host_entry_point_equals_device_entry_point(cuda_device):
    x, dt, dh = lognormal_case(npd=4, seed=8)
    s = FluidSolver()
    prm = SolverParams(dt=dt, dh=dh)
    g = gpu_solve(s, x, prm)
    out, flux, _ = s.solve_host(x, prm)
    assert np.array_equal(out, g["out"]) and np.array_equal(flux, g["flux"])


def test_levels_entry_point_equals_per_level_calls(cuda_device):
    import torch
    parts = [lognormal_case(npd=2, seed=30 + l) for l in range(3)]
    xs = [p[0][: n] for p, n in zip(parts, (8, 3, 5))]
    dts = [p[1] / 2 ** l for l, p in enumerate(parts)]
    dhs = [p[2] / 2 ** l for l, p in enumerate(parts)]
    s = FluidSolver()
    per = [gpu_solve(s, x, SolverParams(dt=dt, dh=dh))["out"] for x, dt, dh in zip(xs, dts, dhs)]
    allx = np.concatenate(xs)
    t_in = torch.from_numpy(allx.astype(np.float32)).cuda()
    t_out = torch.zeros((allx.shape[0], 5, 16, 16, 16), device="cuda")
    t_flux = torch.zeros((allx.shape[0], 9, 5, 16, 16), device="cuda")
    s.solve_levels_device(t_in, t_out, [len(x) for x in xs], dts, dhs, SolverParams(dt=0.0, dh=1.0), flux=t_flux)
    torch.cuda.synchronize()
    assert np.array_equal(t_out.cpu().numpy(), np.concatenate(per))


def test_uniform_state_is_fixed_point_and_npg_edge_cases(cuda_device):
    import torch
    s = FluidSolver()
    x = np.zeros((3, 5, 20, 20, 20), np.float32)
    x[:, 0], x[:, 1], x[:, 4] = 1.3, 0.4, 2.0
    g = gpu_solve(s, x, SolverParams(dt=1e-3, dh=0.01))
    assert np.array_equal(g["out"], x[:, :, 2:18, 2:18, 2:18])
    assert np.allclose(g["flux"][:, 0, 0], 0.4)
    # zero patch groups: a no-op
    e = torch.zeros((0, 5, 20, 20, 20), device="cuda")
    s.solve_device(e, torch.zeros((0, 5, 16, 16, 16), device="cuda"), SolverParams(dt=1e-3, dh=0.01))
    torch.cuda.synchronize()
    assert s.status() == 0


def test_conservation_periodic_box(cuda_device):
    """Fluxes on faces shared by neighbouring patch groups are computed from identical data, so the
    totals over a periodic box are conserved to round-off (the reference's Aux_Check_Conservation)."""
    x, dt, dh = lognormal_case(npd=4, seed=17)
    s = FluidSolver(precision="fp64")
    g = gpu_solve(s, x.astype(np.float64), SolverParams(dt=dt, dh=dh, StoreFlux=False), want_flux=False)
    before = x[:, :, 2:18, 2:18, 2:18].astype(np.float64).sum(axis=(0, 2, 3, 4))
    after = g["out"].sum(axis=(0, 2, 3, 4))
    for v in (0, 4):
        assert abs(after[v] - before[v]) <= 1e-12 * abs(before[v])
    for v in (1, 2, 3):
        assert abs(after[v] - before[v]) <= 1e-12 * np.abs(x[:, v]).sum()


def test_invalid_arguments_are_rejected_not_crashed(cuda_device):
    import torch
    from gamer_b200.fluid import FluidSolverError
    with pytest.raises(FluidSolverError):
        FluidSolver(lr="plm", flu_nxt=18)
    s = FluidSolver()
    x = torch.zeros((2, 5, 20, 20, 20), device="cuda")
    y = torch.zeros((2, 5, 16, 16, 16), device="cuda")
    with pytest.raises(FluidSolverError):
        s.solve_device(x, y, SolverParams(dt=1e-3, dh=-1.0))
    with pytest.raises(FluidSolverError):   # StoreFlux without a flux array
        s.solve_device(x, y, SolverParams(dt=1e-3, dh=0.1, StoreFlux=True), flux=None)
    xm = torch.zeros(2 * 5 * 8000 + 1, device="cuda")[1:].view(2, 5, 20, 20, 20)   # misaligned
    with pytest.raises(FluidSolverError):
        s.solve_device(xm, y, SolverParams(dt=1e-3, dh=0.1, StoreFlux=False))
    # the kernel gives each of the 16x16 interior columns its own thread: fewer than 256 threads,
    # or a shape that is not a whole number of warps, is refused
    for bad in (128, 224, 300, 544):
        with pytest.raises(FluidSolverError):
            s.set_block_size(bad)
    s.set_block_size(256)
    assert s.block_size() == 256


@pytest.mark.parametrize("lr,rs,precision,dual", [("plm", "hllc", "mixed", False), ("plm", "hllc", "fp32", True),
                                                  ("ppm", "roe", "mixed", False), ("plm", "roe", "fp64", False)])
def test_launch_shapes_give_identical_results(cuda_device, lr, rs, precision, dual):
    """Every allowed launch shape (the autotuner may pick any) computes every cell with the same
    arithmetic: bit-identical outputs, fluxes and dual-energy status."""
    nxt = 22 if lr == "ppm" else 20
    x, dt, dh = kh_case(npd=2, seed=17, nxt=nxt, dual=dual)
    prm = SolverParams(dt=dt, dh=dh)
    ref = None
    for block in (0, 256, 288, 352, 416, 512):
        s = FluidSolver(lr=lr, rsolver=rs, precision=precision, dual_energy=dual, flu_nxt=nxt)
        if block:
            s.set_block_size(block)
        g = gpu_solve(s, x, prm)
        if ref is None:
            ref = g
            continue
        for k in ("out", "flux") + (("de",) if dual else ()):
            assert np.array_equal(g[k], ref[k]), (block, k)


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_register_variants_and_cta_caps_give_identical_results(cuda_device, precision):
    """The autotuner's other launches of the headline kernel -- the register-capped instantiations
    (64, 72, 80, 128 per thread) at the thread counts they are meant for, and one CTA per SM -- run
    the same arithmetic: bit-identical outputs and fluxes."""
    x, dt, dh = kh_case(npd=2, seed=19, nxt=20)
    prm = SolverParams(dt=dt, dh=dh)
    s = FluidSolver(precision=precision)
    assert s.launch() == (320, 0, 0)
    ref = gpu_solve(s, x, prm)
    for launch in ((512, 0, 64), (448, 0, 72), (384, 0, 80), (256, 0, 128), (320, 1, 0), (384, 1, 80)):
        s.set_launch(*launch)
        assert s.launch() == launch
        g = gpu_solve(s, x, prm)
        for k in ("out", "flux"):
            assert np.array_equal(g[k], ref[k]), (launch, k)
    # other configurations keep their default instantiation under a register cap
    sp = FluidSolver(lr="ppm", rsolver="roe", precision=precision, flu_nxt=22)
    xp, dtp, dhp = kh_case(npd=2, seed=19, nxt=22)
    want = gpu_solve(sp, xp, SolverParams(dt=dtp, dh=dhp))
    sp.set_launch(0, 0, 80)
    assert np.array_equal(gpu_solve(sp, xp, SolverParams(dt=dtp, dh=dhp))["out"], want["out"])
    for bad in ((300, 0, 0), (320, -1, 0), (320, 9, 0), (320, 0, 96), (320, 0, 100)):
        with pytest.raises(FluidSolverError) as ei:
            s.set_launch(*bad)
        assert ei.value.code == -1


@pytest.mark.parametrize("lr,precision", [("plm", "mixed"), ("ppm", "fp32"), ("plm", "fp64")])
def test_many_patch_groups_per_cta_equal_small_batches(cuda_device, lr, precision):
    """2048 patch groups in one launch (every CTA of the persistent grid sweeps about seven patch
    groups, re-using its plane ring and mbarriers) give bit for bit the outputs and fluxes of 32
    launches of 64 patch groups (one patch group per CTA)."""
    nxt = 22 if lr == "ppm" else 20
    x, dt, dh = kh_case(npd=2, seed=23, nxt=nxt)
    x = np.concatenate([x] * 256)                                   # 2048 patch groups
    # distinct groups: every conserved variable scaled by one factor (same velocities and sound speed)
    x = x * ( 1.0 + 1e-3 * ( np.arange(x.shape[0]) % 7 ) ).reshape(-1, 1, 1, 1, 1)
    rs = "roe" if lr == "ppm" else "hllc"
    prm = SolverParams(dt=dt, dh=dh)
    s = FluidSolver(lr=lr, rsolver=rs, precision=precision, flu_nxt=nxt)
    big = gpu_solve(s, x, prm)
    for p0 in range(0, x.shape[0], 64):
        small = gpu_solve(s, x[p0:p0 + 64], prm)
        assert np.array_equal(small["out"], big["out"][p0:p0 + 64]), p0
        assert np.array_equal(small["flux"], big["flux"][p0:p0 + 64]), p0
    assert s.status() == 0


def test_captured_levels_graph_replays_the_direct_launch(cuda_device):
    """A multi-level launch captured in a CUDA graph equals the direct launch, including after the
    per-level time steps are replaced in the captured graph."""
    import torch
    x, dt, dh = blast_case(npd=2, seed=41, nxt=20, dual=True)
    npg = [3, 2, 3]
    dts, dhs = [dt, dt / 2, dt / 4], [dh, dh / 2, dh / 4]
    s = FluidSolver(dual_energy=True, precision="mixed")
    t_in = torch.from_numpy(x.astype(np.float32)).cuda()
    outs = []
    for _ in range(3):
        outs.append((torch.zeros((8, 6, 16, 16, 16), device="cuda"), torch.zeros((8, 9, 6, 16, 16), device="cuda"),
                     torch.zeros((8, 16, 16, 16), dtype=torch.int8, device="cuda")))
    prm = SolverParams(dt=0.0, dh=1.0)
    s.solve_levels_device(t_in, outs[0][0], npg, dts, dhs, prm, flux=outs[0][1], de_out=outs[0][2])
    g = s.capture_levels(t_in, outs[1][0], npg, dts, dhs, prm, flux=outs[1][1], de_out=outs[1][2])
    g.launch()
    torch.cuda.synchronize()
    assert all(torch.equal(a, b) for a, b in zip(outs[0], outs[1]))
    dts2 = [d * 0.5 for d in dts]
    g.set_dt(dts2)
    outs[1][2].zero_()          # DE status chars are written only where the dual-energy fix applies
    g.launch()
    s.solve_levels_device(t_in, outs[2][0], npg, dts2, dhs, prm, flux=outs[2][1], de_out=outs[2][2])
    torch.cuda.synchronize()
    assert all(torch.equal(a, b) for a, b in zip(outs[1], outs[2]))
    assert not torch.equal(outs[0][0], outs[2][0])
    g.close()
