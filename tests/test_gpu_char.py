"""GPU parity of MHM+PLM and MHM+PPM with CHAR_RECONSTRUCTION against the reference built with that option.

The reference (oracle/_ref, variants ``mhm_plm_*_char``) projects the left, right and centred slopes
of each cell onto the hydro characteristic variables (Hydro_Pri2Char), limits them there, and
projects back (Hydro_Char2Pri) before the PLM face values and their neighbour clamp
(src/Model_Hydro/CPU_Hydro/CPU_Shared_DataReconstruction.cpp:403-430, :1957-2035).
"""
import numpy as np
import pytest

import pyoracle as po
from gamer_b200.fluid import FluidSolver, SolverParams
from parity import (RTOL32, RTOL64, blast_case, gpu_solve, kh_case, l1_rel, lognormal_case,
                    reference_spread, scaled_err)

pytestmark = pytest.mark.gpu

LIMITERS = ["gminmod", "vanleer", "albada", "vl_gminmod", "central"]


def _ref(rs, prec):
    return po.RefSolver(po.ref_variant_name("mhm", "plm", rs, char=True), prec)


@pytest.mark.parametrize("rs", ["hllc", "roe", "hlle"])
@pytest.mark.parametrize("limiter", LIMITERS)
def test_fp32_matches_reference_fp32(cuda_device, rs, limiter):
    if not po.ref_available(po.ref_variant_name("mhm", "plm", rs, char=True)):
        pytest.skip(f"reference variant mhm_plm_{rs}_char not built")
    x, dt, dh = lognormal_case(npd=2, seed=31)
    ref = _ref(rs, "fp32").solve(x, dt, dh, limiter=limiter, minmod_coeff=1.5)
    s = FluidSolver(rsolver=rs, precision="fp32", char_reconstruction=True)
    g = gpu_solve(s, x, SolverParams(dt=dt, dh=dh, LR_Limiter=limiter))
    assert scaled_err(g["out"], ref["out"]) <= RTOL32
    assert scaled_err(g["flux"], ref["flux"], axis_var=2) <= RTOL32
    assert s.status() == 0


@pytest.mark.parametrize("rs", ["hllc", "roe"])
@pytest.mark.parametrize("limiter", ["gminmod", "vl_gminmod"])
def test_fp64_matches_reference_fp64(cuda_device, rs, limiter):
    x, dt, dh = lognormal_case(npd=2, seed=32)
    ref = _ref(rs, "fp64").solve(x, dt, dh, limiter=limiter)
    g = gpu_solve(FluidSolver(rsolver=rs, precision="fp64", char_reconstruction=True), x,
                  SolverParams(dt=dt, dh=dh, LR_Limiter=limiter))
    assert scaled_err(g["out"], ref["out"]) <= RTOL64
    assert scaled_err(g["flux"], ref["flux"], axis_var=2) <= RTOL64


def test_mixed_against_fp64_reference(cuda_device):
    """Mixed precision with characteristic limiting, against the FP64 reference on the same
    float-rounded input: no less accurate than the FP32 path."""
    x, dt, dh = kh_case(npd=2, seed=33, nxt=20)
    x32 = x.astype(np.float32)
    ref64 = _ref("hllc", "fp64").solve(x32.astype(np.float64), dt, dh)
    g32 = gpu_solve(FluidSolver(precision="fp32", char_reconstruction=True), x32, SolverParams(dt=dt, dh=dh))
    gmx = gpu_solve(FluidSolver(precision="mixed", char_reconstruction=True), x32, SolverParams(dt=dt, dh=dh))
    e32, emx = l1_rel(g32["out"], ref64["out"]), l1_rel(gmx["out"], ref64["out"])
    assert emx <= e32 * 1.1 + 1e-12, (emx, e32)
    assert scaled_err(gmx["out"], ref64["out"]) <= 1e-5


def test_blast_with_minmod_retries_fp64(cuda_device):
    """The Mach-10 blast with MinMod retries: the retries lower the MinMod coefficient, which the
    characteristic limiter then applies to the projected slopes."""
    x, dt, dh = blast_case(npd=2, seed=34, nxt=20, dual=False)
    prm = SolverParams(dt=2.0 * dt, dh=dh, MinMod_MaxIter=3)
    ref = _ref("hllc", "fp64").solve(x, 2.0 * dt, dh, minmod_maxiter=3)
    g = gpu_solve(FluidSolver(precision="fp64", char_reconstruction=True), x, prm, pg_fail=True)
    assert scaled_err(g["out"], ref["out"]) <= 1e-8


def test_option_changes_the_result(cuda_device):
    """Characteristic and primitive limiting give different updates on a non-trivial flow, and each
    GPU path follows its own reference build."""
    x, dt, dh = lognormal_case(npd=1, seed=35)
    p = SolverParams(dt=dt, dh=dh)
    gc = gpu_solve(FluidSolver(precision="fp64", char_reconstruction=True), x, p)
    gp = gpu_solve(FluidSolver(precision="fp64"), x, p)
    rp = po.RefSolver(po.ref_variant_name("mhm", "plm", "hllc"), "fp64").solve(x, dt, dh)
    assert scaled_err(gp["out"], rp["out"]) <= RTOL64
    assert scaled_err(gc["out"], gp["out"]) > 1e-6


# ---- PPM with CHAR_RECONSTRUCTION: the slopes of the PPM slope pass limited in each cell's
# characteristic variables (CPU_Shared_DataReconstruction.cpp:884-907 through Hydro_LimitSlope) ----

@pytest.mark.parametrize("rs", ["hllc", "roe"])
@pytest.mark.parametrize("prec,tol", [("fp32", RTOL32), ("mixed", RTOL32), ("fp64", RTOL64)])
@pytest.mark.parametrize("limiter", ["gminmod", "vl_gminmod", "albada"])
def test_ppm_char_matches_reference(cuda_device, rs, prec, tol, limiter):
    variant = po.ref_variant_name("mhm", "ppm", rs, char=True)
    rprec = "fp64" if prec == "fp64" else "fp32"
    if not po.ref_available(variant, rprec):
        pytest.skip(f"reference variant {variant} not built")
    x, dt, dh = lognormal_case(npd=2, seed=41, nxt=22)
    ref = po.RefSolver(variant, rprec).solve(x, dt, dh, limiter=limiter)
    s = FluidSolver(lr="ppm", rsolver=rs, precision=prec, char_reconstruction=True, flu_nxt=22)
    # the same window inside a 24^3 input (FLU_NXT + 2): the kernel reads its central 22^3
    x24, _, _ = lognormal_case(npd=2, seed=41, nxt=24)
    g24 = gpu_solve(FluidSolver(lr="ppm", rsolver=rs, precision=prec, char_reconstruction=True, flu_nxt=24), x24,
                    SolverParams(dt=dt, dh=dh, LR_Limiter=limiter))
    assert scaled_err(g24["out"], ref["out"]) <= tol
    g = gpu_solve(s, x, SolverParams(dt=dt, dh=dh, LR_Limiter=limiter))
    assert scaled_err(g["out"], ref["out"]) <= tol
    assert scaled_err(g["flux"], ref["flux"], axis_var=2) <= tol
    # characteristic limiting changes the result: the primitive-limited build differs
    plain = po.RefSolver(f"mhm_ppm_{rs}", rprec).solve(x, dt, dh, limiter=limiter)
    assert scaled_err(plain["out"], ref["out"]) > 10 * tol


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_ppm_char_dual_energy_blast(cuda_device, prec):
    """PPM, CHAR_RECONSTRUCTION and dual energy on the Mach-10 blast."""
    variant = po.ref_variant_name("mhm", "ppm", "hllc", dual=True, char=True)
    if not po.ref_available(variant, prec):
        pytest.skip(f"reference variant {variant} not built")
    x, dt, dh = blast_case(npd=2, seed=43, nxt=22, dual=True)
    ref = po.RefSolver(variant, prec).solve(x, dt, dh)
    s = FluidSolver(lr="ppm", rsolver="hllc", precision=prec, char_reconstruction=True, dual_energy=True, flu_nxt=22)
    g = gpu_solve(s, x, SolverParams(dt=dt, dh=dh))
    # the characteristic PPM limiter at the 1e3 pressure jump turns last-bit differences (FMA
    # contraction) into limiter branch flips: the reference itself moves by 7e-8 (FP64) and 1.3e-2
    # (FP32) in scaled_err when its input is perturbed by one part in 1e15 / 1e7, so the bound is
    # twice that measured spread, and the bulk must agree to round-off (L1)
    spread = reference_spread(po.RefSolver(variant, prec), x, dt, dh, 1e-15 if prec == "fp64" else 1e-7)
    assert scaled_err(g["out"], ref["out"]) <= max(1e-8 if prec == "fp64" else 2e-3, 2 * spread)
    assert l1_rel(g["out"], ref["out"]) <= (1e-9 if prec == "fp64" else 3e-5)
    assert int(np.sum(g["de"] != ref["de"])) <= (0 if prec == "fp64" else 4)


def test_ppm_char_configurations_not_built(cuda_device):
    from gamer_b200.fluid import FluidSolverError
    for kw in ({"rsolver": "exact", "flu_nxt": 24}, {"npassive_user": 2, "flu_nxt": 24},
               {"rsolver": "exact", "npassive_user": 2}):
        with pytest.raises(FluidSolverError) as ei:
            FluidSolver(**dict(dict(lr="ppm", rsolver="hllc", char_reconstruction=True), **kw))
        assert ei.value.code == -5
