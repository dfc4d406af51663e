"""GPU parity of MHM with the exact Riemann solver (RSOLVER = EXACT) against the reference built
with it (oracle/_ref variants mhm_{plm,ppm}_exact[_de];
src/Model_Hydro/CPU_Hydro/CPU_Shared_RiemannSolver_Exact.cpp).

The star pressure comes from a bisection that stops once |f(p*)| < MAX_ERROR (1e-6 in FP32, 1e-14
in FP64, include/Macro.h:1023-1031), so where the two sides round f differently near the root
their p* can differ by the last bracket: the FP32 bound below allows for that.
"""
import numpy as np
import pytest

import pyoracle as po
from gamer_b200.fluid import FluidSolver, FluidSolverError, SolverParams
from parity import RTOL64, blast_case, gpu_solve, kh_case, l1_rel, lognormal_case, scaled_err

pytestmark = pytest.mark.gpu

TOL32 = 3e-5


@pytest.mark.parametrize("lr", ["plm", "ppm"])
@pytest.mark.parametrize("dual", [False, True])
def test_fp32_matches_reference_fp32(cuda_device, lr, dual):
    nxt = 22 if lr == "ppm" else 20
    x, dt, dh = lognormal_case(npd=2, seed=42, nxt=nxt, dual=dual)
    ref = po.RefSolver(po.ref_variant_name("mhm", lr, "exact", dual=dual), "fp32").solve(x, dt, dh)
    s = FluidSolver(lr=lr, rsolver="exact", precision="fp32", dual_energy=dual, flu_nxt=nxt)
    g = gpu_solve(s, x, SolverParams(dt=dt, dh=dh))
    assert scaled_err(g["out"], ref["out"]) <= TOL32
    assert scaled_err(g["flux"], ref["flux"], axis_var=2) <= TOL32
    if dual:
        assert np.array_equal(g["de"], ref["de"])
    assert s.status() == 0


@pytest.mark.parametrize("lr", ["plm", "ppm"])
@pytest.mark.parametrize("limiter", ["gminmod", "vanleer"])
def test_fp64_matches_reference_fp64(cuda_device, lr, limiter):
    nxt = 22 if lr == "ppm" else 20
    x, dt, dh = lognormal_case(npd=2, seed=43, nxt=nxt)
    ref = po.RefSolver(f"mhm_{lr}_exact", "fp64").solve(x, dt, dh, limiter=limiter)
    g = gpu_solve(FluidSolver(lr=lr, rsolver="exact", precision="fp64", flu_nxt=nxt), x,
                  SolverParams(dt=dt, dh=dh, LR_Limiter=limiter))
    assert scaled_err(g["out"], ref["out"]) <= RTOL64
    assert scaled_err(g["flux"], ref["flux"], axis_var=2) <= RTOL64


def test_mixed_against_fp64_reference(cuda_device):
    x, dt, dh = kh_case(npd=2, seed=44, nxt=20)
    x32 = x.astype(np.float32)
    ref64 = po.RefSolver("mhm_plm_exact", "fp64").solve(x32.astype(np.float64), dt, dh)
    g32 = gpu_solve(FluidSolver(rsolver="exact", precision="fp32"), x32, SolverParams(dt=dt, dh=dh))
    gmx = gpu_solve(FluidSolver(rsolver="exact", precision="mixed"), x32, SolverParams(dt=dt, dh=dh))
    e32, emx = l1_rel(g32["out"], ref64["out"]), l1_rel(gmx["out"], ref64["out"])
    assert emx <= e32 * 1.1 + 1e-12, (emx, e32)
    assert scaled_err(gmx["out"], ref64["out"]) <= TOL32


def test_blast_with_minmod_retries_fp64(cuda_device):
    """The Mach-10 blast at twice the CFL step with MinMod retries: strong shocks and rarefactions
    through every branch of the exact solver (shock / rarefaction / sonic rarefaction)."""
    x, dt, dh = blast_case(npd=2, seed=13, nxt=20, dual=False)
    ref = po.RefSolver("mhm_plm_exact", "fp64").solve(x, 2.0 * dt, dh, minmod_maxiter=3)
    g = gpu_solve(FluidSolver(rsolver="exact", precision="fp64"), x,
                  SolverParams(dt=2.0 * dt, dh=dh, MinMod_MaxIter=3), pg_fail=True)
    assert scaled_err(g["out"], ref["out"]) <= 1e-8


@pytest.mark.parametrize("lr", ["plm", "ppm"])
@pytest.mark.parametrize("prec,tol", [("fp32", TOL32), ("fp64", RTOL64)])
@pytest.mark.parametrize("limiter", ["gminmod", "vanleer"])
def test_char_reconstruction_matches_reference(cuda_device, lr, prec, tol, limiter):
    """The exact solver behind slopes limited in characteristic variables (CHAR_RECONSTRUCTION)."""
    nxt = 22 if lr == "ppm" else 20
    variant = po.ref_variant_name("mhm", lr, "exact", char=True)
    if not po.ref_available(variant, prec):
        pytest.skip(f"reference variant {variant} not built")
    x, dt, dh = lognormal_case(npd=2, seed=45, nxt=nxt)
    ref = po.RefSolver(variant, prec).solve(x, dt, dh, limiter=limiter)
    s = FluidSolver(lr=lr, rsolver="exact", precision=prec, flu_nxt=nxt, char_reconstruction=True)
    g = gpu_solve(s, x, SolverParams(dt=dt, dh=dh, LR_Limiter=limiter))
    assert scaled_err(g["out"], ref["out"]) <= tol
    assert scaled_err(g["flux"], ref["flux"], axis_var=2) <= tol
    plain = po.RefSolver(f"mhm_{lr}_exact", prec).solve(x, dt, dh, limiter=limiter)
    assert scaled_err(plain["out"], ref["out"]) > 10 * tol
    assert s.status() == 0


def test_exact_is_not_offered_where_it_is_not_built(cuda_device):
    with pytest.raises(FluidSolverError):
        FluidSolver(scheme="mhm_rp", rsolver="exact", flu_nxt=22)
