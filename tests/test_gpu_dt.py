"""CFL time-step solver on the GPU against the reference's own CPU_dtSolver_HydroCFL (oracle/_ref),
on GAMER's dt arrays and straight from the fluid solver's output arrays."""
import numpy as np
import pytest

import pyoracle as po
from gamer_b200 import ic
from gamer_b200.fluid import FluidSolver, SolverParams
from parity import GAMMA, gpu_solve, gpu_solve_mhd, lognormal_case, mhd_case

pytestmark = pytest.mark.gpu

TOL = {"fp32": 2e-6, "mixed": 2e-6, "fp64": 1e-13}


def _dt_case(precision, dual=False):
    """One solver step of a lognormal box, then the dt of its 8 patches per patch group."""
    x, dt, dh = lognormal_case(npd=2, seed=5, dual=dual)
    s = FluidSolver(precision=precision, dual_energy=dual, gamma=GAMMA)
    g = gpu_solve(s, x, SolverParams(dt=dt, dh=dh, StoreFlux=False))
    return s, g["out"], dh


@pytest.mark.parametrize("precision", ["fp32", "mixed", "fp64"])
def test_dt_hydro_matches_reference(cuda_device, precision):
    import torch
    s, out, dh = _dt_case(precision)
    flu, _ = ic.patches_from_output(out)
    ref = po.RefSolver("mhm_plm_hllc", "fp64" if precision == "fp64" else "fp32").dt(flu, dh, safety=0.5)
    got = s.dt_cfl(torch.from_numpy(flu).cuda(), dh, safety=0.5).cpu().numpy()
    assert np.max(np.abs(got - ref) / ref) <= TOL[precision]
    # the same from the solver's output arrays, patches in LocalID order: identical
    got2 = s.dt_cfl(torch.from_numpy(out).cuda(), dh, safety=0.5, from_output=True).cpu().numpy()
    assert np.array_equal(got, got2)


def test_dt_from_output_with_dual_energy(cuda_device):
    import torch
    s, out, dh = _dt_case("fp32", dual=True)
    flu, _ = ic.patches_from_output(out)
    s5 = FluidSolver(precision="fp32", gamma=GAMMA)
    want = s5.dt_cfl(torch.from_numpy(flu).cuda(), dh).cpu().numpy()
    got = s.dt_cfl(torch.from_numpy(out).cuda(), dh, from_output=True).cpu().numpy()
    assert np.array_equal(got, want)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_dt_mhd_matches_reference(cuda_device, precision):
    import torch
    x, b, dt, dh = mhd_case(npd=2, seed=6)
    s = FluidSolver(scheme="ctu", lr="plm", rsolver="hlld", precision=precision, gamma=GAMMA)
    g = gpu_solve_mhd(s, x, b, SolverParams(dt=dt, dh=dh, StoreFlux=False))
    flu, mag = ic.patches_from_output(g["out"], g["mag_out"])
    ref = po.RefSolver("ctu_plm_hlld_mhd", precision).dt(flu, dh, mag=mag, safety=0.4)
    got = s.dt_cfl(torch.from_numpy(flu).cuda(), dh, mag=torch.from_numpy(mag).cuda(), safety=0.4).cpu().numpy()
    assert np.max(np.abs(got - ref) / ref) <= TOL[precision]
    got2 = s.dt_cfl(torch.from_numpy(g["out"]).cuda(), dh, mag=torch.from_numpy(g["mag_out"]).cuda(), safety=0.4,
                    from_output=True).cpu().numpy()
    assert np.array_equal(got, got2)
