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


def test_dt_is_the_same_for_every_hydro_scheme_and_mhd_scheme(cuda_device):
    """The CFL solver depends on the fluid model only: hydro CTU and MHM_RP (no magnetic arrays)
    give MHM's dt, and MHM_RP with MHD gives CTU+MHD's."""
    import torch
    s, out, dh = _dt_case("fp32")
    flu = torch.from_numpy(ic.patches_from_output(out)[0]).cuda()
    want = s.dt_cfl(flu, dh).cpu().numpy()
    for kw in (dict(scheme="ctu", rsolver="hllc"), dict(scheme="mhm_rp", rsolver="hllc")):
        got = FluidSolver(precision="fp32", gamma=GAMMA, **kw).dt_cfl(flu, dh).cpu().numpy()
        assert np.array_equal(got, want), kw
    x, b, dt, dhm = mhd_case(npd=1, seed=7)
    sm = FluidSolver(scheme="ctu", lr="plm", rsolver="hlld", precision="fp32", gamma=GAMMA)
    g = gpu_solve_mhd(sm, x, b, SolverParams(dt=dt, dh=dhm, StoreFlux=False))
    flu_m, mag_m = (torch.from_numpy(a).cuda() for a in ic.patches_from_output(g["out"], g["mag_out"]))
    want_m = sm.dt_cfl(flu_m, dhm, mag=mag_m).cpu().numpy()
    got_m = FluidSolver(scheme="mhm_rp", lr="plm", rsolver="hlld", precision="fp32", gamma=GAMMA).dt_cfl(
        flu_m, dhm, mag=mag_m).cpu().numpy()
    assert np.array_equal(got_m, want_m)
