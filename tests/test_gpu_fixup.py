"""GPU parity of the coarse-fine flux fix-up (gb_flux_fixup_device) against the reference's own
Flu_FixUp_Flux() (src/Fluid/Flu_FixUp_Flux.cpp:23), compiled from source into oracle/_ref
(oracle/ref_fixup.cpp builds the level's patch_t objects from the same arrays).

Seeded batches of physical patch states with random flux differences on a random half of the
faces: small ones (every correction applies) and large ones (many corrections would leave a
negative density or internal energy and are refused), with and without dual energy (cells of
every dual-energy status), and a mask that corrects the density only."""
import numpy as np
import pytest

import pyoracle as po
from gamer_b200.fluid import FluidSolver, FluidSolverError, SolverParams
from parity import GAMMA, RTOL32, RTOL64, scaled_err

pytestmark = pytest.mark.gpu

NP = 64
DH = 1.0 / 128


def _patches(dual, scale, seed):
    rng = np.random.default_rng(seed)
    nc = 6 if dual else 5
    u = np.zeros((NP, nc, 8, 8, 8))
    rho = 0.5 + rng.random((NP, 8, 8, 8))
    vel = 0.3 * rng.standard_normal((NP, 3, 8, 8, 8))
    pres = 0.5 + rng.random((NP, 8, 8, 8))
    u[:, 0] = rho
    u[:, 1:4] = rho[:, None] * vel
    u[:, 4] = pres / (GAMMA - 1) + 0.5 * rho * (vel ** 2).sum(axis=1)
    if dual:
        u[:, 5] = pres * rho ** (1.0 - GAMMA)
    flux = scale * DH * rng.standard_normal((NP, 6, nc, 8, 8))
    has = (rng.random((NP, 6)) < 0.5).astype(np.uint8)
    de = rng.choice(np.frombuffer(b"0123", np.int8), size=(NP, 8, 8, 8)) if dual else None
    return u, flux, has, de


def _gpu(solver, u, flux, has, de):
    import torch
    t_u = torch.from_numpy(u.astype(solver.np_dtype)).cuda()
    t_f = torch.from_numpy(flux.astype(solver.np_dtype)).cuda()
    t_h = torch.from_numpy(has).cuda()
    t_d = torch.from_numpy(de).cuda() if de is not None else None
    solver.flux_fixup_device(t_u, t_f, t_h, SolverParams(dt=0.0, dh=DH), de_status=t_d)
    torch.cuda.synchronize()
    return t_u.cpu().numpy()


@pytest.mark.parametrize("prec", ["fp32", "fp64", "mixed"])
@pytest.mark.parametrize("dual", [False, True])
@pytest.mark.parametrize("scale", [0.05, 3.0])
def test_matches_reference_flu_fixup_flux(cuda_device, prec, dual, scale):
    u, flux, has, de = _patches(dual, scale, seed=7 + int(dual) + int(10 * scale))
    rprec = "fp64" if prec == "fp64" else "fp32"
    ref = po.RefSolver(po.ref_variant_name("mhm", "plm", "hllc", dual=dual), rprec)
    r = ref.fixup_flux(u.astype(ref.dtype), flux.astype(ref.dtype), has, DH, de=de)
    s = FluidSolver(precision=prec, dual_energy=dual)
    g = _gpu(s, u.astype(ref.dtype), flux.astype(ref.dtype), has, de)
    u0 = u.astype(ref.dtype)
    chg_r, chg_g = np.any(r != u0, axis=1), np.any(g != u0, axis=1)
    assert np.array_equal(chg_r, chg_g), (chg_r.sum(), chg_g.sum())
    assert chg_r.sum() > 1000
    assert scaled_err(g, r) <= (RTOL64 if prec == "fp64" else RTOL32)


def test_density_only_mask_and_floors(cuda_device):
    """FixUpVar_Flux = density only, with floors that refuse part of the corrections."""
    import torch
    u, flux, has, _ = _patches(False, 1.0, seed=31)
    ref = po.RefSolver("mhm_plm_hllc", "fp64")
    r = ref.fixup_flux(u, flux, has, DH, tvar=1, min_dens=0.6, min_eint=0.2, min_pres=0.1)
    s = FluidSolver(precision="fp64")
    t_u = torch.from_numpy(u.copy()).cuda()
    s.flux_fixup_device(t_u, torch.from_numpy(flux).cuda(), torch.from_numpy(has).cuda(),
                        SolverParams(dt=0.0, dh=DH, MinDens=0.6, MinEint=0.2, MinPres=0.1), tvar=1)
    g = t_u.cpu().numpy()
    assert np.array_equal(np.any(r != u, axis=1), np.any(g != u, axis=1))
    assert np.array_equal(g[:, 1:], u[:, 1:]) and np.array_equal(r[:, 1:], u[:, 1:])
    assert scaled_err(g, r) <= RTOL64


def test_invalid_arguments(cuda_device):
    import torch
    u = torch.zeros((1, 6, 8, 8, 8), dtype=torch.float32, device="cuda")
    f = torch.zeros((1, 6, 6, 8, 8), dtype=torch.float32, device="cuda")
    h = torch.zeros((1, 6), dtype=torch.uint8, device="cuda")
    with pytest.raises(FluidSolverError) as ei:            # dual energy needs the status array
        FluidSolver(precision="fp32", dual_energy=True).flux_fixup_device(u, f, h, SolverParams(dt=0.0, dh=DH))
    assert ei.value.code == -1
    u5 = torch.zeros((1, 5, 8, 8, 8), dtype=torch.float32, device="cuda")
    f5 = torch.zeros((1, 6, 5, 8, 8), dtype=torch.float32, device="cuda")
    with pytest.raises(ValueError):                        # MHD needs the patches' magnetic field
        FluidSolver(scheme="ctu", rsolver="hlld", precision="fp32").flux_fixup_device(
            u5, f5, h, SolverParams(dt=0.0, dh=DH))
