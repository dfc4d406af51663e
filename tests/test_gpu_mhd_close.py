"""GPU parity of the MHD close consumers against the reference's own routines compiled under MHD into
oracle/_ref (libgref_ctu_plm_hlld_mhd_*):

* gb_fluid_correct_unphysical_mhd_device — the MHD branch of CorrectUnphysical()
  (src/Fluid/Flu_Close.cpp:542-1200): magnetic energy in every test, ResetLongB and the MHD Roe /
  HLLE / HLLD first-order fluxes.  Input: a magnetised flow advanced by the reference CTU+MHD solver
  with 1.5 (every failed cell repairable) and 2.5 (some cells beyond repair: the reference aborts)
  times the CFL step, plus planted unphysical cells on both sides of the patch-group middle planes.
* gb_flux_fixup_mhd_device — Flu_FixUp_Flux() (src/Fluid/Flu_FixUp_Flux.cpp:23) with the magnetic
  energy of each patch's face-centred field.
* gb_mhd_fixup_electric_device — MHD_FixUp_Electric() (src/Model_Hydro/MHD_FixUp_Electric.cpp:22),
  bit for bit.
"""
import numpy as np
import pytest

import pyoracle as po
from gamer_b200.fluid import ELE_PER_PATCH, FluidSolver, FluidSolverError, SolverParams
from parity import GAMMA, RTOL32, RTOL64, mhd_case, scaled_err
from test_oracle_mhd_close import electric_case, present

pytestmark = pytest.mark.gpu

VARIANT = "ctu_plm_hlld_mhd"
# FP32 bound of a corrected cell: the first-order update of a Mach-3 magnetised flow advanced with
# 1.5-2.5 times the CFL step (the same bound as the hydro blast's corrections); all but one cell in a
# thousand within the 1e-5 of the smooth cases
TOL32 = 1e-4
TOL32_MOST = 1e-5
PLANT = [(7, 3, 5), (8, 3, 5), (4, 7, 2), (4, 8, 2), (9, 10, 7), (9, 10, 8), (0, 0, 0), (15, 15, 15),
         (15, 0, 8), (7, 7, 7), (8, 8, 8)]
CASES = {"repairable": dict(cfl=1.5, mach=3.0, db=1.5),
         "harsh": dict(cfl=2.5, mach=5.0, db=2.0, b0=(2.0, 1.0, 0.5))}


def _case(prec, kind):
    ref = po.RefSolver(VARIANT, prec)
    x, b, dt, dh = mhd_case(npd=2, seed=5, **CASES[kind])
    x, b = x.astype(ref.dtype), b.astype(ref.dtype)
    r = ref.solve(x, dt, dh, mag_in=b)
    out = r["out"].copy()
    for p in range(out.shape[0]):
        for (i, j, k) in PLANT:
            out[p, 0, k, j, i] = -abs(out[p, 0, k, j, i])
    return ref, x, b, out, r["mag_out"], r["flux"], dt, dh


def _gpu_close(solver, x, b, out, bout, flux, prm, **opt):
    import torch
    dev = "cuda:0"
    t = [torch.from_numpy(np.ascontiguousarray(a).copy()).to(dev) for a in (x, b, out, bout, flux)]
    counts = solver.correct_unphysical_device(t[0], t[2], prm, flux=t[4], mag_in=t[1], mag_out=t[3], **opt)
    torch.cuda.synchronize()
    return t[2].cpu().numpy(), t[4].cpu().numpy(), t[3].cpu().numpy(), counts.cpu().numpy()


def _cell_err(g, r, mask):
    g, r = np.asarray(g, np.float64), np.asarray(r, np.float64)
    rms = np.sqrt(np.mean(r * r, axis=(0, 2, 3, 4), keepdims=True))
    e = np.max(np.abs(g - r) / (np.abs(r) + rms), axis=1)
    return e[mask]


@pytest.mark.parametrize("kind", ["repairable", "harsh"])
@pytest.mark.parametrize("scheme", ["roe", "hlle", "hlld"])
@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
def test_matches_reference_mhd_correct_unphysical(cuda_device, tmp_path, prec, scheme, kind):
    rprec = "fp64" if prec == "fp64" else "fp32"
    ref, x, b, out, bout, flux, dt, dh = _case(rprec, kind)
    r = ref.correct_unphysical_mhd(x, b, out, bout, dt, dh, flux=flux, scheme=scheme, outdir=str(tmp_path))
    s = FluidSolver(scheme="ctu", rsolver="hlld", precision=prec, flu_nxt=22)
    g_out, g_flux, g_bout, counts = _gpu_close(s, x, b, out, bout, flux, SolverParams(dt=dt, dh=dh),
                                               OPT__1ST_FLUX_CORR="3d", OPT__1ST_FLUX_CORR_SCHEME=scheme)
    tol = TOL32 if rprec == "fp32" else RTOL64
    # B is read only; the same cells are replaced and the others stay bit for bit
    assert np.array_equal(g_bout, bout)
    chg_r = np.any(r["out"] != out, axis=1)
    chg_g = np.any(g_out != out, axis=1)
    assert np.array_equal(chg_r, chg_g), (chg_r.sum(), chg_g.sum())
    assert chg_r.sum() > 8 * len(PLANT)
    err = _cell_err(g_out, r["out"], chg_r)
    assert err.max() <= tol
    if rprec == "fp32":
        assert np.mean(err <= TOL32_MOST) >= 0.999
    assert scaled_err(g_flux, r["flux"], axis_var=2) <= tol
    # the reference aborts exactly when some cell fails
    assert (r["rc"] != 0) == (counts[1] > 0), (r["rc"], counts)
    if kind == "repairable":
        assert r["rc"] == 0 and counts[0] == r["ncorr"]
    assert counts[0] == chg_g.sum()


@pytest.mark.parametrize("cont,floor", [(True, True), (False, False)])
def test_mhd_floor_and_auto_reduce_dt_modes(cuda_device, tmp_path, cont, floor):
    ref, x, b, out, bout, flux, dt, dh = _case("fp64", "harsh")
    r = ref.correct_unphysical_mhd(x, b, out, bout, dt, dh, flux=flux, scheme="hlld", last_resort_floor=floor,
                                   auto_reduce_dt_continue=cont, min_dens=1e-6, min_eint=1e-8, outdir=str(tmp_path))
    s = FluidSolver(scheme="ctu", rsolver="hlld", precision="fp64", flu_nxt=22)
    g_out, g_flux, _, counts = _gpu_close(s, x, b, out, bout, flux, SolverParams(dt=dt, dh=dh, MinDens=1e-6, MinEint=1e-8),
                                          OPT__1ST_FLUX_CORR="3d", OPT__1ST_FLUX_CORR_SCHEME="hlld",
                                          OPT__LAST_RESORT_FLOOR=floor, AutoReduceDt_Continue=cont)
    chg = np.any(r["out"] != out, axis=1)
    assert np.array_equal(chg, np.any(g_out != out, axis=1))
    assert _cell_err(g_out, r["out"], chg).max() <= RTOL64
    assert scaled_err(g_flux, r["flux"], axis_var=2) <= RTOL64
    assert (r["rc"] != 0) == (counts[1] > 0)


def test_mhd_without_first_order_correction_only_floors(cuda_device, tmp_path):
    ref, x, b, out, bout, flux, dt, dh = _case("fp64", "repairable")
    r = ref.correct_unphysical_mhd(x, b, out, bout, dt, dh, flux=flux, corr="none", min_dens=1e-3, min_eint=1e-6,
                                   outdir=str(tmp_path))
    s = FluidSolver(scheme="ctu", rsolver="hlld", precision="fp64", flu_nxt=22)
    g_out, g_flux, _, counts = _gpu_close(s, x, b, out, bout, flux, SolverParams(dt=dt, dh=dh, MinDens=1e-3, MinEint=1e-6),
                                          OPT__1ST_FLUX_CORR="none")
    assert np.array_equal(g_flux, flux)
    chg = np.any(r["out"] != out, axis=1)
    assert np.array_equal(chg, np.any(g_out != out, axis=1))
    assert _cell_err(g_out, r["out"], chg).max() <= RTOL64
    assert (r["rc"] != 0) == (counts[1] > 0)


def test_mhd_close_arguments(cuda_device):
    import torch
    s = FluidSolver(scheme="ctu", rsolver="hlld", precision="fp32", flu_nxt=22)
    t = torch.zeros((1, 5, 22, 22, 22), device="cuda")
    o = torch.zeros((1, 5, 16, 16, 16), device="cuda")
    bi = torch.zeros((1, 3, 23 * 22 * 22), device="cuda")
    bo = torch.zeros((1, 3, 17 * 16 * 16), device="cuda")
    prm = SolverParams(dt=1e-3, dh=1e-2)
    with pytest.raises(ValueError):                       # the MHD branch needs the field
        s.correct_unphysical_device(t, o, prm)
    with pytest.raises(FluidSolverError) as ei:           # 3D1D does not exist for MHD
        s.correct_unphysical_device(t, o, prm, mag_in=bi, mag_out=bo, OPT__1ST_FLUX_CORR="3d1d")
    assert ei.value.code == -5
    with pytest.raises(FluidSolverError) as ei:           # HLLC is not an MHD solver
        s.correct_unphysical_device(t, o, prm, mag_in=bi, mag_out=bo, OPT__1ST_FLUX_CORR_SCHEME="hllc")
    assert ei.value.code == -1


# ---- Flu_FixUp_Flux with MHD ----------------------------------------------------------------------

NP = 64
DH = 1.0 / 128


def _mhd_patches(scale, seed):
    rng = np.random.default_rng(seed)
    u = np.zeros((NP, 5, 8, 8, 8))
    rho = 0.5 + rng.random((NP, 8, 8, 8))
    vel = 0.3 * rng.standard_normal((NP, 3, 8, 8, 8))
    pres = 0.5 + rng.random((NP, 8, 8, 8))
    mag = 0.8 * rng.standard_normal((NP, 3, 9 * 8 * 8))
    bx = mag[:, 0].reshape(NP, 8, 8, 9)
    by = mag[:, 1].reshape(NP, 8, 9, 8)
    bz = mag[:, 2].reshape(NP, 9, 8, 8)
    emag = 0.5 * ((0.5 * (bx[..., :-1] + bx[..., 1:])) ** 2 + (0.5 * (by[:, :, :-1] + by[:, :, 1:])) ** 2 +
                  (0.5 * (bz[:, :-1] + bz[:, 1:])) ** 2)
    u[:, 0] = rho
    u[:, 1:4] = rho[:, None] * vel
    u[:, 4] = pres / (GAMMA - 1) + 0.5 * rho * (vel ** 2).sum(axis=1) + emag
    flux = scale * DH * rng.standard_normal((NP, 6, 5, 8, 8))
    has = (rng.random((NP, 6)) < 0.5).astype(np.uint8)
    return u, mag, flux, has


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
@pytest.mark.parametrize("scale", [0.05, 3.0])
def test_matches_reference_mhd_flu_fixup_flux(cuda_device, prec, scale):
    import torch
    u, mag, flux, has = _mhd_patches(scale, seed=17 + int(10 * scale))
    rprec = "fp64" if prec == "fp64" else "fp32"
    ref = po.RefSolver(VARIANT, rprec)
    u, mag, flux = u.astype(ref.dtype), mag.astype(ref.dtype), flux.astype(ref.dtype)
    r = ref.fixup_flux_mhd(u, mag, flux, has, DH)
    s = FluidSolver(scheme="ctu", rsolver="hlld", precision=prec, flu_nxt=22)
    t_u = torch.from_numpy(u.copy()).cuda()
    s.flux_fixup_device(t_u, torch.from_numpy(flux).cuda(), torch.from_numpy(has).cuda(),
                        SolverParams(dt=0.0, dh=DH), magnetic=torch.from_numpy(mag).cuda())
    g = t_u.cpu().numpy()
    chg_r, chg_g = np.any(r != u, axis=1), np.any(g != u, axis=1)
    assert np.array_equal(chg_r, chg_g), (chg_r.sum(), chg_g.sum())
    assert chg_r.sum() > 1000
    assert scaled_err(g, r) <= (RTOL64 if prec == "fp64" else RTOL32)


def test_mhd_fixup_flux_needs_the_field(cuda_device):
    import torch
    u = torch.zeros((1, 5, 8, 8, 8), device="cuda")
    f = torch.zeros((1, 6, 5, 8, 8), device="cuda")
    h = torch.zeros((1, 6), dtype=torch.uint8, device="cuda")
    with pytest.raises(ValueError):
        FluidSolver(scheme="ctu", rsolver="hlld", flu_nxt=22).flux_fixup_device(u, f, h, SolverParams(dt=0.0, dh=DH))


# ---- MHD_FixUp_Electric -----------------------------------------------------------------------------

@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_fixup_electric_matches_reference_bit_for_bit(cuda_device, prec):
    import torch
    dtype = np.float64 if prec == "fp64" else np.float32
    ref = po.RefSolver(VARIANT, prec)
    mag, ele, elb, has, sib = electric_case(300, dtype, seed=11)
    r_mag, r_ele, r_elb = ref.fixup_electric(mag, ele, elb, has, sib, DH)
    s = FluidSolver(scheme="ctu", rsolver="hlld", precision=prec, flu_nxt=22)
    t = [torch.from_numpy(a.copy()).cuda() for a in (mag, ele, elb, has, sib)]
    s.fixup_electric_device(*t, DH)
    torch.cuda.synchronize()
    g_mag, g_ele, g_elb = (a.cpu().numpy() for a in t[:3])
    assert np.array_equal(g_mag, r_mag)
    assert (g_mag != mag).sum() > 100_000
    pm = present(has)
    assert np.array_equal(g_ele[pm], r_ele[pm]) and np.array_equal(g_elb[pm], r_elb[pm])
    assert not np.any(g_ele[pm]) and not np.any(g_elb[pm])
    # a patch with no side on a coarse-fine boundary is left as it was
    none = ~has.any(axis=1)
    assert none.any()
    assert np.array_equal(g_ele[none], ele[none]) and np.array_equal(g_mag[none], mag[none])


def test_fixup_electric_arguments(cuda_device):
    import torch
    s = FluidSolver(scheme="ctu", rsolver="hlld", precision="fp32", flu_nxt=22)
    mag = torch.zeros((2, 3, 576), device="cuda")
    e = torch.zeros((2, ELE_PER_PATCH), device="cuda")
    h = torch.zeros((2, 18), dtype=torch.uint8, device="cuda")
    sl = torch.zeros((2, 6), dtype=torch.uint8, device="cuda")
    with pytest.raises(ValueError):
        s.fixup_electric_device(mag, e, e.clone(), h, sl[:, :5], DH)
    with pytest.raises(FluidSolverError) as ei:
        s.fixup_electric_device(mag, e, e.clone(), h, sl, -1.0)
    assert ei.value.code == -1
    with pytest.raises(FluidSolverError) as ei:            # a hydro configuration has no B
        FluidSolver(precision="fp32").fixup_electric_device(mag, e, e.clone(), h, sl, DH)
    assert ei.value.code == -1
