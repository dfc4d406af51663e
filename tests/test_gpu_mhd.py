"""CTU + MHD (PLM, HLLD with the HLLE rescue, constrained transport) on the GPU against the reference's
own CPU_FluidSolver_CTU built with MHD (oracle/_ref), through the C ABI."""
import numpy as np
import pytest

import pyoracle as po
from gamer_b200 import ic
from gamer_b200.fluid import FluidSolver, FluidSolverError, SolverParams
from parity import GAMMA, RTOL32, RTOL64, gpu_solve_mhd, l1_rel, mhd_case, reference_spread, scaled_err

pytestmark = pytest.mark.gpu

VARIANT = "ctu_plm_hlld_mhd"


def _need_ref(prec):
    if not po.ref_available(VARIANT, prec):
        pytest.skip(f"oracle/_ref/libgref_{VARIANT}_{prec}.so not built")


def _bscale(b):
    # face fields judged against the rms of |B| (components cross zero)
    return float(np.sqrt(np.mean(np.asarray(b, np.float64) ** 2)))


def _rel(g, r):
    g = np.asarray(g, np.float64)
    r = np.asarray(r, np.float64)
    return float(np.max(np.abs(g - r)) / _bscale(r))


@pytest.mark.parametrize("precision,tol", [("fp32", RTOL32), ("fp64", RTOL64)])
def test_ctu_mhd_matches_reference(cuda_device, precision, tol):
    _need_ref(precision)
    x, b, dt, dh = mhd_case(npd=2, seed=1)
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True)
    s = FluidSolver(scheme="ctu", lr="plm", rsolver="hlld", precision=precision, gamma=GAMMA)
    g = gpu_solve_mhd(s, x, b, prm)
    r = po.RefSolver(VARIANT, precision).solve(x, dt, dh, mag_in=b, store_flux=True, store_ele=True)
    assert scaled_err(g["out"], r["out"]) <= tol
    assert scaled_err(g["mag_out"], r["mag_out"]) <= tol
    assert scaled_err(g["flux"], r["flux"], axis_var=2) <= tol
    assert scaled_err(g["ele"], r["ele"], axis_var=2) <= tol


MHD_CASES = {
    "no_field": dict(b0=(0.0, 0.0, 0.0), db=0.0),           # HLLD and eigen-system with B = 0
    "x_aligned": dict(b0=(1.0, 0.0, 0.0), db=0.0),          # transverse B = 0 along x, B_n = 0 along y, z
    "supersonic": dict(mach=3.0),                            # upwind HLLD branches
}


@pytest.mark.parametrize("case", sorted(MHD_CASES))
def test_ctu_mhd_field_regimes(cuda_device, case):
    _need_ref("fp32")
    x, b, dt, dh = mhd_case(npd=2, seed=7, **MHD_CASES[case])
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True)
    s = FluidSolver(scheme="ctu", lr="plm", rsolver="hlld", precision="fp32", gamma=GAMMA)
    g = gpu_solve_mhd(s, x, b, prm)
    r = po.RefSolver(VARIANT, "fp32").solve(x, dt, dh, mag_in=b, store_flux=True, store_ele=True)
    assert scaled_err(g["out"], r["out"]) <= RTOL32
    assert scaled_err(g["mag_out"], r["mag_out"]) <= RTOL32
    assert scaled_err(g["flux"], r["flux"], axis_var=2) <= RTOL32


def test_ctu_mhd_zero_field_stays_zero(cuda_device):
    """With B = 0 the magnetic output is exactly zero, as in the reference (the Alfven waves of the
    characteristic tracing cancel exactly)."""
    x, b, dt, dh = mhd_case(npd=2, seed=7, **MHD_CASES["no_field"])
    for prec in ("fp32", "mixed", "fp64"):
        s = FluidSolver(scheme="ctu", lr="plm", rsolver="hlld", precision=prec, gamma=GAMMA)
        g = gpu_solve_mhd(s, x, b, SolverParams(dt=dt, dh=dh, StoreFlux=False, StoreElectric=True))
        assert not np.any(g["mag_out"]) and not np.any(g["ele"]), prec


def test_ctu_mhd_strong_field(cuda_device):
    """beta ~ 0.01: E - K - B^2/2 cancels by two orders of magnitude, so float arithmetic is
    ill-conditioned (the FP32 reference itself differs from the FP64 one by ~4e-4).  FP64 must match
    the FP64 reference; FP32 must stay within the FP32 reference's own distance from FP64."""
    _need_ref("fp64")
    x, b, dt, dh = mhd_case(npd=2, seed=7, b0=(8.0, 6.0, 5.0), db=3.0)
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=False)
    r64 = po.RefSolver(VARIANT, "fp64").solve(x, dt, dh, mag_in=b, store_flux=False)
    r32 = po.RefSolver(VARIANT, "fp32").solve(x, dt, dh, mag_in=b, store_flux=False)
    g64 = gpu_solve_mhd(FluidSolver(scheme="ctu", lr="plm", rsolver="hlld", precision="fp64", gamma=GAMMA), x, b, prm)
    g32 = gpu_solve_mhd(FluidSolver(scheme="ctu", lr="plm", rsolver="hlld", precision="fp32", gamma=GAMMA), x, b, prm)
    assert scaled_err(g64["out"], r64["out"]) <= 1e-9
    assert scaled_err(g64["mag_out"], r64["mag_out"]) <= 1e-9
    ref_floor = scaled_err(r32["out"], r64["out"])
    assert l1_rel(g32["out"], r64["out"]) <= 2.0 * l1_rel(r32["out"], r64["out"])
    assert scaled_err(g32["out"], r32["out"]) <= max(RTOL32, 2.0 * ref_floor)


@pytest.mark.parametrize("limiter", ["vanleer", "albada", "central", "vl_gminmod"])
def test_ctu_mhd_limiters(cuda_device, limiter):
    _need_ref("fp32")
    x, b, dt, dh = mhd_case(npd=2, seed=8)
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=False, LR_Limiter=limiter)
    s = FluidSolver(scheme="ctu", lr="plm", rsolver="hlld", precision="fp32", gamma=GAMMA)
    g = gpu_solve_mhd(s, x, b, prm)
    r = po.RefSolver(VARIANT, "fp32").solve(x, dt, dh, mag_in=b, store_flux=False, limiter=limiter)
    assert scaled_err(g["out"], r["out"]) <= RTOL32
    assert scaled_err(g["mag_out"], r["mag_out"]) <= RTOL32


def test_ctu_mhd_mixed_matches_fp64_reference(cuda_device):
    _need_ref("fp64")
    x, b, dt, dh = mhd_case(npd=2, seed=2)
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=False)
    r = po.RefSolver(VARIANT, "fp64").solve(x, dt, dh, mag_in=b, store_flux=False)
    g = {}
    for prec in ("mixed", "fp32"):
        s = FluidSolver(scheme="ctu", lr="plm", rsolver="hlld", precision=prec, gamma=GAMMA)
        g[prec] = gpu_solve_mhd(s, x, b, prm)
    # float arithmetic bounds both (and a float run takes dE_Upwind's tie branch for |v_face| dt/dh
    # up to 1e-6 where FP64 uses 1e-14, flipping a few edge EMFs); FP64 energy recovery and
    # accumulation keep the mixed L1 at or below the plain FP32 one
    for k in ("out", "mag_out"):
        assert l1_rel(g["mixed"][k], r[k]) <= 1e-6
        assert l1_rel(g["mixed"][k], r[k]) <= 1.1 * l1_rel(g["fp32"][k], r[k])


@pytest.mark.parametrize("precision,tol", [("fp32", 2e-6), ("fp64", 1e-13)])
def test_ctu_mhd_divergence_free(cuda_device, precision, tol):
    """Constrained transport keeps the discrete div B of every output cell at round-off, and the
    faces two neighbouring patch groups both update agree."""
    x, b, dt, dh = mhd_case(npd=2, seed=3)
    s = FluidSolver(scheme="ctu", lr="plm", rsolver="hlld", precision=precision, gamma=GAMMA)
    g = gpu_solve_mhd(s, x, b, SolverParams(dt=dt, dh=dh, StoreFlux=False))
    scale = _bscale(g["mag_out"])
    div_g = np.abs(ic.div_b(g["mag_out"])).max()
    assert div_g <= tol * scale
    # and no larger than the reference build's own div B at the same precision (to round-off: both
    # are sums of a few products rounded to the storage type)
    _need_ref(precision)
    r = po.RefSolver(VARIANT, precision).solve(x, dt, dh, mag_in=b, store_flux=False)
    div_r = np.abs(ic.div_b(r["mag_out"])).max()
    assert div_g <= 4.0 * div_r + 4.0 * np.finfo(g["mag_out"].dtype).eps * scale
    fx, fy, fz = ic.mag_out_faces(g["mag_out"])
    # patch groups in x-fastest order on a 2x2x2 periodic box: PG p+1 is the +x neighbour of p (px = 0)
    for p in (0, 2, 4, 6):
        assert np.array_equal(fx[p][..., 16], fx[p + 1][..., 0])
    for p in (0, 1, 4, 5):
        assert np.array_equal(fy[p][:, 16, :], fy[p + 2][:, 0, :])
    for p in (0, 1, 2, 3):
        assert np.array_equal(fz[p][16], fz[p + 4][0])


def test_ctu_mhd_host_equals_device_and_chunking(cuda_device):
    x, b, dt, dh = mhd_case(npd=2, seed=4)
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True)
    s = FluidSolver(scheme="ctu", lr="plm", rsolver="hlld", precision="fp32", gamma=GAMMA)
    g = gpu_solve_mhd(s, x, b, prm)
    s.set_mhd_chunk(3)          # 8 PGs in chunks of 3, 3, 2 over the three host streams
    out, flux, _, bout, ele = s.solve_host(x, prm, mag_in=b)
    assert np.array_equal(out, g["out"])
    assert np.array_equal(bout, g["mag_out"])
    assert np.array_equal(flux, g["flux"])
    assert np.array_equal(ele, g["ele"])


def test_ctu_mhd_rejects_bad_arguments(cuda_device):
    import torch
    x, b, dt, dh = mhd_case(npd=1, seed=5)
    s = FluidSolver(scheme="ctu", lr="plm", rsolver="hlld", precision="fp32", gamma=GAMMA)
    t_in = torch.from_numpy(x.astype(np.float32)).cuda()
    t_out = torch.zeros((1, 5, 16, 16, 16), device="cuda")
    with pytest.raises(FluidSolverError) as ei:       # no magnetic arrays
        s.solve_device(t_in, t_out, SolverParams(dt=dt, dh=dh, StoreFlux=False))
    assert ei.value.code == -1
    t_b = torch.from_numpy(b.astype(np.float32)).cuda()
    t_bout = torch.zeros((1, 3, 17 * 256), device="cuda")
    with pytest.raises(FluidSolverError) as ei:       # StoreElectric without an Ele array
        s.solve_device(t_in, t_out, SolverParams(dt=dt, dh=dh, StoreFlux=False, StoreElectric=True),
                       mag_in=t_b, mag_out=t_bout)
    assert ei.value.code == -1
    for kw in ({"dual_energy": True},):
        cfg = dict(scheme="ctu", lr="plm", rsolver="hlld", precision="fp32", gamma=GAMMA)
        cfg.update(kw)
        with pytest.raises(FluidSolverError) as ei:
            FluidSolver(**cfg)
        assert ei.value.code == -5


VARIANT_CHAR = "ctu_plm_hlld_char_mhd"


@pytest.mark.parametrize("limiter", ["gminmod", "vanleer", "vl_gminmod"])
@pytest.mark.parametrize("precision,tol", [("fp32", RTOL32), ("fp64", RTOL64)])
def test_ctu_mhd_char_reconstruction_matches_reference(cuda_device, precision, tol, limiter):
    """CTU + MHD with CHAR_RECONSTRUCTION: the PLM slopes limited in the seven MHD wave amplitudes of
    each cell (its eigenvectors along the direction), the normal B carrying no slope."""
    if not po.ref_available(VARIANT_CHAR, precision):
        pytest.skip(f"oracle/_ref/libgref_{VARIANT_CHAR}_{precision}.so not built")
    x, b, dt, dh = mhd_case(npd=2, seed=1)
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True, LR_Limiter=limiter)
    s = FluidSolver(scheme="ctu", lr="plm", rsolver="hlld", precision=precision, gamma=GAMMA,
                    char_reconstruction=True)
    g = gpu_solve_mhd(s, x, b, prm)
    ref = po.RefSolver(VARIANT_CHAR, precision)
    r = ref.solve(x, dt, dh, mag_in=b, store_flux=True, store_ele=True, limiter=limiter)
    # the projections onto the MHD waves amplify rounding (1/a^2, the fast/slow normalisations): the
    # reference's own FP32 build moves by up to 1.3e-5 (cells) and 1.8e-4 (fluxes) when its input is
    # perturbed by one part in 1e7, so in FP32 the bound is twice the spread measured here
    def bound(key, axis_var=1):
        if precision == "fp64":
            return tol
        sp = reference_spread(ref, x, dt, dh, 1e-7, key=key, axis_var=axis_var, mag_in=b, store_flux=True,
                              store_ele=True, limiter=limiter)
        return max(tol, 2 * sp)
    assert scaled_err(g["out"], r["out"]) <= bound("out")
    assert scaled_err(g["mag_out"], r["mag_out"]) <= bound("mag_out")
    assert scaled_err(g["flux"], r["flux"], axis_var=2) <= bound("flux", 2)
    assert scaled_err(g["ele"], r["ele"], axis_var=2) <= bound("ele", 2)
    # the option acts
    _need_ref(precision)
    plain = po.RefSolver(VARIANT, precision).solve(x, dt, dh, mag_in=b, store_flux=False, limiter=limiter)
    assert scaled_err(g["out"], plain["out"]) > 100 * tol


@pytest.mark.parametrize("case", ["no_field", "x_aligned"])
def test_ctu_mhd_char_degenerate_fields(cuda_device, case):
    """Wave amplitudes where the eigenvectors take their degenerate forms (B = 0; B along x)."""
    if not po.ref_available(VARIANT_CHAR, "fp64"):
        pytest.skip(f"oracle/_ref/libgref_{VARIANT_CHAR}_fp64.so not built")
    x, b, dt, dh = mhd_case(npd=2, seed=9, **MHD_CASES[case])
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=False)
    s = FluidSolver(scheme="ctu", lr="plm", rsolver="hlld", precision="fp64", gamma=GAMMA, char_reconstruction=True)
    g = gpu_solve_mhd(s, x, b, prm)
    r = po.RefSolver(VARIANT_CHAR, "fp64").solve(x, dt, dh, mag_in=b, store_flux=False)
    assert scaled_err(g["out"], r["out"]) <= RTOL64
    if case == "no_field":
        assert not np.any(g["mag_out"]) and not np.any(r["mag_out"])
    else:
        assert _rel(g["mag_out"], r["mag_out"]) <= RTOL64


# ---- MHM_RP with MHD: a first-order Riemann predictor with its own constrained-transport half
# step, PLM (or characteristic limiting) on the half-step state, then the full step
# (CPU_FluidSolver_MHM.cpp:396-565), against the reference built with FLU_SCHEME=MHM_RP and MHD ----

VARIANT_RP = "mhmrp_plm_hlld_mhd"
VARIANT_RP_CHAR = "mhmrp_plm_hlld_char_mhd"


def _rp(precision, **kw):
    return FluidSolver(scheme="mhm_rp", lr="plm", rsolver="hlld", precision=precision, gamma=GAMMA, **kw)


def _need_rp(variant, precision):
    if not po.ref_available(variant, precision):
        pytest.skip(f"oracle/_ref/libgref_{variant}_{precision}.so not built")
    return po.RefSolver(variant, precision)


@pytest.mark.parametrize("precision,tol", [("fp32", RTOL32), ("fp64", RTOL64)])
def test_mhmrp_mhd_matches_reference(cuda_device, precision, tol):
    ref = _need_rp(VARIANT_RP, precision)
    x, b, dt, dh = mhd_case(npd=2, seed=2)
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True)
    s = _rp(precision)
    assert s.mhd and s.flu_nxt == 22
    g = gpu_solve_mhd(s, x, b, prm)
    r = ref.solve(x, dt, dh, mag_in=b, store_flux=True, store_ele=True)
    # FP32: the reference's own MHM_RP build moves by up to 3e-5 (fluxes, EMF planes) when its input
    # is perturbed by one part in 1e7 (the first-order predictor feeds the limiter), so the bound
    # is twice the spread measured here
    kw = dict(mag_in=b, store_flux=True, store_ele=True)
    for key, ax in (("out", 1), ("mag_out", 1), ("flux", 2), ("ele", 2)):
        bound = tol if precision == "fp64" else max(tol, 2 * reference_spread(ref, x, dt, dh, 1e-7, key=key, axis_var=ax, **kw))
        assert scaled_err(g[key], r[key], axis_var=ax) <= bound, key
    # not the CTU answer
    c = po.RefSolver(VARIANT, precision).solve(x, dt, dh, mag_in=b, store_flux=False)
    assert scaled_err(g["out"], c["out"]) > 100 * tol


@pytest.mark.parametrize("limiter", ["vanleer", "albada", "central", "vl_gminmod"])
def test_mhmrp_mhd_limiters(cuda_device, limiter):
    ref = _need_rp(VARIANT_RP, "fp64")
    x, b, dt, dh = mhd_case(npd=2, seed=10)
    g = gpu_solve_mhd(_rp("fp64"), x, b, SolverParams(dt=dt, dh=dh, StoreFlux=False, LR_Limiter=limiter))
    r = ref.solve(x, dt, dh, mag_in=b, store_flux=False, limiter=limiter)
    assert scaled_err(g["out"], r["out"]) <= RTOL64
    assert scaled_err(g["mag_out"], r["mag_out"]) <= RTOL64


@pytest.mark.parametrize("case", sorted(MHD_CASES))
def test_mhmrp_mhd_field_regimes(cuda_device, case):
    ref = _need_rp(VARIANT_RP, "fp64")
    x, b, dt, dh = mhd_case(npd=2, seed=11, **MHD_CASES[case])
    g = gpu_solve_mhd(_rp("fp64"), x, b, SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True))
    r = ref.solve(x, dt, dh, mag_in=b, store_flux=True, store_ele=True)
    assert scaled_err(g["out"], r["out"]) <= RTOL64
    assert scaled_err(g["flux"], r["flux"], axis_var=2) <= RTOL64
    if case == "no_field":
        assert not np.any(g["mag_out"]) and not np.any(g["ele"])
    else:
        assert _rel(g["mag_out"], r["mag_out"]) <= RTOL64


@pytest.mark.parametrize("precision,tol", [("fp32", RTOL32), ("fp64", RTOL64)])
def test_mhmrp_mhd_char_reconstruction(cuda_device, precision, tol):
    """MHM_RP + MHD with CHAR_RECONSTRUCTION: the half-step state's slopes limited in its seven MHD
    wave amplitudes.  In FP32 the bound is twice the reference's own spread under input round-off
    (the projections amplify rounding, as in CTU)."""
    ref = _need_rp(VARIANT_RP_CHAR, precision)
    x, b, dt, dh = mhd_case(npd=2, seed=12)
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True)
    g = gpu_solve_mhd(_rp(precision, char_reconstruction=True), x, b, prm)
    r = ref.solve(x, dt, dh, mag_in=b, store_flux=True, store_ele=True)
    kw = dict(mag_in=b, store_flux=True, store_ele=True)
    for key, ax in (("out", 1), ("mag_out", 1), ("flux", 2), ("ele", 2)):
        bound = tol if precision == "fp64" else max(tol, 2 * reference_spread(ref, x, dt, dh, 1e-7, key=key, axis_var=ax, **kw))
        assert scaled_err(g[key], r[key], axis_var=ax) <= bound, key
    plain = _need_rp(VARIANT_RP, precision).solve(x, dt, dh, mag_in=b, store_flux=False)
    assert scaled_err(g["out"], plain["out"]) > 100 * tol


@pytest.mark.parametrize("precision,tol", [("fp32", 2e-6), ("fp64", 1e-13)])
def test_mhmrp_mhd_divergence_free(cuda_device, precision, tol):
    x, b, dt, dh = mhd_case(npd=2, seed=13)
    g = gpu_solve_mhd(_rp(precision), x, b, SolverParams(dt=dt, dh=dh, StoreFlux=False))
    scale = _bscale(g["mag_out"])
    assert np.abs(ic.div_b(g["mag_out"])).max() <= tol * scale
    fx, fy, fz = ic.mag_out_faces(g["mag_out"])
    for p in (0, 2, 4, 6):
        assert np.array_equal(fx[p][..., 16], fx[p + 1][..., 0])
    for p in (0, 1, 4, 5):
        assert np.array_equal(fy[p][:, 16, :], fy[p + 2][:, 0, :])
    for p in (0, 1, 2, 3):
        assert np.array_equal(fz[p][16], fz[p + 4][0])


def test_mhmrp_mhd_host_equals_device_and_chunking(cuda_device):
    x, b, dt, dh = mhd_case(npd=2, seed=14)
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True)
    s = _rp("fp32")
    g = gpu_solve_mhd(s, x, b, prm)
    s.set_mhd_chunk(3)
    out, flux, _, bout, ele = s.solve_host(x, prm, mag_in=b)
    assert np.array_equal(out, g["out"]) and np.array_equal(bout, g["mag_out"])
    assert np.array_equal(flux, g["flux"]) and np.array_equal(ele, g["ele"])


def test_mhmrp_mhd_configurations_not_built(cuda_device):
    for kw in ({"dual_energy": True}, {"lr": "ppm", "dual_energy": True}):
        cfg = dict(scheme="mhm_rp", lr="plm", rsolver="hlld", precision="fp32", gamma=GAMMA)
        cfg.update(kw)
        with pytest.raises(FluidSolverError) as ei:
            FluidSolver(**cfg)
        assert ei.value.code == -5


# ---- MHM with MHD (FLU_NXT = 20): a half-step EMF from the input cells, the Hancock predictor with
# MHD fluxes and the half-step update of the face B, the half-step cell primitives as the average of
# the six face states, then the full step (CPU_FluidSolver_MHM.cpp:489-565 with
# Hydro_DataReconstruction's MHD branch), against the reference built with FLU_SCHEME=MHM and MHD ----

VARIANT_MM = "mhm_plm_hlld_mhd"
VARIANT_MM_CHAR = "mhm_plm_hlld_char_mhd"


def _mm(precision, **kw):
    return FluidSolver(scheme="mhm", lr="plm", rsolver="hlld", precision=precision, gamma=GAMMA, **kw)


@pytest.mark.parametrize("precision,tol", [("fp32", RTOL32), ("fp64", RTOL64)])
@pytest.mark.parametrize("char", [False, True])
def test_mhm_mhd_matches_reference(cuda_device, precision, tol, char):
    ref = _need_rp(VARIANT_MM_CHAR if char else VARIANT_MM, precision)
    x, b, dt, dh = mhd_case(npd=2, seed=21, nxt=20)
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True)
    s = _mm(precision, char_reconstruction=char)
    assert s.mhd and s.flu_nxt == 20
    g = gpu_solve_mhd(s, x, b, prm)
    r = ref.solve(x, dt, dh, mag_in=b, store_flux=True, store_ele=True)
    # FP32: twice the reference FP32 build's own spread under one part in 1e7 of input noise
    kw = dict(mag_in=b, store_flux=True, store_ele=True)
    for key, ax in (("out", 1), ("mag_out", 1), ("flux", 2), ("ele", 2)):
        bound = tol if precision == "fp64" else max(tol, 2 * reference_spread(ref, x, dt, dh, 1e-7, key=key, axis_var=ax, **kw))
        assert scaled_err(g[key], r[key], axis_var=ax) <= bound, key


@pytest.mark.parametrize("limiter", ["vanleer", "albada", "central", "vl_gminmod"])
def test_mhm_mhd_limiters(cuda_device, limiter):
    ref = _need_rp(VARIANT_MM, "fp64")
    x, b, dt, dh = mhd_case(npd=2, seed=22, nxt=20)
    g = gpu_solve_mhd(_mm("fp64"), x, b, SolverParams(dt=dt, dh=dh, StoreFlux=False, LR_Limiter=limiter))
    r = ref.solve(x, dt, dh, mag_in=b, store_flux=False, limiter=limiter)
    bound = max(RTOL64, 2 * reference_spread(ref, x, dt, dh, 1e-15, mag_in=b, limiter=limiter))
    assert scaled_err(g["out"], r["out"]) <= bound
    assert scaled_err(g["mag_out"], r["mag_out"]) <= bound


@pytest.mark.parametrize("case", sorted(MHD_CASES))
def test_mhm_mhd_field_regimes(cuda_device, case):
    ref = _need_rp(VARIANT_MM, "fp64")
    x, b, dt, dh = mhd_case(npd=2, seed=23, nxt=20, **MHD_CASES[case])
    g = gpu_solve_mhd(_mm("fp64"), x, b, SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True))
    r = ref.solve(x, dt, dh, mag_in=b, store_flux=True, store_ele=True)
    assert scaled_err(g["out"], r["out"]) <= RTOL64
    assert scaled_err(g["flux"], r["flux"], axis_var=2) <= RTOL64
    if case == "no_field":
        assert not np.any(g["mag_out"]) and not np.any(g["ele"])
    else:
        assert _rel(g["mag_out"], r["mag_out"]) <= RTOL64


@pytest.mark.parametrize("precision,tol", [("fp32", 2e-6), ("fp64", 1e-13)])
def test_mhm_mhd_divergence_free_and_host_entry(cuda_device, precision, tol):
    x, b, dt, dh = mhd_case(npd=2, seed=24, nxt=20)
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True)
    s = _mm(precision)
    g = gpu_solve_mhd(s, x, b, prm)
    assert np.abs(ic.div_b(g["mag_out"])).max() <= tol * _bscale(g["mag_out"])
    s.set_mhd_chunk(3)
    out, flux, _, bout, ele = s.solve_host(x, prm, mag_in=b)
    assert np.array_equal(out, g["out"]) and np.array_equal(bout, g["mag_out"])
    assert np.array_equal(flux, g["flux"]) and np.array_equal(ele, g["ele"])


def test_mhm_mhd_configurations_not_built(cuda_device):
    with pytest.raises(FluidSolverError) as ei:       # dual energy
        FluidSolver(scheme="mhm", lr="plm", rsolver="hlld", precision="fp32", gamma=GAMMA, dual_energy=True)
    assert ei.value.code == -5



# ---- CTU + MHD with PPM (FLU_NXT = 24; GAMER's default MHD configuration): PPM face values and the
# tracing of the parabola over the seven MHD waves, with the MHD source terms ----

VARIANT_PPM = "ctu_ppm_hlld_mhd"
VARIANT_PPM_CHAR = "ctu_ppm_hlld_char_mhd"


@pytest.mark.parametrize("precision,tol", [("fp32", RTOL32), ("fp64", RTOL64)])
@pytest.mark.parametrize("char", [False, True])
def test_ctu_mhd_ppm_matches_reference(cuda_device, precision, tol, char):
    ref = _need_rp(VARIANT_PPM_CHAR if char else VARIANT_PPM, precision)
    x, b, dt, dh = mhd_case(npd=2, seed=31, nxt=24)
    s = FluidSolver(scheme="ctu", lr="ppm", rsolver="hlld", precision=precision, gamma=GAMMA,
                    char_reconstruction=char)
    assert s.flu_nxt == 24
    g = gpu_solve_mhd(s, x, b, SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True))
    r = ref.solve(x, dt, dh, mag_in=b, store_flux=True, store_ele=True)
    kw = dict(mag_in=b, store_flux=True, store_ele=True)
    for key, ax in (("out", 1), ("mag_out", 1), ("flux", 2), ("ele", 2)):
        bound = tol if precision == "fp64" else max(tol, 2 * reference_spread(ref, x, dt, dh, 1e-7, key=key, axis_var=ax, **kw))
        assert scaled_err(g[key], r[key], axis_var=ax) <= bound, key


@pytest.mark.parametrize("limiter", ["vanleer", "albada", "central", "vl_gminmod"])
def test_ctu_mhd_ppm_limiters(cuda_device, limiter):
    ref = _need_rp(VARIANT_PPM, "fp64")
    x, b, dt, dh = mhd_case(npd=2, seed=32, nxt=24)
    s = FluidSolver(scheme="ctu", lr="ppm", rsolver="hlld", precision="fp64", gamma=GAMMA)
    g = gpu_solve_mhd(s, x, b, SolverParams(dt=dt, dh=dh, StoreFlux=False, LR_Limiter=limiter))
    r = ref.solve(x, dt, dh, mag_in=b, store_flux=False, limiter=limiter)
    bound = max(RTOL64, 2 * reference_spread(ref, x, dt, dh, 1e-15, mag_in=b, limiter=limiter))
    assert scaled_err(g["out"], r["out"]) <= bound
    assert scaled_err(g["mag_out"], r["mag_out"]) <= bound


@pytest.mark.parametrize("case", sorted(MHD_CASES))
def test_ctu_mhd_ppm_field_regimes_and_div_b(cuda_device, case):
    ref = _need_rp(VARIANT_PPM, "fp64")
    x, b, dt, dh = mhd_case(npd=2, seed=33, nxt=24, **MHD_CASES[case])
    s = FluidSolver(scheme="ctu", lr="ppm", rsolver="hlld", precision="fp64", gamma=GAMMA)
    g = gpu_solve_mhd(s, x, b, SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True))
    r = ref.solve(x, dt, dh, mag_in=b, store_flux=True, store_ele=True)
    assert scaled_err(g["out"], r["out"]) <= RTOL64
    if case == "no_field":
        assert not np.any(g["mag_out"])
    else:
        assert _rel(g["mag_out"], r["mag_out"]) <= RTOL64
        assert np.abs(ic.div_b(g["mag_out"])).max() <= 1e-13 * _bscale(g["mag_out"])


def test_ctu_mhd_ppm_host_equals_device(cuda_device):
    x, b, dt, dh = mhd_case(npd=2, seed=34, nxt=24)
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True)
    s = FluidSolver(scheme="ctu", lr="ppm", rsolver="hlld", precision="fp32", gamma=GAMMA)
    g = gpu_solve_mhd(s, x, b, prm)
    s.set_mhd_chunk(3)
    out, flux, _, bout, ele = s.solve_host(x, prm, mag_in=b)
    assert np.array_equal(out, g["out"]) and np.array_equal(bout, g["mag_out"])
    assert np.array_equal(flux, g["flux"]) and np.array_equal(ele, g["ele"])



# ---- MHM + MHD with PPM (FLU_NXT = 22) ----

@pytest.mark.parametrize("precision,tol", [("fp32", RTOL32), ("fp64", RTOL64)])
@pytest.mark.parametrize("char", [False, True])
def test_mhm_mhd_ppm_matches_reference(cuda_device, precision, tol, char):
    ref = _need_rp("mhm_ppm_hlld_char_mhd" if char else "mhm_ppm_hlld_mhd", precision)
    x, b, dt, dh = mhd_case(npd=2, seed=41, nxt=22)
    s = FluidSolver(scheme="mhm", lr="ppm", rsolver="hlld", precision=precision, gamma=GAMMA,
                    char_reconstruction=char)
    assert s.flu_nxt == 22
    g = gpu_solve_mhd(s, x, b, SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True))
    r = ref.solve(x, dt, dh, mag_in=b, store_flux=True, store_ele=True)
    kw = dict(mag_in=b, store_flux=True, store_ele=True)
    for key, ax in (("out", 1), ("mag_out", 1), ("flux", 2), ("ele", 2)):
        bound = tol if precision == "fp64" else max(tol, 2 * reference_spread(ref, x, dt, dh, 1e-7, key=key, axis_var=ax, **kw))
        assert scaled_err(g[key], r[key], axis_var=ax) <= bound, key
    if precision == "fp64":
        assert np.abs(ic.div_b(g["mag_out"])).max() <= 1e-13 * _bscale(g["mag_out"])


@pytest.mark.parametrize("limiter", ["vanleer", "central", "vl_gminmod"])
def test_mhm_mhd_ppm_limiters(cuda_device, limiter):
    ref = _need_rp("mhm_ppm_hlld_mhd", "fp64")
    x, b, dt, dh = mhd_case(npd=2, seed=42, nxt=22)
    s = FluidSolver(scheme="mhm", lr="ppm", rsolver="hlld", precision="fp64", gamma=GAMMA)
    g = gpu_solve_mhd(s, x, b, SolverParams(dt=dt, dh=dh, StoreFlux=False, LR_Limiter=limiter))
    r = ref.solve(x, dt, dh, mag_in=b, store_flux=False, limiter=limiter)
    bound = max(RTOL64, 2 * reference_spread(ref, x, dt, dh, 1e-15, mag_in=b, limiter=limiter))
    assert scaled_err(g["out"], r["out"]) <= bound
    assert scaled_err(g["mag_out"], r["mag_out"]) <= bound


# ---- MHM_RP + MHD with PPM (FLU_NXT = 24): the first-order half step over 22^3 half-step cells
# (23 EMF edges, the CT update of B over dt/2), then PPM face values of the half-step state without
# tracing, and the full step of CTU+PPM, against the reference built with FLU_SCHEME=MHM_RP,
# LR_SCHEME=PPM and MHD ----

def _rp_ppm(precision, **kw):
    return FluidSolver(scheme="mhm_rp", lr="ppm", rsolver="hlld", precision=precision, gamma=GAMMA, **kw)


@pytest.mark.parametrize("precision,tol", [("fp32", RTOL32), ("fp64", RTOL64)])
@pytest.mark.parametrize("char", [False, True])
def test_mhmrp_mhd_ppm_matches_reference(cuda_device, precision, tol, char):
    ref = _need_rp("mhmrp_ppm_hlld_char_mhd" if char else "mhmrp_ppm_hlld_mhd", precision)
    x, b, dt, dh = mhd_case(npd=2, seed=51, nxt=24)
    s = _rp_ppm(precision, char_reconstruction=char)
    assert s.mhd and s.flu_nxt == 24
    g = gpu_solve_mhd(s, x, b, SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True))
    r = ref.solve(x, dt, dh, mag_in=b, store_flux=True, store_ele=True)
    kw = dict(mag_in=b, store_flux=True, store_ele=True)
    for key, ax in (("out", 1), ("mag_out", 1), ("flux", 2), ("ele", 2)):
        bound = tol if precision == "fp64" else max(tol, 2 * reference_spread(ref, x, dt, dh, 1e-7, key=key, axis_var=ax, **kw))
        assert scaled_err(g[key], r[key], axis_var=ax) <= bound, key
    # neither the PLM nor the CTU+PPM answer
    x22, b22, _, _ = mhd_case(npd=2, seed=51, nxt=22)
    for other, xo, bo in (("mhmrp_plm_hlld_mhd", x22, b22), (VARIANT_PPM, x, b)):
        o = _need_rp(other, precision).solve(xo, dt, dh, mag_in=bo, store_flux=False)
        assert scaled_err(g["out"], o["out"]) > 100 * tol, other
    if precision == "fp64":
        assert np.abs(ic.div_b(g["mag_out"])).max() <= 1e-13 * _bscale(g["mag_out"])


@pytest.mark.parametrize("limiter", ["vanleer", "albada", "central", "vl_gminmod"])
def test_mhmrp_mhd_ppm_limiters(cuda_device, limiter):
    ref = _need_rp("mhmrp_ppm_hlld_mhd", "fp64")
    x, b, dt, dh = mhd_case(npd=2, seed=52, nxt=24)
    g = gpu_solve_mhd(_rp_ppm("fp64"), x, b, SolverParams(dt=dt, dh=dh, StoreFlux=False, LR_Limiter=limiter))
    r = ref.solve(x, dt, dh, mag_in=b, store_flux=False, limiter=limiter)
    bound = max(RTOL64, 2 * reference_spread(ref, x, dt, dh, 1e-15, mag_in=b, limiter=limiter))
    assert scaled_err(g["out"], r["out"]) <= bound
    assert scaled_err(g["mag_out"], r["mag_out"]) <= bound


@pytest.mark.parametrize("case", sorted(MHD_CASES))
def test_mhmrp_mhd_ppm_field_regimes_and_div_b(cuda_device, case):
    ref = _need_rp("mhmrp_ppm_hlld_mhd", "fp64")
    x, b, dt, dh = mhd_case(npd=2, seed=53, nxt=24, **MHD_CASES[case])
    g = gpu_solve_mhd(_rp_ppm("fp64"), x, b, SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True))
    r = ref.solve(x, dt, dh, mag_in=b, store_flux=True, store_ele=True)
    assert scaled_err(g["out"], r["out"]) <= RTOL64
    assert scaled_err(g["flux"], r["flux"], axis_var=2) <= RTOL64
    if case == "no_field":
        assert not np.any(g["mag_out"]) and not np.any(g["ele"])
    else:
        assert _rel(g["mag_out"], r["mag_out"]) <= RTOL64
        assert np.abs(ic.div_b(g["mag_out"])).max() <= 1e-13 * _bscale(g["mag_out"])


def test_mhmrp_mhd_ppm_host_equals_device(cuda_device):
    x, b, dt, dh = mhd_case(npd=2, seed=54, nxt=24)
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True)
    s = _rp_ppm("fp32")
    g = gpu_solve_mhd(s, x, b, prm)
    s.set_mhd_chunk(3)
    out, flux, _, bout, ele = s.solve_host(x, prm, mag_in=b)
    assert np.array_equal(out, g["out"]) and np.array_equal(bout, g["mag_out"])
    assert np.array_equal(flux, g["flux"]) and np.array_equal(ele, g["ele"])


# ---- the MinMod retries of MHM and MHM_RP with MHD (CPU_FluidSolver_MHM.cpp:466-585): a patch group
# whose output holds an unphysical cell (Hydro_IsUnphysical with the magnetic energy of the updated
# face B) is solved again with the MinMod coefficient reduced by coeff/MinMod_MaxIter per pass; a
# weak field at Mach 3 and CFL 0.6 leaves 1 to 4 of the 8 patch groups unphysical on the first pass ----

RETRY_CASES = [("mhm", "plm", 20, "mhm_plm_hlld_mhd"), ("mhm_rp", "plm", 22, "mhmrp_plm_hlld_mhd"),
               ("mhm", "ppm", 22, "mhm_ppm_hlld_mhd"), ("mhm_rp", "ppm", 24, "mhmrp_ppm_hlld_mhd")]


@pytest.mark.parametrize("scheme,lr,nxt,variant", RETRY_CASES)
@pytest.mark.parametrize("precision,tol", [("fp32", RTOL32), ("fp64", RTOL64)])
def test_mhd_minmod_retries_match_reference(cuda_device, scheme, lr, nxt, variant, precision, tol):
    ref = _need_rp(variant, precision)
    x, b, dt, dh = mhd_case(npd=2, seed=60, nxt=nxt, cfl=0.6, b0=(0.1, 0.1, 0.1), mach=3.0)
    kw = dict(mag_in=b, store_flux=True, store_ele=True, limiter="gminmod", minmod_maxiter=3)
    r = ref.solve(x, dt, dh, **kw)
    once = ref.solve(x, dt, dh, **dict(kw, minmod_maxiter=0))["out"]
    retried = np.any((r["out"] != once).reshape(len(x), -1), axis=1)
    assert 0 < retried.sum() < len(x)              # the case retries some patch groups, not all
    s = FluidSolver(scheme=scheme, lr=lr, rsolver="hlld", precision=precision, gamma=GAMMA)
    assert s.flu_nxt == nxt
    g = gpu_solve_mhd(s, x, b, SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True, MinMod_MaxIter=3))
    for key, ax in (("out", 1), ("mag_out", 1), ("flux", 2), ("ele", 2)):
        bound = tol if precision == "fp64" else max(tol, 2 * reference_spread(ref, x, dt, dh, 1e-7, key=key, axis_var=ax, **kw))
        assert scaled_err(g[key], r[key], axis_var=ax) <= bound, key
    # the patch groups the reference did not retry are those of a solve without retries, bit for bit
    g0 = gpu_solve_mhd(s, x, b, SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True))
    keep = ~retried
    for key in ("out", "mag_out", "flux", "ele"):
        assert np.array_equal(g[key][keep], g0[key][keep]), key
    if precision == "fp64":
        assert np.abs(ic.div_b(g["mag_out"])).max() <= 1e-13 * _bscale(g["mag_out"])


def test_mhd_minmod_retries_host_entry_equals_device(cuda_device):
    x, b, dt, dh = mhd_case(npd=2, seed=60, nxt=22, cfl=0.6, b0=(0.1, 0.1, 0.1), mach=3.0)
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True, MinMod_MaxIter=3)
    s = _rp("fp32")
    g = gpu_solve_mhd(s, x, b, prm)
    s.set_mhd_chunk(3)
    out, flux, _, bout, ele = s.solve_host(x, prm, mag_in=b)
    assert np.array_equal(out, g["out"]) and np.array_equal(bout, g["mag_out"])
    assert np.array_equal(flux, g["flux"]) and np.array_equal(ele, g["ele"])
