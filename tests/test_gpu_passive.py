"""GPU parity of the run-time options of CPU_FluidSolver (src/Fluid/CPU_FluidSolver.cpp:210-232) that
act on passive scalars and on the pressure floor, and of the asynchronous host-array call.

* User passive scalars (NCOMP_PASSIVE_USER = 2, with and without the dual-energy field after them)
  against the reference built with them (oracle/_ref libgref_mhm_plm_hllc_p2*): reconstructed as
  densities or, with FracPassive, as mass fractions; upwinded with the mass flux; floored where
  PassiveFloor says so; rescaled to the density with NormPassive (Hydro_NormalizePassive,
  CPU_Shared_FluUtility.cpp:1536).
* JeansMinPres: the pressure floor JeansMinPres_Coeff*rho^2 of the cell-centred primitive variables
  (CPU_Shared_FluUtility.cpp:272-281), MHM and hydro CTU.
* gb_fluid_solve_host_async + gb_fluid_synchronize (CUAPI_Asyn_FluidSolver + CUAPI_Synchronize):
  host work between the call and the synchronisation; the result equals the synchronous call's.
"""
import numpy as np
import pytest

import pyoracle as po
from gamer_b200.fluid import FluidSolver, FluidSolverError, PinnedArray, SolverParams
from parity import (GAMMA, RTOL32, RTOL64, blast_case, gpu_solve, kh_case, lognormal_case, scaled_err,
                    with_passive)

pytestmark = pytest.mark.gpu

TOL = {"fp32": RTOL32, "mixed": RTOL32, "fp64": RTOL64}


def _ref(dual, prec):
    return po.RefSolver("mhm_plm_hllc_p2" + ("_de" if dual else ""), "fp64" if prec == "fp64" else "fp32")


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
@pytest.mark.parametrize("dual", [False, True])
def test_passive_scalars_match_reference(cuda_device, dual, prec):
    x, dt, dh = lognormal_case(npd=2, seed=70, dual=dual)
    x = with_passive(x, dual, 3)
    s = FluidSolver(precision=prec, dual_energy=dual, npassive_user=2)
    assert s.ncomp == 7 + int(dual)
    # (8 double variables: 211 KB of shared memory per CTA with single-buffered flux planes)
    ref = _ref(dual, prec).solve(x, dt, dh)
    g = gpu_solve(s, x, SolverParams(dt=dt, dh=dh))
    assert scaled_err(g["out"], ref["out"]) <= TOL[prec]
    assert scaled_err(g["flux"], ref["flux"], axis_var=2) <= TOL[prec]
    if dual:
        assert np.mean(g["de"] == ref["de"]) > 0.999 if prec != "fp64" else np.array_equal(g["de"], ref["de"])
    assert s.status() == 0


@pytest.mark.parametrize("prec,dual", [("fp32", True), ("mixed", True), ("fp64", False)])
def test_passive_scalars_blast_with_retries(cuda_device, prec, dual):
    """Mach-10 blast with MinMod retries (and dual energy in float): the Hancock reset, the retry
    loop and the dual-energy fix act on the last variable, after the user passive scalars."""
    x, dt, dh = blast_case(npd=2, seed=72, nxt=20, dual=dual)
    x = with_passive(x, dual, 5)
    ref = _ref(dual, prec).solve(x, 2.0 * dt, dh, minmod_maxiter=3)
    g = gpu_solve(FluidSolver(precision=prec, dual_energy=dual, npassive_user=2), x,
                  SolverParams(dt=2.0 * dt, dh=dh, MinMod_MaxIter=3), pg_fail=True)
    assert scaled_err(g["out"], ref["out"]) <= (1e-9 if prec == "fp64" else 2e-3)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("norm,frac", [((0, 1), ()), ((), (0, 1)), ((1, 0), (1,))])
def test_norm_and_frac_passive_match_reference(cuda_device, prec, norm, frac):
    """NormPassive (the listed scalars rescaled to sum to the density, summed in list order) and
    FracPassive (the listed scalars reconstructed as mass fractions) against the reference with the
    same NormIdx / FracIdx."""
    x, dt, dh = kh_case(npd=2, seed=71, nxt=20, dual=False)
    x = with_passive(x, False, 4)
    ref = _ref(False, prec).solve(x, dt, dh, norm_idx=norm, frac_idx=frac)
    g = gpu_solve(FluidSolver(precision=prec, npassive_user=2), x,
                  SolverParams(dt=dt, dh=dh, NormIdx=norm, FracIdx=frac))
    assert scaled_err(g["out"], ref["out"]) <= TOL[prec]
    assert scaled_err(g["flux"], ref["flux"], axis_var=2) <= TOL[prec]
    if norm:
        # the normalised scalars sum to the density up to round-off
        tot = g["out"][:, 5].astype(np.float64) + g["out"][:, 6]
        rho = g["out"][:, 0].astype(np.float64)
        assert np.max(np.abs(tot - rho) / rho) <= (1e-6 if prec != "fp64" else 1e-14)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("floor", [0, 1 << 5, (1 << 5) | (1 << 6)])
def test_passive_floor_mask_matches_reference(cuda_device, prec, floor):
    """Negative passive densities in a band of cells: floored (and flagged unphysical) only for the
    variables whose PassiveFloor bit is set, as in the reference."""
    x, dt, dh = lognormal_case(npd=2, seed=75, dual=False)
    x = with_passive(x, False, 6)
    x[:, 5, :, :, 3:6] *= -0.01
    x[:, 6, :, 7:9, :] *= -0.01
    ref = _ref(False, prec).solve(x, dt, dh, passive_floor=floor)
    g = gpu_solve(FluidSolver(precision=prec, npassive_user=2), x, SolverParams(dt=dt, dh=dh, PassiveFloor=floor))
    assert scaled_err(g["out"], ref["out"]) <= TOL[prec]
    # with the bit cleared the negative densities survive; with it set they are floored
    if floor & (1 << 5):
        assert not np.any(g["out"][:, 5] < 0)
    else:
        assert np.any(g["out"][:, 5] < 0)


def test_passive_options_are_checked(cuda_device):
    x, dt, dh = lognormal_case(npd=1, seed=7)
    x = with_passive(x, False, 1)
    s = FluidSolver(npassive_user=2)
    for bad in (dict(NormIdx=(0, 0)), dict(NormIdx=(2,)), dict(FracIdx=(0, 1, 1)), dict(JeansMinPres=True,
                                                                                         JeansMinPres_Coeff=-1.0)):
        with pytest.raises(FluidSolverError) as ei:
            gpu_solve(s, x, SolverParams(dt=dt, dh=dh, **bad))
        assert ei.value.code == -1
    # no passive scalars: NormPassive has nothing to act on
    with pytest.raises(FluidSolverError):
        gpu_solve(FluidSolver(), x[:, :5], SolverParams(dt=dt, dh=dh, NormIdx=(0,)))
    # passive scalars are built for hydro MHM, MHM_RP and CTU, not for MHD or FP64 MHM / MHM_RP with
    # PPM and dual energy
    for kw in (dict(scheme="ctu", rsolver="hlld"), dict(scheme="mhm_rp", lr="ppm", precision="fp64", dual_energy=True),
               dict(scheme="mhm", lr="ppm", precision="fp64", dual_energy=True)):
        with pytest.raises(FluidSolverError) as ei:
            FluidSolver(npassive_user=2, **kw)
        assert ei.value.code == -5


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
@pytest.mark.parametrize("lr,rs", [("plm", "hllc"), ("ppm", "roe")])
def test_jeans_min_pres_matches_reference(cuda_device, prec, lr, rs):
    """JeansMinPres_Coeff = 1: the floor rho^2 lies above the pressure in about half of the cells."""
    nxt = 22 if lr == "ppm" else 20
    x, dt, dh = lognormal_case(npd=2, seed=77, nxt=nxt)
    rv = po.RefSolver(f"mhm_{lr}_{rs}", "fp64" if prec == "fp64" else "fp32")
    ref = rv.solve(x, dt, dh, jeans=True, jeans_coeff=1.0)
    plain = rv.solve(x, dt, dh)
    g = gpu_solve(FluidSolver(lr=lr, rsolver=rs, precision=prec, flu_nxt=nxt), x,
                  SolverParams(dt=dt, dh=dh, JeansMinPres=True, JeansMinPres_Coeff=1.0))
    assert scaled_err(g["out"], ref["out"]) <= TOL[prec]
    # the floor acted: the result is not the plain solve's
    assert scaled_err(plain["out"], ref["out"]) > 100 * TOL[prec]


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_jeans_min_pres_ctu_matches_reference(cuda_device, prec):
    x, dt, dh = lognormal_case(npd=2, seed=78, nxt=20)
    ref = po.RefSolver("ctu_plm_hllc", prec).solve(x, dt, dh, jeans=True, jeans_coeff=1.0)
    g = gpu_solve(FluidSolver(scheme="ctu", precision=prec), x,
                  SolverParams(dt=dt, dh=dh, JeansMinPres=True, JeansMinPres_Coeff=1.0))
    assert scaled_err(g["out"], ref["out"]) <= (RTOL32 if prec == "fp32" else RTOL64)


@pytest.mark.parametrize("scheme,prec", [("mhm", "mixed"), ("mhm", "fp64"), ("ctu", "fp32")])
def test_async_host_call_equals_synchronous_call(cuda_device, scheme, prec):
    """CUAPI_Asyn_FluidSolver's contract: the call returns before the result exists, the caller
    prepares the next batch meanwhile (here: fills the other pinned buffer set), and
    gb_fluid_synchronize ends it.  Two batches in flight back to back on ping-pong buffers give the
    synchronous call's results bit for bit."""
    s = FluidSolver(scheme=scheme, precision=prec)
    batches = [lognormal_case(npd=3, seed=80 + b) for b in range(3)]
    prm = [SolverParams(dt=dt, dh=dh) for _, dt, dh in batches]
    want = [s.solve_host(x, p)[:2] for (x, _, _), p in zip(batches, prm)]
    npg, nc = batches[0][0].shape[0], s.ncomp
    sets = [dict(inp=PinnedArray((npg, nc, 20, 20, 20), s.np_dtype), out=PinnedArray((npg, nc, 16, 16, 16), s.np_dtype),
                 flux=PinnedArray((npg, 9, nc, 16, 16), s.np_dtype)) for _ in range(2)]
    sets[0]["inp"].array[...] = batches[0][0]
    got = []
    for b in range(3):
        cur, nxt = sets[b % 2], sets[(b + 1) % 2]
        s.solve_host_async(cur["inp"].array, cur["out"].array, prm[b], flux=cur["flux"].array)
        if b + 1 < 3:
            nxt["inp"].array[...] = batches[b + 1][0]      # host-side preparation of the next batch
        s.synchronize()
        got.append((cur["out"].array.copy(), cur["flux"].array.copy()))
    for (go, gf), (wo, wf) in zip(got, want):
        assert np.array_equal(go, wo) and np.array_equal(gf, wf)
    for st in sets:
        for a in st.values():
            a.free()


def test_async_host_call_orders_with_a_torch_stream(cuda_device):
    """The call waits for the work already on the given stream and the stream waits for the call,
    so synchronising the stream alone ends it."""
    import torch
    x, dt, dh = lognormal_case(npd=2, seed=90)
    s = FluidSolver()
    want, _, _ = s.solve_host(x, SolverParams(dt=dt, dh=dh))
    inp = PinnedArray(x.shape, np.float32)
    out = PinnedArray((x.shape[0], 5, 16, 16, 16), np.float32)
    inp.array[...] = x
    out.array[...] = np.nan
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        torch.cuda._sleep(2_000_000)            # earlier work on the stream: the copies must wait for it
    s.solve_host_async(inp.array, out.array, SolverParams(dt=dt, dh=dh, StoreFlux=False), stream=st)
    st.synchronize()
    assert np.array_equal(out.array, want)
    inp.free()
    out.free()



# ---- hydro CTU with user passive scalars: traced with the entropy wave alone, PassiveFloor,
# FracPassive in the reconstruction and NormPassive in the update, against the reference's CTU
# builds with NCOMP_PASSIVE_USER = 2 (oracle/_ref libgref_ctu_plm_*_p2*) ----

def _ref_ctu(rs, dual, prec):
    variant = f"ctu_plm_{rs}_p2" + ("_de" if dual else "")
    rprec = "fp64" if prec == "fp64" else "fp32"
    if not po.ref_available(variant, rprec):
        pytest.skip(f"oracle/_ref/libgref_{variant}_{rprec}.so not built")
    return po.RefSolver(variant, rprec)


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
@pytest.mark.parametrize("rs,dual", [("hllc", False), ("roe", False), ("hllc", True)])
def test_ctu_passive_scalars_match_reference(cuda_device, rs, dual, prec):
    x, dt, dh = lognormal_case(npd=2, seed=76, dual=dual)
    x = with_passive(x, dual, 7)
    s = FluidSolver(scheme="ctu", rsolver=rs, precision=prec, dual_energy=dual, npassive_user=2)
    assert s.ncomp == 7 + int(dual)
    ref = _ref_ctu(rs, dual, prec).solve(x, dt, dh)
    g = gpu_solve(s, x, SolverParams(dt=dt, dh=dh))
    assert scaled_err(g["out"], ref["out"]) <= TOL[prec]
    assert scaled_err(g["flux"], ref["flux"], axis_var=2) <= TOL[prec]
    if dual:
        assert np.mean(g["de"] == ref["de"]) > 0.999 if prec != "fp64" else np.array_equal(g["de"], ref["de"])


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("norm,frac,floor", [((0, 1), (), 0), ((), (0, 1), 0), ((1, 0), (1,), (1 << 5) | (1 << 6))])
def test_ctu_norm_frac_and_floor_match_reference(cuda_device, prec, norm, frac, floor):
    x, dt, dh = lognormal_case(npd=2, seed=77, dual=False)
    x = with_passive(x, False, 8)
    if floor:
        x[:, 5, :, :, 3:6] *= -0.01
    ref = _ref_ctu("hllc", False, prec).solve(x, dt, dh, norm_idx=norm, frac_idx=frac, passive_floor=floor)
    g = gpu_solve(FluidSolver(scheme="ctu", precision=prec, npassive_user=2), x,
                  SolverParams(dt=dt, dh=dh, NormIdx=norm, FracIdx=frac, PassiveFloor=floor))
    assert scaled_err(g["out"], ref["out"]) <= TOL[prec]
    assert scaled_err(g["flux"], ref["flux"], axis_var=2) <= TOL[prec]



# ---- user passive scalars in MHM_RP: the half step solves and advances them with the fluid (floored
# by PassiveFloor, converted to mass fractions by FracPassive in Hydro_Con2Pri), the full step
# reconstructs them from the half-step state ----

@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
@pytest.mark.parametrize("variant,lr,rs,dual,char", [("mhmrp_plm_hllc_p2", "plm", "hllc", False, False),
                                                     ("mhmrp_plm_roe_p2_de", "plm", "roe", True, False),
                                                     ("mhmrp_plm_hllc_p2_char", "plm", "hllc", False, True),
                                                     ("mhmrp_ppm_hllc_p2", "ppm", "hllc", False, False),
                                                     ("mhmrp_ppm_hllc_p2_char", "ppm", "hllc", False, True),
                                                     ("mhmrp_ppm_hlle_p2_de", "ppm", "hlle", True, False)])
def test_mhm_rp_passive_scalars_match_reference(cuda_device, prec, variant, lr, rs, dual, char):
    rprec = "fp64" if prec == "fp64" else "fp32"
    if not po.ref_available(variant, rprec):
        pytest.skip(f"reference variant {variant} not built")
    if prec == "fp64" and lr == "ppm" and dual:
        pytest.skip("not built: FP64 MHM_RP+PPM with 8 variables")
    nxt = 24 if lr == "ppm" else 22
    x, dt, dh = lognormal_case(npd=2, seed=78, nxt=nxt, dual=dual)
    x = with_passive(x, dual, 9)
    s = FluidSolver(scheme="mhm_rp", lr=lr, rsolver=rs, precision=prec, dual_energy=dual, npassive_user=2,
                    char_reconstruction=char)
    assert s.ncomp == 7 + int(dual) and s.flu_nxt == nxt
    ref = po.RefSolver(variant, rprec).solve(x, dt, dh)
    g = gpu_solve(s, x, SolverParams(dt=dt, dh=dh))
    assert scaled_err(g["out"], ref["out"]) <= TOL[prec]
    assert scaled_err(g["flux"], ref["flux"], axis_var=2) <= TOL[prec]
    if dual:
        assert np.mean(g["de"] == ref["de"]) > 0.999
    assert s.status() == 0


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("norm,frac,floor", [((0, 1), (), 0), ((), (0, 1), 0), ((1, 0), (1,), (1 << 5) | (1 << 6))])
def test_mhm_rp_norm_frac_and_floor_match_reference(cuda_device, prec, norm, frac, floor):
    x, dt, dh = kh_case(npd=2, seed=79, nxt=22, dual=False)
    x = with_passive(x, False, 10)
    if floor:
        x[:, 5, :, :, 3:6] *= -0.01
    ref = po.RefSolver("mhmrp_plm_hllc_p2", prec).solve(x, dt, dh, norm_idx=norm, frac_idx=frac, passive_floor=floor,
                                                         limiter="vanleer")
    g = gpu_solve(FluidSolver(scheme="mhm_rp", precision=prec, npassive_user=2), x,
                  SolverParams(dt=dt, dh=dh, NormIdx=norm, FracIdx=frac, PassiveFloor=floor, LR_Limiter="vanleer"))
    assert scaled_err(g["out"], ref["out"]) <= TOL[prec]
    assert scaled_err(g["flux"], ref["flux"], axis_var=2) <= TOL[prec]


def test_mhm_rp_passive_blast_with_retries(cuda_device):
    x, dt, dh = blast_case(npd=2, seed=80, nxt=22, dual=False)
    x = with_passive(x, False, 11)
    ref = po.RefSolver("mhmrp_plm_hllc_p2", "fp64")
    r = ref.solve(x, 1.5 * dt, dh, minmod_maxiter=3)
    assert not np.array_equal(r["out"], ref.solve(x, 1.5 * dt, dh, minmod_maxiter=0)["out"])
    g = gpu_solve(FluidSolver(scheme="mhm_rp", precision="fp64", npassive_user=2), x,
                  SolverParams(dt=1.5 * dt, dh=dh, MinMod_MaxIter=3), pg_fail=True)
    assert scaled_err(g["out"], r["out"]) <= 1e-9


def test_mhm_rp_passive_host_entry_equals_device(cuda_device):
    x, dt, dh = lognormal_case(npd=2, seed=81, nxt=24)
    x = with_passive(x, False, 12)
    s = FluidSolver(scheme="mhm_rp", lr="ppm", npassive_user=2)
    prm = SolverParams(dt=dt, dh=dh)
    g = gpu_solve(s, x, prm)
    out, flux, _ = s.solve_host(x, prm)[:3]
    assert np.array_equal(out, g["out"]) and np.array_equal(flux, g["flux"])


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
def test_mhm_ppm_char_passive_dual_energy_matches_reference(cuda_device, prec):
    """MHM+PPM with CHAR_RECONSTRUCTION, two passive scalars and dual energy (8 variables; float
    storage: in FP64 the planes do not fit a CTA's shared memory): the fluid slopes limited in
    characteristic variables, the passive and dual-energy slopes as they are."""
    rprec = "fp64" if prec == "fp64" else "fp32"
    variant = "mhm_ppm_roe_p2_de_char"
    if not po.ref_available(variant, rprec):
        pytest.skip(f"reference variant {variant} not built")
    x, dt, dh = lognormal_case(npd=2, seed=82, nxt=22, dual=True)
    x = with_passive(x, True, 13)
    s = FluidSolver(lr="ppm", rsolver="roe", precision=prec, dual_energy=True, npassive_user=2,
                    char_reconstruction=True)
    assert s.ncomp == 8 and s.flu_nxt == 22
    ref = po.RefSolver(variant, rprec).solve(x, dt, dh)
    g = gpu_solve(s, x, SolverParams(dt=dt, dh=dh))
    assert scaled_err(g["out"], ref["out"]) <= TOL[prec]
    assert scaled_err(g["flux"], ref["flux"], axis_var=2) <= TOL[prec]
    assert np.mean(g["de"] == ref["de"]) > 0.999

