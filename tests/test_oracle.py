"""CPU tests of the oracle: the C restatement (oracle/gamer_oracle.c) against the reference's own
outputs — the committed golden fixtures (tests/golden, made by tests/golden/make_golden.py from the
reference compiled from source) and, where oracle/_ref is built, the reference library directly."""
import glob
import os

import numpy as np
import pytest

import pyoracle as po
from gamer_b200 import ic
from parity import GAMMA, blast_case, kh_case, lognormal_case

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_restated_oracle_matches_golden_bit_for_bit(path):
    d = np.load(path)
    r = po.restated_mhm(d["flu_in"], float(d["dt"]), float(d["dh"]), lr=str(d["lr"]), rsolver=str(d["rsolver"]),
                        dual=bool(d["dual"]), limiter=str(d["limiter"]), minmod_maxiter=int(d["minmod_maxiter"]),
                        precision=str(d["precision"]), gamma=float(d["gamma"]),
                        char=bool(d["char"]) if "char" in d.files else False,
                        scheme=str(d["scheme"]) if "scheme" in d.files else "mhm")
    assert np.array_equal(r["out"], d["flu_out"])
    assert np.array_equal(r["flux"], d["flux"])
    if bool(d["dual"]):
        assert np.array_equal(r["de"], d["de"])


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 4


def _need_ref(variant, prec):
    if not po.ref_available(variant, prec):
        pytest.skip(f"oracle/_ref/libgref_{variant}_{prec}.so not built (needs the reference tree)")


CASES = [
    ("plm", "hllc", False), ("plm", "roe", False), ("plm", "hlle", False),
    ("ppm", "roe", False), ("ppm", "hllc", False), ("plm", "hllc", True),
    ("plm", "exact", False), ("ppm", "exact", False), ("plm", "exact", True),
]


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("lr,rs,dual", CASES)
@pytest.mark.parametrize("kind", ["lognormal", "kh", "blast"])
def test_restated_oracle_matches_reference_bit_for_bit(kind, lr, rs, dual, prec):
    variant = po.ref_variant_name("mhm", lr, rs, dual=dual)
    _need_ref(variant, prec)
    nxt = 22 if lr == "ppm" else 20
    if kind == "lognormal":
        x, dt, dh = lognormal_case(npd=2, seed=99, nxt=nxt, dual=dual)
        kw = dict(limiter="gminmod", minmod_maxiter=0)
    elif kind == "kh":
        x, dt, dh = kh_case(npd=2, seed=98, nxt=nxt, dual=dual)
        kw = dict(limiter="vl_gminmod", minmod_maxiter=0)
    else:
        x, dt, dh = blast_case(npd=2, seed=97, nxt=nxt, dual=dual)
        dt *= 2.0          # CFL 1: provokes Hancock resets, rescues and MinMod retries
        kw = dict(limiter="gminmod", minmod_maxiter=3)
    x = x[:4]
    ref = po.RefSolver(variant, prec).solve(x, dt, dh, **kw)
    res = po.restated_mhm(x, dt, dh, lr=lr, rsolver=rs, dual=dual, precision=prec, **kw)
    assert np.array_equal(res["out"], ref["out"])
    assert np.array_equal(res["flux"], ref["flux"])
    if dual:
        assert np.array_equal(res["de"], ref["de"])


@pytest.mark.parametrize("limiter", ["vanleer", "albada", "vl_gminmod", "central"])
def test_restated_limiters_match_reference(limiter):
    _need_ref("mhm_plm_hllc", "fp32")
    x, dt, dh = lognormal_case(npd=2, seed=3)
    x = x[:2]
    ref = po.RefSolver("mhm_plm_hllc", "fp32").solve(x, dt, dh, limiter=limiter)
    res = po.restated_mhm(x, dt, dh, limiter=limiter)
    assert np.array_equal(res["out"], ref["out"])


def test_oracle_rotation_symmetry():
    """A state rotated x->y->z->x gives the rotated result (size-independent property)."""
    box = ic.lognormal_box(1, seed=5, gamma=GAMMA)
    dh = 1.0 / 16
    dt = ic.cfl_dt(box, GAMMA, dh)
    rot = np.stack([box[0], box[3], box[1], box[2], box[4]])          # (x,y,z) -> (y,z,x) components
    rot = np.transpose(rot, (0, 3, 1, 2))                              # and coordinates
    a = po.restated_mhm(ic.cut_patch_groups(box, 20), dt, dh, precision="fp64")["out"]
    b = po.restated_mhm(ic.cut_patch_groups(rot, 20), dt, dh, precision="fp64")["out"]
    A = ic.assemble_box(a, 1)
    B = ic.assemble_box(b, 1)
    A_rot = np.transpose(np.stack([A[0], A[3], A[1], A[2], A[4]]), (0, 3, 1, 2))
    assert np.max(np.abs(A_rot - B)) <= 1e-12 * np.max(np.abs(A))


def test_oracle_uniform_state_fixed_point():
    x = np.zeros((2, 5, 20, 20, 20))
    x[:, 0], x[:, 1], x[:, 2], x[:, 4] = 2.0, 0.3, -0.2, 3.0
    r = po.restated_mhm(x, 1e-3, 1e-2, precision="fp64")
    assert np.array_equal(r["out"], x[:, :, 2:18, 2:18, 2:18])


def test_oracle_rejects_too_small_input():
    with pytest.raises(ValueError):
        po.restated_mhm(np.ones((1, 5, 18, 18, 18)), 1e-3, 1e-2)


def test_reference_dt_solver_matches_a_direct_cfl_bound():
    """The reference CFL solver on patches cut from a box (LocalID order) against the CFL bound of
    the whole box written out in numpy: the minimum agrees, and each patch's dt is its own bound."""
    from gamer_b200 import ic
    from parity import GAMMA
    box = ic.lognormal_box(2, seed=3, gamma=GAMMA)
    dh = 1.0 / 32
    out = np.stack([np.transpose(box[:, 16 * px:16 * px + 16, 16 * py:16 * py + 16, 16 * pz:16 * pz + 16], (0, 3, 2, 1))
                    for pz in range(2) for py in range(2) for px in range(2)])
    flu, _ = ic.patches_from_output(out)
    dt = po.RefSolver("mhm_plm_hllc", "fp64").dt(flu, dh, safety=0.5)
    rho = box[0]
    v = np.abs(box[1:4] / rho)
    p = (GAMMA - 1.0) * (box[4] - 0.5 * (box[1] ** 2 + box[2] ** 2 + box[3] ** 2) / rho)
    smax = (v + np.sqrt(GAMMA * p / rho)).max(axis=0)
    assert abs(dt.min() - 0.5 * dh / smax.max()) <= 1e-14 * dt.min()
    # patch LocalID 7 of patch group 0 covers cells [8,16)^3
    assert abs(dt[7] - 0.5 * dh / smax[8:16, 8:16, 8:16].max()) <= 1e-14 * dt[7]


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_reference_char_reconstruction_build_differs_from_primitive_build(prec):
    """The CHAR_RECONSTRUCTION build of the reference is a different scheme (the option reached the
    compiler)."""
    _need_ref("mhm_plm_hllc_char", prec)
    x, dt, dh = lognormal_case(npd=1, seed=36)
    rc = po.RefSolver("mhm_plm_hllc_char", prec).solve(x, dt, dh)
    rp = po.RefSolver("mhm_plm_hllc", prec).solve(x, dt, dh)
    assert np.all(np.isfinite(rc["out"]))
    assert not np.allclose(rc["out"], rp["out"], rtol=1e-6, atol=0)


def test_reference_correct_unphysical_repairs_planted_cells_only(tmp_path):
    """The reference's CorrectUnphysical() (src/Fluid/Flu_Close.cpp:542) through the oracle entry:
    on a smooth flow with a few cells made unphysical, exactly those cells are replaced, each by a
    state with positive density, and the fluxes that change are the coarse-fine faces they touch."""
    _need_ref("mhm_plm_hllc", "fp64")
    x, dt, dh = lognormal_case(npd=1, seed=37)
    ref = po.RefSolver("mhm_plm_hllc", "fp64")
    r = ref.solve(x, dt, dh)
    out = r["out"].copy()
    cells = [(0, 0, 0), (7, 3, 5), (8, 3, 5), (5, 9, 15)]
    for (i, j, k) in cells:
        out[0, 0, k, j, i] = -1.0
    c = ref.correct_unphysical(x, out, dt, dh, flux=r["flux"], corr="3d", scheme="hllc", outdir=str(tmp_path))
    assert c["rc"] == 0 and c["ncorr"] == len(cells)
    changed = np.argwhere(np.any(c["out"] != out, axis=1))
    assert sorted(map(tuple, changed[:, [3, 2, 1]].tolist())) == sorted(cells)
    assert all(c["out"][0, 0, k, j, i] > 0 for (i, j, k) in cells)
    # (0,0,0): x, y, z low faces; (7,3,5)/(8,3,5): the x middle face (twice); (5,9,15): z high face
    assert int(np.any(c["flux"] != r["flux"], axis=2).sum()) == 5


@pytest.mark.parametrize("lr", ["plm", "ppm"])
def test_reference_exact_solver_builds_run(lr):
    """The RSOLVER = EXACT builds of the reference (the oracle of the device exact solver): finite
    output, and FP32 within 1e-5 of FP64 on a smooth flow."""
    _need_ref(f"mhm_{lr}_exact", "fp64")
    nxt = 22 if lr == "ppm" else 20
    x, dt, dh = lognormal_case(npd=1, seed=45, nxt=nxt)
    r64 = po.RefSolver(f"mhm_{lr}_exact", "fp64").solve(x, dt, dh)["out"]
    r32 = po.RefSolver(f"mhm_{lr}_exact", "fp32").solve(x, dt, dh)["out"]
    assert np.all(np.isfinite(r64))
    rms = np.sqrt((r64 ** 2).mean(axis=(0, 2, 3, 4), keepdims=True))
    assert np.max(np.abs(r32 - r64) / (np.abs(r64) + rms)) < 1e-5


def test_reference_flux_fixup_applies_faces_in_order():
    """Flu_FixUp_Flux() (src/Fluid/Flu_FixUp_Flux.cpp:23) through the oracle entry: a patch with a
    density flux difference on its x-low and y-low faces changes only the cells of those layers,
    each by -F/dh per face, the corner column twice; the energy is rebuilt from the unchanged
    internal energy."""
    _need_ref("mhm_plm_hllc", "fp64")
    ref = po.RefSolver("mhm_plm_hllc", "fp64")
    u = np.zeros((1, 5, 8, 8, 8))
    u[:, 0], u[:, 4] = 1.0, 1.5
    flux = np.zeros((1, 6, 5, 8, 8))
    flux[0, 0, 0], flux[0, 2, 0] = 1e-3, 2e-3
    has = np.array([[1, 0, 1, 0, 0, 0]], np.uint8)
    dh = 0.01
    o = ref.fixup_flux(u, flux, has, dh)
    changed = np.any(o != u, axis=1)[0]
    assert changed[:, :, 0].all() and changed[:, 0, :].all() and changed.sum() == 8 * 8 + 8 * 8 - 8
    assert np.isclose(o[0, 0, 3, 5, 0], 1.0 - 0.1)           # x-low face only
    assert np.isclose(o[0, 0, 3, 0, 5], 1.0 - 0.2)           # y-low face only
    assert np.isclose(o[0, 0, 3, 0, 0], 1.0 - 0.3)           # both, in order
    assert np.allclose(o[0, 4], 1.5)                         # no momentum: E = Eint unchanged


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("rs", ["hllc", "roe", "hlle"])
@pytest.mark.parametrize("kind,limiter", [("lognormal", "gminmod"), ("kh", "vl_gminmod"), ("blast", "vanleer")])
def test_restated_char_reconstruction_matches_reference_bit_for_bit(kind, limiter, rs, prec):
    """The restatement with CHAR_RECONSTRUCTION against the reference built with it."""
    variant = po.ref_variant_name("mhm", "plm", rs, char=True)
    _need_ref(variant, prec)
    if kind == "lognormal":
        x, dt, dh = lognormal_case(npd=2, seed=96)
        kw = dict(minmod_maxiter=0)
    elif kind == "kh":
        x, dt, dh = kh_case(npd=2, seed=95, nxt=20)
        kw = dict(minmod_maxiter=0)
    else:
        x, dt, dh = blast_case(npd=2, seed=94, nxt=20, dual=False)
        dt *= 2.0
        kw = dict(minmod_maxiter=3)
    x = x[:4]
    ref = po.RefSolver(variant, prec).solve(x, dt, dh, limiter=limiter, **kw)
    res = po.restated_mhm(x, dt, dh, rsolver=rs, precision=prec, limiter=limiter, char=True, **kw)
    assert np.array_equal(res["out"], ref["out"])
    assert np.array_equal(res["flux"], ref["flux"])


def test_reference_mhm_rp_build_runs():
    """The MHM_RP build of the reference (Riemann-predictor half step, FLU_NXT = 22): finite output
    and FP32 within 1e-5 of FP64 on a smooth flow -- the oracle for a device MHM_RP."""
    _need_ref("mhmrp_plm_hllc", "fp64")
    r64 = po.RefSolver("mhmrp_plm_hllc", "fp64")
    assert r64.flu_nxt == 22
    x, dt, dh = kh_case(npd=1, seed=48, nxt=22)
    a = r64.solve(x, dt, dh)["out"]
    b = po.RefSolver("mhmrp_plm_hllc", "fp32").solve(x, dt, dh)["out"]
    assert np.all(np.isfinite(a))
    rms = np.sqrt((a ** 2).mean(axis=(0, 2, 3, 4), keepdims=True))
    rms = np.maximum(rms, 1e-2 * rms.max())
    assert np.max(np.abs(b - a) / (np.abs(a) + rms)) < 1e-5


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("kind", ["lognormal", "kh", "blast"])
def test_restated_mhm_rp_matches_reference_bit_for_bit(kind, prec):
    """The restated MHM_RP scheme (Riemann-predictor half step, then PLM without the Hancock
    predictor) against the reference built with FLU_SCHEME = MHM_RP."""
    _need_ref("mhmrp_plm_hllc", prec)
    if kind == "lognormal":
        x, dt, dh = lognormal_case(npd=2, seed=90, nxt=22)
        kw = {}
    elif kind == "kh":
        x, dt, dh = kh_case(npd=2, seed=91, nxt=22)
        kw = dict(limiter="vl_gminmod")
    else:
        x, dt, dh = blast_case(npd=2, seed=92, nxt=22, dual=False)
        dt *= 2.0
        kw = dict(minmod_maxiter=3)
    x = x[:4]
    ref = po.RefSolver("mhmrp_plm_hllc", prec).solve(x, dt, dh, **kw)
    res = po.restated_mhm(x, dt, dh, scheme="mhm_rp", precision=prec, **kw)
    assert np.array_equal(res["out"], ref["out"])
    assert np.array_equal(res["flux"], ref["flux"])


def _with_passive(x, dual, seed, npass=2):
    """Append npass passive scalars (positive fractions of the density) after the fluid variables
    and before the dual-energy field, the reference's order (include/Macro.h:302-305)."""
    rng = np.random.default_rng(seed)
    rho = x[:, 0]
    p = np.stack([rho * (0.2 + 0.6 * rng.random(rho.shape)) for _ in range(npass)], axis=1)
    return np.concatenate([x[:, :5], p, x[:, 5:6]], axis=1) if dual else np.concatenate([x, p], axis=1)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("dual", [False, True])
@pytest.mark.parametrize("kind", ["lognormal", "kh", "blast"])
def test_restated_passive_scalars_match_reference_bit_for_bit(kind, dual, prec):
    """Two user passive scalars (NCOMP_PASSIVE_USER = 2), with and without the dual-energy field
    after them: reconstructed as densities, upwinded with the mass flux, floored only where
    PassiveFloor says so (the dual-energy field)."""
    variant = "mhm_plm_hllc_p2" + ("_de" if dual else "")
    _need_ref(variant, prec)
    if kind == "lognormal":
        x, dt, dh = lognormal_case(npd=2, seed=70, dual=dual)
        kw = {}
    elif kind == "kh":
        x, dt, dh = kh_case(npd=2, seed=71, nxt=20, dual=dual)
        kw = dict(limiter="vl_gminmod")
    else:
        x, dt, dh = blast_case(npd=2, seed=72, nxt=20, dual=dual)
        dt *= 2.0
        kw = dict(minmod_maxiter=3)
    ref = po.RefSolver(variant, prec)
    x = _with_passive(x[:4], dual, 3).astype(ref.dtype)
    r = ref.solve(x, dt, dh, **kw)
    res = po.restated_mhm(x, dt, dh, dual=dual, npass=2, precision=prec, **kw)
    assert np.array_equal(res["out"], r["out"])
    assert np.array_equal(res["flux"], r["flux"])
    if dual:
        assert np.array_equal(res["de"], r["de"])
