"""CPU checks of the MHD close-consumer oracles (oracle/_ref libgref_ctu_plm_hlld_mhd_*: the reference's
MHD_FixUp_Electric, Flu_FixUp_Flux and CorrectUnphysical compiled under MHD).

* MHD_FixUp_Electric (src/Model_Hydro/MHD_FixUp_Electric.cpp:22) is restated here as a gather: every
  face-centred B component collects, in the reference's order (faces 0-5, then edges 6-17), the
  corrections of the sides that reach it.  That is the formulation of the device kernel
  (gamer_b200/csrc/ele_fixup.cu); the restatement must equal the reference's scatter bit for bit.
* The reference's MHD CorrectUnphysical repairs a magnetised flow advanced with 1.5 times the CFL
  step, cell by cell, and leaves the physical cells untouched.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "oracle"))
import pyoracle as po  # noqa: E402
from parity import mhd_case  # noqa: E402

VARIANT = "ctu_plm_hlld_mhd"
PS1, M1, EFACE, EDGE0 = 8, 7, 56, 672


def _need_ref(prec):
    if not po.ref_available(VARIANT, prec):
        pytest.skip(f"oracle/_ref/libgref_{VARIANT}_{prec}.so not built (needs the reference tree)")


def gather_fixup_electric(mag, ele, elb, has, sib, dh, dtype):
    """The gather form of MHD_FixUp_Electric, one B component at a time, every product rounded to
    dtype before it is added (the reference's CPU build has no FMA contraction)."""
    R = dtype
    idh = R(1.0 / dh)
    mag = mag.copy()
    E = (ele + elb).astype(R)
    shapes = {0: (8, 8, 9), 1: (8, 9, 8), 2: (9, 8, 8)}        # [k][j][i] of Bx, By, Bz
    for p in range(mag.shape[0]):
        h, s = has[p], sib[p]
        for c in range(3):
            B = mag[p, c].reshape(shapes[c])
            for k, j, i in np.ndindex(*shapes[c]):
                terms = []
                if c == 0:
                    terms += [(2 * L - 1, (2 + L) * 2 * EFACE + (i - 1) * PS1 + k) for L in range(2)
                              if h[2 + L] and j == M1 * L and 1 <= i < PS1]
                    terms += [(1 - 2 * L, (4 + L) * 2 * EFACE + EFACE + j * M1 + (i - 1)) for L in range(2)
                              if h[4 + L] and k == M1 * L and 1 <= i < PS1]
                    terms += [(2 * (q // 2) - 1, EDGE0 + q * PS1 + k) for q in range(4)
                              if h[6 + q] and i == PS1 * (q % 2) and j == M1 * (q // 2) and s[q % 2]]
                    terms += [(1 - 2 * (q % 2), EDGE0 + q * PS1 + j) for q in range(8, 12)
                              if h[6 + q] and i == PS1 * (q % 4 // 2) and k == M1 * (q % 2) and s[q % 4 // 2]]
                elif c == 1:
                    terms += [(1 - 2 * L, L * 2 * EFACE + EFACE + k * M1 + (j - 1)) for L in range(2)
                              if h[L] and i == M1 * L and 1 <= j < PS1]
                    terms += [(2 * L - 1, (4 + L) * 2 * EFACE + (j - 1) * PS1 + i) for L in range(2)
                              if h[4 + L] and k == M1 * L and 1 <= j < PS1]
                    terms += [(1 - 2 * (q % 2), EDGE0 + q * PS1 + k) for q in range(4)
                              if h[6 + q] and i == M1 * (q % 2) and j == PS1 * (q // 2) and s[2 + q // 2]]
                    terms += [(2 * (q % 4 // 2) - 1, EDGE0 + q * PS1 + i) for q in range(4, 8)
                              if h[6 + q] and j == PS1 * (q % 2) and k == M1 * (q % 4 // 2) and s[2 + q % 2]]
                else:
                    terms += [(2 * L - 1, L * 2 * EFACE + (k - 1) * PS1 + j) for L in range(2)
                              if h[L] and i == M1 * L and 1 <= k < PS1]
                    terms += [(1 - 2 * L, (2 + L) * 2 * EFACE + EFACE + i * M1 + (k - 1)) for L in range(2)
                              if h[2 + L] and j == M1 * L and 1 <= k < PS1]
                    terms += [(1 - 2 * (q % 2), EDGE0 + q * PS1 + i) for q in range(4, 8)
                              if h[6 + q] and j == M1 * (q % 2) and k == PS1 * (q % 4 // 2) and s[4 + q % 4 // 2]]
                    terms += [(2 * (q % 4 // 2) - 1, EDGE0 + q * PS1 + j) for q in range(8, 12)
                              if h[6 + q] and k == PS1 * (q % 2) and i == M1 * (q % 4 // 2) and s[4 + q % 2]]
                b = B[k, j, i]
                for sgn, e in terms:
                    b = R(b + R(R(sgn * idh) * E[p, e]))
                B[k, j, i] = b
    return mag


def electric_case(npatch, dtype, seed):
    rng = np.random.default_rng(seed)
    mag = rng.standard_normal((npatch, 3, 9 * 8 * 8)).astype(dtype)
    ele = (1e-2 * rng.standard_normal((npatch, po.ELE_PER_PATCH))).astype(dtype)
    elb = (1e-2 * rng.standard_normal((npatch, po.ELE_PER_PATCH))).astype(dtype)
    has = rng.integers(0, 2, (npatch, 18)).astype(np.uint8)
    sib = rng.integers(0, 2, (npatch, 6)).astype(np.uint8)
    has[0] = 1                      # one patch with every side on a coarse-fine boundary
    sib[0] = 1
    has[1] = 0                      # and one with none
    return mag, ele, elb, has, sib


def present(has):
    """[npatch][ELE_PER_PATCH] mask of the packed electric elements of the sides that exist."""
    m = np.zeros((has.shape[0], po.ELE_PER_PATCH), bool)
    for s in range(18):
        lo, n = (s * 2 * EFACE, 2 * EFACE) if s < 6 else (EDGE0 + (s - 6) * PS1, PS1)
        m[:, lo:lo + n] = has[:, s:s + 1].astype(bool)
    return m


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_gather_restatement_of_fixup_electric_equals_reference(prec):
    _need_ref(prec)
    dtype = np.float64 if prec == "fp64" else np.float32
    ref = po.RefSolver(VARIANT, prec)
    mag, ele, elb, has, sib = electric_case(6, dtype, seed=3)
    r_mag, r_ele, r_elb = ref.fixup_electric(mag, ele, elb, has, sib, 0.037)
    assert np.array_equal(gather_fixup_electric(mag, ele, elb, has, sib, 0.037, dtype), r_mag)
    # every side on a coarse-fine boundary changed some B of patch 0; patch 1 (no side) is untouched
    assert np.any(r_mag[0] != mag[0]) and np.array_equal(r_mag[1], mag[1])
    # the electric arrays of the sides that exist are zero afterwards
    pm = present(has)
    assert not np.any(r_ele[pm]) and not np.any(r_elb[pm])


def test_reference_mhd_correct_unphysical_repairs_failed_cells_only(tmp_path):
    _need_ref("fp64")
    ref = po.RefSolver(VARIANT, "fp64")
    x, b, dt, dh = mhd_case(npd=2, seed=5, cfl=1.5, mach=3.0, db=1.5)
    r = ref.solve(x, dt, dh, mag_in=b)
    c = ref.correct_unphysical_mhd(x, b, r["out"], r["mag_out"], dt, dh, flux=r["flux"], scheme="hlle",
                                   outdir=str(tmp_path))
    chg = np.any(c["out"] != r["out"], axis=1)
    assert c["rc"] == 0 and c["ncorr"] == chg.sum() > 100
    # the corrected cells have a positive density
    assert np.all(c["out"][:, 0][chg] > 0)
