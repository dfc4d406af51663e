"""Test infrastructure only: Python bindings of the two CPU checkers.

* ``RefSolver``  — GAMER's own ``CPU_FluidSolver`` (src/Fluid/CPU_FluidSolver.cpp:210) compiled,
  unmodified, from the reference sources by ``oracle/build_ref.sh`` into ``oracle/_ref/``; one
  library per compile-time variant.
* ``restated_mhm`` — the plain-C restatement ``oracle/gamer_oracle.c`` (built by ``make -C oracle``).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import this
module.  The product never does.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
BUILD_DIR = os.path.join(HERE, "_build")

# include/Typedef.h:184-194
LR_LIMITER = {"vanleer": 1, "gminmod": 2, "albada": 3, "vl_gminmod": 4, "central": 6}
# include/Macro.h solver ids
RSOLVER_ID = {"exact": 1, "roe": 2, "hlle": 3, "hllc": 4, "hlld": 5}
LR_ID = {"plm": 1, "ppm": 2}

_c_void_p = ctypes.c_void_p


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_c_void_p)


def ref_variant_name(scheme: str, lr: str, rsolver: str, mhd: bool = False, dual: bool = False,
                     char: bool = False) -> str:
    name = f"{scheme}_{lr}_{rsolver}"
    if dual:
        name += "_de"
    if char:
        name += "_char"
    if mhd:
        name += "_mhd"
    return name


def ref_available(variant: str, precision: str = "fp32") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libgref_{variant}_{precision}.so"))


# OPT__1ST_FLUX_CORR and OPT__1ST_FLUX_CORR_SCHEME (include/Typedef.h:461-474)
FIRST_FLUX_CORR = {"none": 0, "3d": 1, "3d1d": 2}
RSOLVER_1ST = {"roe": 1, "hllc": 2, "hlle": 3, "hlld": 4}
# patch_t::electric[s] of the 18 sides packed per patch: faces [2][7*8] then edges [8]
ELE_PER_PATCH = 6 * 2 * 7 * 8 + 12 * 8


class RefSolver:
    """One compile-time variant of the reference CPU solver (e.g. ``mhm_plm_hllc`` / ``fp64``)."""

    _cache: dict = {}

    def __init__(self, variant: str, precision: str = "fp32"):
        path = os.path.join(REF_DIR, f"libgref_{variant}_{precision}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference tree exists")
        key = path
        if key not in RefSolver._cache:
            lib = ctypes.CDLL(path)
            lib.gref_solve.restype = ctypes.c_int
            lib.gref_solve.argtypes = [_c_void_p] * 5 + [_c_void_p, _c_void_p] + [
                ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                ctypes.c_double, ctypes.c_double, ctypes.c_int]
            if hasattr(lib, "gref_set_options"):
                lib.gref_set_options.restype = ctypes.c_int
                lib.gref_set_options.argtypes = [ctypes.c_int, ctypes.c_long, ctypes.c_int, _c_void_p,
                                                 ctypes.c_int, _c_void_p, ctypes.c_int, ctypes.c_double]
            lib.gref_dt.restype = ctypes.c_int
            lib.gref_dt.argtypes = [_c_void_p] * 3 + [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                     ctypes.c_double, ctypes.c_double, ctypes.c_int]
            if hasattr(lib, "gref_correct_unphysical"):
                lib.gref_correct_unphysical.restype = ctypes.c_int
                lib.gref_correct_unphysical.argtypes = [_c_void_p] * 4 + [
                    ctypes.c_int, ctypes.c_double, ctypes.c_double] + [ctypes.c_int] * 6 + [
                    ctypes.c_double] * 5 + [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_long)]
            if hasattr(lib, "gref_correct_unphysical_mhd"):
                lib.gref_correct_unphysical_mhd.restype = ctypes.c_int
                lib.gref_correct_unphysical_mhd.argtypes = [_c_void_p] * 5 + [
                    ctypes.c_int, ctypes.c_double, ctypes.c_double] + [ctypes.c_int] * 6 + [
                    ctypes.c_double] * 4 + [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_long)]
            if hasattr(lib, "gref_fixup_flux_mhd"):
                lib.gref_fixup_flux_mhd.restype = ctypes.c_int
                lib.gref_fixup_flux_mhd.argtypes = [_c_void_p] * 4 + [ctypes.c_int, ctypes.c_double, ctypes.c_long] + [
                    ctypes.c_double] * 4 + [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
            if hasattr(lib, "gref_fixup_electric"):
                lib.gref_fixup_electric.restype = ctypes.c_int
                lib.gref_fixup_electric.argtypes = [_c_void_p] * 5 + [ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                                                       ctypes.POINTER(ctypes.c_double)]
            if hasattr(lib, "gref_interpolate"):
                lib.gref_interpolate.restype = ctypes.c_int
                lib.gref_interpolate.argtypes = [_c_void_p, _c_void_p] + [_c_void_p] * 5 + [
                    ctypes.c_int, ctypes.c_int, _c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                    ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int]
            if hasattr(lib, "gref_fixup_flux"):
                lib.gref_fixup_flux.restype = ctypes.c_int
                lib.gref_fixup_flux.argtypes = [_c_void_p] * 4 + [ctypes.c_int, ctypes.c_double, ctypes.c_long] + [
                    ctypes.c_double] * 4 + [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
            RefSolver._cache[key] = lib
        self.lib = RefSolver._cache[key]
        info = (ctypes.c_int * 12)()
        self.lib.gref_info(info)
        self.flu_nxt, self.ncomp, self.real_size, self.mhd = info[0], info[1], info[2], bool(info[3])
        self.ghost = info[8]
        self.dtype = np.float64 if self.real_size == 8 else np.float32
        self.ncomp_ele = info[11]

    def solve(self, flu_in, dt, dh, *, mag_in=None, store_flux=True, store_ele=False,
              limiter="gminmod", minmod_coeff=1.5, minmod_maxiter=0, min_dens=0.0, min_pres=0.0,
              min_eint=0.0, de_switch=2e-2, gamma=5.0 / 3.0, nthreads=0, passive_floor=None,
              norm_idx=(), frac_idx=(), jeans=False, jeans_coeff=0.0):
        """Run CPU_FluidSolver on ``flu_in[npg][ncomp][N][N][N]``.  If ``N`` exceeds this variant's
        FLU_NXT the central window is used (the scheme never reads the outer layers).
        ``passive_floor`` (None: the dual-energy field, GAMER's registration), ``norm_idx`` /
        ``frac_idx`` (NormPassive / FracPassive; empty = off) and ``jeans`` / ``jeans_coeff``
        (JeansMinPres) are the remaining run-time options of CPU_FluidSolver."""
        flu_in = np.asarray(flu_in)
        npg, nc, n = flu_in.shape[0], flu_in.shape[1], flu_in.shape[2]
        assert nc == self.ncomp, (nc, self.ncomp)
        if n != self.flu_nxt:
            s = (n - self.flu_nxt) // 2
            assert s >= 0 and 2 * s + self.flu_nxt == n
            flu_in = flu_in[:, :, s:s + self.flu_nxt, s:s + self.flu_nxt, s:s + self.flu_nxt]
        flu_in = np.ascontiguousarray(flu_in, dtype=self.dtype)
        out = np.zeros((npg, nc, 16, 16, 16), self.dtype)
        flux = np.zeros((npg, 9, nc, 16, 16), self.dtype) if store_flux else None
        de = np.zeros((npg, 16, 16, 16), np.int8)
        mag_out = ele = None
        if self.mhd:
            assert mag_in is not None
            mag_in = np.ascontiguousarray(mag_in, dtype=self.dtype)
            mag_out = np.zeros((npg, 3, 17 * 16 * 16), self.dtype)
            ele = np.zeros((npg, 9, self.ncomp_ele, 17 * 16), self.dtype) if store_ele else None
        nidx = np.ascontiguousarray(list(norm_idx) or [0], dtype=np.int32)
        fidx = np.ascontiguousarray(list(frac_idx) or [0], dtype=np.int32)
        if hasattr(self.lib, "gref_set_options"):
            assert self.lib.gref_set_options(int(passive_floor is None), int(passive_floor or 0), len(norm_idx),
                                             _ptr(nidx), len(frac_idx), _ptr(fidx), int(jeans), jeans_coeff) == 0
        elif passive_floor is not None or norm_idx or frac_idx or jeans:
            raise RuntimeError("this reference build has no run-time options: rebuild oracle/_ref")
        rc = self.lib.gref_solve(_ptr(flu_in), _ptr(out), _ptr(mag_in), _ptr(mag_out), _ptr(de), _ptr(flux),
                                 _ptr(ele), npg, dt, dh, int(store_flux), int(store_ele),
                                 LR_LIMITER[limiter], minmod_coeff, minmod_maxiter, min_dens, min_pres,
                                 min_eint, de_switch, gamma, nthreads)
        assert rc == 0
        res = {"out": out, "flux": flux, "de": de}
        if self.mhd:
            res["mag_out"] = mag_out
            res["ele"] = ele
        return res


    def correct_unphysical(self, flu_in, flu_out, dt, dh, *, de=None, flux=None, corr="3d", scheme="hlle",
                           fixup_flux=True, last_resort_floor=True, auto_reduce_dt_continue=False,
                           check_pres_after_flu=False, min_dens=0.0, min_pres=0.0, min_eint=0.0,
                           de_switch=2e-2, gamma=5.0 / 3.0, outdir=".", nthreads=0):
        """CorrectUnphysical() of src/Fluid/Flu_Close.cpp:542 on copies of the solver outputs.
        Returns {"rc", "ncorr", "out", "de", "flux"}: rc 0 all cells physical afterwards, 1 a cell
        failed under AUTO_REDUCE_DT (the step would be redone with a smaller dt), 2 the reference
        would have aborted."""
        flu_in = np.asarray(flu_in)
        n = flu_in.shape[2]
        if n != self.flu_nxt:
            s = (n - self.flu_nxt) // 2
            flu_in = flu_in[:, :, s:s + self.flu_nxt, s:s + self.flu_nxt, s:s + self.flu_nxt]
        flu_in = np.ascontiguousarray(flu_in, dtype=self.dtype)
        out = np.array(flu_out, dtype=self.dtype, copy=True, order="C")
        npg = out.shape[0]
        de = (np.array(de, dtype=np.int8, copy=True, order="C") if de is not None
              else np.zeros((npg, 16, 16, 16), np.int8))
        flux = (np.array(flux, dtype=self.dtype, copy=True, order="C") if flux is not None
                else np.zeros((npg, 9, self.ncomp, 16, 16), self.dtype))
        ncorr = ctypes.c_long(0)
        rc = self.lib.gref_correct_unphysical(
            _ptr(flu_in), _ptr(out), _ptr(de), _ptr(flux), npg, dt, dh, FIRST_FLUX_CORR[corr],
            RSOLVER_1ST[scheme], int(fixup_flux), int(last_resort_floor), int(auto_reduce_dt_continue),
            int(check_pres_after_flu), min_dens, min_pres, min_eint, de_switch, gamma,
            os.fsencode(outdir), nthreads, ctypes.byref(ncorr))
        return {"rc": rc, "ncorr": ncorr.value, "out": out, "de": de, "flux": flux}

    def correct_unphysical_mhd(self, flu_in, mag_in, flu_out, mag_out, dt, dh, *, flux=None, corr="3d",
                               scheme="hlle", fixup_flux=True, last_resort_floor=True,
                               auto_reduce_dt_continue=False, check_pres_after_flu=False, min_dens=0.0,
                               min_pres=0.0, min_eint=0.0, gamma=5.0 / 3.0, outdir=".", nthreads=0):
        """The MHD branch of CorrectUnphysical() (src/Fluid/Flu_Close.cpp:542-1200) on copies of the
        CTU+MHD solver outputs: mag_in [NPG][3][(FLU_NXT+1)*FLU_NXT^2] and mag_out
        [NPG][3][17*16*16] are the face-centred B field of the solver's input and output.  Returns
        {"rc", "ncorr", "out", "flux"} as correct_unphysical."""
        flu_in = np.ascontiguousarray(flu_in, dtype=self.dtype)
        mag_in = np.ascontiguousarray(mag_in, dtype=self.dtype)
        mag_out = np.ascontiguousarray(mag_out, dtype=self.dtype)
        out = np.array(flu_out, dtype=self.dtype, copy=True, order="C")
        npg = out.shape[0]
        flux = (np.array(flux, dtype=self.dtype, copy=True, order="C") if flux is not None
                else np.zeros((npg, 9, self.ncomp, 16, 16), self.dtype))
        ncorr = ctypes.c_long(0)
        rc = self.lib.gref_correct_unphysical_mhd(
            _ptr(flu_in), _ptr(mag_in), _ptr(out), _ptr(mag_out), _ptr(flux), npg, dt, dh,
            FIRST_FLUX_CORR[corr], RSOLVER_1ST[scheme], int(fixup_flux), int(last_resort_floor),
            int(auto_reduce_dt_continue), int(check_pres_after_flu), min_dens, min_pres, min_eint, gamma,
            os.fsencode(outdir), nthreads, ctypes.byref(ncorr))
        return {"rc": rc, "ncorr": ncorr.value, "out": out, "flux": flux}

    def fixup_flux_mhd(self, fluid, magnetic, flux, has_flux, dh, *, tvar=None, min_dens=0.0, min_pres=0.0,
                       min_eint=0.0, gamma=5.0 / 3.0, nthreads=0, timing=None):
        """Flu_FixUp_Flux() of an MHD build: as fixup_flux, with the patches' face-centred B field
        magnetic [NP][3][9*8*8] for the magnetic energy."""
        out = np.array(fluid, dtype=self.dtype, copy=True, order="C")
        mag = np.ascontiguousarray(magnetic, dtype=self.dtype)
        flux = np.ascontiguousarray(flux, dtype=self.dtype)
        hf = np.ascontiguousarray(has_flux, dtype=np.uint8)
        if tvar is None:
            tvar = (1 << self.ncomp) - 1
        sec = ctypes.c_double(0.0)
        assert self.lib.gref_fixup_flux_mhd(_ptr(out), _ptr(mag), _ptr(flux), _ptr(hf), out.shape[0], dh, tvar,
                                            min_dens, min_pres, min_eint, gamma, nthreads, ctypes.byref(sec)) == 0
        if timing is not None:
            timing.append(sec.value)
        return out

    def fixup_electric(self, magnetic, electric, electric_bitrep, has_ele, sib_leaf, dh, *, nthreads=0,
                       timing=None):
        """MHD_FixUp_Electric() (src/Model_Hydro/MHD_FixUp_Electric.cpp:22) on a batch of patches:
        magnetic [NP][3][9*8*8], electric / electric_bitrep [NP][ELE_PER_PATCH] (the 18 sides
        packed), has_ele [NP][18], sib_leaf [NP][6].  Returns (magnetic, electric, electric_bitrep)
        after the call."""
        mag = np.array(magnetic, dtype=self.dtype, copy=True, order="C")
        ele = np.array(electric, dtype=self.dtype, copy=True, order="C")
        elb = np.array(electric_bitrep, dtype=self.dtype, copy=True, order="C")
        he = np.ascontiguousarray(has_ele, dtype=np.uint8)
        sl = np.ascontiguousarray(sib_leaf, dtype=np.uint8)
        sec = ctypes.c_double(0.0)
        assert self.lib.gref_fixup_electric(_ptr(mag), _ptr(ele), _ptr(elb), _ptr(he), _ptr(sl), mag.shape[0], dh,
                                            nthreads, ctypes.byref(sec)) == 0
        if timing is not None:
            timing.append(sec.value)
        return mag, ele, elb

    def fixup_flux(self, fluid, flux, has_flux, dh, *, de=None, tvar=None, min_dens=0.0, min_pres=0.0,
                   min_eint=0.0, gamma=5.0 / 3.0, nthreads=0, timing=None):
        """Flu_FixUp_Flux() of src/Fluid/Flu_FixUp_Flux.cpp:23 on a batch of patches of one level:
        fluid [NP][NCOMP][8][8][8] (a corrected copy is returned), flux [NP][6][NCOMP][8][8] the
        flux differences, has_flux [NP][6] which faces carry one, de [NP][8][8][8] the dual-energy
        status (dual-energy builds); tvar = bit mask of the corrected variables (all by default)."""
        out = np.array(fluid, dtype=self.dtype, copy=True, order="C")
        npatch = out.shape[0]
        flux = np.ascontiguousarray(flux, dtype=self.dtype)
        hf = np.ascontiguousarray(has_flux, dtype=np.uint8)
        if de is not None:
            de = np.ascontiguousarray(de, dtype=np.int8)
        if tvar is None:
            tvar = (1 << self.ncomp) - 1
        sec = ctypes.c_double(0.0)
        assert self.lib.gref_fixup_flux(_ptr(out), _ptr(de), _ptr(flux), _ptr(hf), npatch, dh, tvar, min_dens,
                                        min_pres, min_eint, gamma, nthreads, ctypes.byref(sec)) == 0
        if timing is not None:
            timing.append(sec.value)     # seconds spent in Flu_FixUp_Flux itself
        return out

    def dt(self, flu, dh, *, mag=None, safety=0.5, min_pres=0.0, gamma=5.0 / 3.0, nthreads=0):
        """CPU_dtSolver_HydroCFL on patches: flu [8*NPG][5][8^3] (+ mag [8*NPG][3][9*8*8] for MHD);
        returns dt [8*NPG]."""
        flu = np.ascontiguousarray(flu, dtype=self.dtype)
        npatch = flu.shape[0]
        assert npatch % 8 == 0 and flu.shape[1] == 5
        if self.mhd:
            assert mag is not None
            mag = np.ascontiguousarray(mag, dtype=self.dtype)
        dt = np.zeros(npatch, self.dtype)
        assert self.lib.gref_dt(_ptr(flu), _ptr(mag), _ptr(dt), npatch // 8, dh, safety, min_pres, gamma,
                                nthreads) == 0
        return dt


_restated = None


def _restated_lib():
    global _restated
    if _restated is None:
        path = os.path.join(BUILD_DIR, "libgamer_oracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        lib = ctypes.CDLL(path)
        for name in ("gor32_solve_mhm", "gor64_solve_mhm"):
            f = getattr(lib, name)
            f.restype = ctypes.c_int
            f.argtypes = [_c_void_p] * 4 + [ctypes.c_int] * 6 + [ctypes.c_double, ctypes.c_int] + \
                [ctypes.c_double] * 7 + [ctypes.c_int]
        for name in ("gor32_solve_mhm_passive", "gor64_solve_mhm_passive"):
            f = getattr(lib, name)
            f.restype = ctypes.c_int
            f.argtypes = [_c_void_p] * 4 + [ctypes.c_int] * 7 + [ctypes.c_double, ctypes.c_int] + \
                [ctypes.c_double] * 7
        for name in ("gor32_solve_mhm_rp", "gor64_solve_mhm_rp"):
            f = getattr(lib, name)
            f.restype = ctypes.c_int
            f.argtypes = [_c_void_p] * 4 + [ctypes.c_int] * 5 + [ctypes.c_double, ctypes.c_int] + \
                [ctypes.c_double] * 7
        _restated = lib
    return _restated


def restated_mhm(flu_in, dt, dh, *, lr="plm", rsolver="hllc", dual=False, limiter="gminmod",
                 minmod_coeff=1.5, minmod_maxiter=0, min_dens=0.0, min_pres=0.0, min_eint=0.0,
                 de_switch=2e-2, gamma=5.0 / 3.0, precision="fp32", store_flux=True, char=False,
                 scheme="mhm", npass=0):
    """The C restatement of the MHM solver (oracle/gamer_oracle.c); char = CHAR_RECONSTRUCTION;
    scheme "mhm_rp" = the MHM_RP scheme (PLM); npass = user passive scalars (NCOMP_PASSIVE_USER),
    stored after the 5 fluid variables and before the dual-energy field."""
    lib = _restated_lib()
    dtype = np.float64 if precision == "fp64" else np.float32
    flu_in = np.ascontiguousarray(flu_in, dtype=dtype)
    npg, nc, n = flu_in.shape[0], flu_in.shape[1], flu_in.shape[2]
    out = np.zeros((npg, nc, 16, 16, 16), dtype)
    flux = np.zeros((npg, 9, nc, 16, 16), dtype) if store_flux else None
    de = np.zeros((npg, 16, 16, 16), np.int8)
    if npass:
        fn = lib.gor64_solve_mhm_passive if precision == "fp64" else lib.gor32_solve_mhm_passive
        rc = fn(_ptr(flu_in), _ptr(out), _ptr(flux), _ptr(de), npg, n, LR_ID[lr], RSOLVER_ID[rsolver], int(dual),
                npass, LR_LIMITER[limiter], minmod_coeff, minmod_maxiter, dt, dh, min_dens, min_pres, min_eint,
                de_switch, gamma)
        if rc != 0:
            raise ValueError(f"restated oracle rejected the input (rc={rc})")
        return {"out": out, "flux": flux, "de": de}
    if scheme == "mhm_rp":
        fn = lib.gor64_solve_mhm_rp if precision == "fp64" else lib.gor32_solve_mhm_rp
        rc = fn(_ptr(flu_in), _ptr(out), _ptr(flux), _ptr(de), npg, n, RSOLVER_ID[rsolver], int(dual),
                LR_LIMITER[limiter], minmod_coeff, minmod_maxiter, dt, dh, min_dens, min_pres, min_eint,
                de_switch, gamma)
        if rc != 0:
            raise ValueError(f"restated oracle rejected the input (rc={rc})")
        return {"out": out, "flux": flux, "de": de}
    fn = lib.gor64_solve_mhm if precision == "fp64" else lib.gor32_solve_mhm
    rc = fn(_ptr(flu_in), _ptr(out), _ptr(flux), _ptr(de), npg, n, LR_ID[lr], RSOLVER_ID[rsolver], int(dual),
            LR_LIMITER[limiter], minmod_coeff, minmod_maxiter, dt, dh, min_dens, min_pres, min_eint,
            de_switch, gamma, int(char))
    if rc != 0:
        raise ValueError(f"restated oracle rejected the input (rc={rc})")
    return {"out": out, "flux": flux, "de": de}


INT_SCHEME = {"minmod3d": 1, "minmod1d": 2, "vanleer": 3, "cquad": 4, "quad": 5, "cquar": 6, "quar": 7}


def ref_interpolate(cdata, fdata, scheme, cstart, crange, fstart=(0, 0, 0), monotonic=True, mono_coeff=2.0,
                    opp_sign_0th_order=False, iterate=False, int_prim=True, mono_max_iter=10, gamma=5.0 / 3.0,
                    min_pres=0.0):
    """The reference's Interpolate() on every region of a batch (numpy arrays, the layout of
    gamer_b200.fluid.interpolate_device); fdata is written in place.  Returns the reference's status:
    0, or 2 where Interpolate_Iterate gave up (the reference aborts the run there)."""
    precision = "fp64" if cdata.dtype == np.float64 else "fp32"
    lib = RefSolver("mhm_plm_hllc", precision).lib
    nb, nc = cdata.shape[0], cdata.shape[1]
    mono = [bool(monotonic)] * nc if isinstance(monotonic, bool) else list(monotonic)

    def ai(v):
        return np.ascontiguousarray(list(v), dtype=np.int32)

    cs, fs = ai([cdata.shape[4], cdata.shape[3], cdata.shape[2]]), ai([fdata.shape[4], fdata.shape[3], fdata.shape[2]])
    c0, cr, f0, mo = ai(cstart), ai(crange), ai(fstart), ai([int(m) for m in mono])
    cdata = np.ascontiguousarray(cdata)
    assert fdata.flags["C_CONTIGUOUS"] and fdata.dtype == cdata.dtype
    return lib.gref_interpolate(_ptr(cdata), _ptr(fdata), _ptr(cs), _ptr(c0), _ptr(cr), _ptr(fs), _ptr(f0), nc,
                                INT_SCHEME[scheme], _ptr(mo), int(opp_sign_0th_order), int(iterate), int(int_prim),
                                mono_coeff, int(mono_max_iter), gamma, min_pres, nb)


class RefGpuSolver:
    """The reference's own GPU kernel CUFLU_FluidSolver_MHM, built unmodified for sm_100a by
    ``oracle/build_ref_gpu.sh`` (oracle/ref_gpu.cu adds the launch of CUAPI_Asyn_FluidSolver and the
    reference's global-memory scratch).  Works on torch CUDA tensors; the bench times it beside this
    repository's solver, and a GPU test checks it against the reference CPU solver."""

    _cache: dict = {}

    def __init__(self, variant: str, precision: str = "fp32"):
        path = os.path.join(REF_DIR, f"libgrefgpu_{variant}_{precision}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run oracle/build_ref_gpu.sh where the reference tree exists")
        if path not in RefGpuSolver._cache:
            lib = ctypes.CDLL(path)
            lib.grefgpu_info.argtypes = [ctypes.POINTER(ctypes.c_long)]
            lib.grefgpu_solve.restype = ctypes.c_int
            lib.grefgpu_solve.argtypes = [_c_void_p] * 4 + [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                            ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                                            ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                            ctypes.c_double, ctypes.c_double, _c_void_p]
            RefGpuSolver._cache[path] = lib
        self.lib = RefGpuSolver._cache[path]
        info = (ctypes.c_long * 5)()
        self.lib.grefgpu_info(info)
        self.flu_nxt, self.ncomp, self.real_size, self.block, self.scratch_bytes_per_pg = (int(v) for v in info)

    def solve_device(self, t_in, t_out, dt, dh, t_flux=None, *, limiter="gminmod", minmod_coeff=1.5,
                     minmod_maxiter=0, min_dens=0.0, min_pres=0.0, min_eint=0.0, de_switch=2e-2,
                     gamma=5.0 / 3.0, stream=None):
        """One launch over the patch groups of t_in [npg][NCOMP][FLU_NXT^3] (contiguous CUDA tensors
        of the build's real type); asynchronous on ``stream`` (torch stream, default: current)."""
        import torch
        npg = t_in.shape[0]
        esz = t_in.element_size()
        assert esz == self.real_size and t_out.element_size() == esz
        assert tuple(t_in.shape) == (npg, self.ncomp, self.flu_nxt, self.flu_nxt, self.flu_nxt)
        assert tuple(t_out.shape) == (npg, self.ncomp, 16, 16, 16)
        assert t_in.is_contiguous() and t_out.is_contiguous()
        if t_flux is not None:
            assert tuple(t_flux.shape) == (npg, 9, self.ncomp, 16, 16) and t_flux.is_contiguous()
        if stream is None:
            stream = torch.cuda.current_stream(t_in.device)
        rc = self.lib.grefgpu_solve(_c_void_p(t_in.data_ptr()), _c_void_p(t_out.data_ptr()),
                                    _c_void_p(t_flux.data_ptr()) if t_flux is not None else None, None, npg,
                                    dt, dh, int(t_flux is not None), LR_LIMITER[limiter], minmod_coeff,
                                    minmod_maxiter, min_dens, min_pres, min_eint, de_switch, gamma,
                                    _c_void_p(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError("reference GPU solver: scratch allocation or launch failed")
