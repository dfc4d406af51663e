"""Python front end of the B200 patch-group fluid solver (ctypes over the C ABI in
include/gamer_b200_fluid.h; the shared library is gamer_b200/lib/libgamer_b200_fluid.so).

``FluidSolver`` mirrors GAMER's solver call: ``CPU_FluidSolver`` (src/Fluid/CPU_FluidSolver.cpp:210)
for host (numpy) arrays and the kernel launch of ``CUAPI_Asyn_FluidSolver``
(src/GPU_API/CUAPI_Asyn_FluidSolver.cu:266) for device (torch CUDA) tensors, with the same array
shapes and the same run-time parameters (``dt, dh, StoreFlux, LR_Limiter, MinMod_Coeff,
MinMod_MaxIter, MinDens, MinPres, MinEint, DualEnergySwitch``).  Compile-time choices of the
reference (scheme, reconstruction, Riemann solver, precision, dual energy, FLU_NXT) are constructor
arguments.

There is no CPU fallback: if the library is missing, constructing a solver raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgamer_b200_fluid.so")

SCHEME = {"mhm": 3, "mhm_rp": 4, "ctu": 5}
LR = {"plm": 1, "ppm": 2}
RSOLVER = {"exact": 1, "roe": 2, "hlle": 3, "hllc": 4, "hlld": 5}
LIMITER = {"vanleer": 1, "gminmod": 2, "albada": 3, "vl_gminmod": 4, "central": 6}
PRECISION = {"fp32": 0, "mixed": 1, "fp64": 2}
STATUS_TMA_TIMEOUT = 1
STATUS_UNPHYSICAL = 2

_ERR = {0: "success", -1: "invalid argument", -2: "array not 16-byte aligned", -3: "CUDA runtime error",
        -4: "out of memory", -5: "configuration not supported"}


class FluidSolverError(RuntimeError):
    def __init__(self, code, where):
        super().__init__(f"{where}: {_ERR.get(code, 'unknown error')} (code {code})")
        self.code = code


class _Config(ctypes.Structure):
    _fields_ = [("scheme", ctypes.c_int), ("lr_scheme", ctypes.c_int), ("rsolver", ctypes.c_int),
                ("precision", ctypes.c_int), ("dual_energy", ctypes.c_int), ("flu_nxt", ctypes.c_int),
                ("gamma", ctypes.c_double), ("char_reconstruction", ctypes.c_int), ("npassive_user", ctypes.c_int)]


# NCOMP_PASSIVE_USER built into the MHM kernels, and the largest NCOMP_PASSIVE (+ the dual-energy field)
NPASSIVE_USER = 2
MAX_PASSIVE = 3


class _CloseParams(ctypes.Structure):
    _fields_ = [("first_flux_corr", ctypes.c_int), ("first_flux_scheme", ctypes.c_int),
                ("last_resort_floor", ctypes.c_int), ("auto_reduce_dt_continue", ctypes.c_int),
                ("check_pres_after_flu", ctypes.c_int)]


# OPT__1ST_FLUX_CORR and OPT__1ST_FLUX_CORR_SCHEME of the reference (include/Typedef.h:461-474)
FIRST_FLUX_CORR = {"none": 0, "3d": 1, "3d1d": 2}
RSOLVER_1ST = {"roe": 1, "hllc": 2, "hlle": 3, "hlld": 4}
# patch groups per chunk of the host-array entry point (its launches see batches of this size)
HOST_CHUNK = 256
# patch_t::electric[s] of the 18 sides of a patch, packed: faces [2][7*8], then edges [8]
ELE_PER_PATCH = 6 * 2 * 7 * 8 + 12 * 8


class _Params(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("dh", ctypes.c_double), ("store_flux", ctypes.c_int),
                ("store_electric", ctypes.c_int), ("lr_limiter", ctypes.c_int),
                ("minmod_coeff", ctypes.c_double), ("minmod_maxiter", ctypes.c_int),
                ("min_dens", ctypes.c_double), ("min_pres", ctypes.c_double), ("min_eint", ctypes.c_double),
                ("dual_energy_switch", ctypes.c_double), ("passive_floor", ctypes.c_longlong),
                ("norm_passive", ctypes.c_int), ("nnorm", ctypes.c_int), ("norm_idx", ctypes.c_int * 3),
                ("frac_passive", ctypes.c_int), ("nfrac", ctypes.c_int), ("frac_idx", ctypes.c_int * 3),
                ("jeans_min_pres", ctypes.c_int), ("jeans_min_pres_coeff", ctypes.c_double)]


class _InterpParams(ctypes.Structure):
    _fields_ = [("scheme", ctypes.c_int), ("precision", ctypes.c_int), ("ncomp", ctypes.c_int),
                ("csize", ctypes.c_int * 3), ("cstart", ctypes.c_int * 3), ("crange", ctypes.c_int * 3),
                ("fsize", ctypes.c_int * 3), ("fstart", ctypes.c_int * 3), ("monotonic", ctypes.c_uint),
                ("mono_coeff", ctypes.c_double), ("opp_sign_0th_order", ctypes.c_int), ("mode", ctypes.c_int),
                ("int_prim", ctypes.c_int), ("mono_max_iter", ctypes.c_int), ("gamma", ctypes.c_double),
                ("min_pres", ctypes.c_double), ("status", ctypes.c_void_p)]


# IntScheme_t of the reference (include/Typedef.h:171-180)
INT_SCHEME = {"minmod3d": 1, "minmod1d": 2, "vanleer": 3, "cquad": 4, "quad": 5, "cquar": 6, "quar": 7}
INTERP_FAILED = 1


# every symbol the header declares (checked by the CPU test suite)
EXPORTED = ["gb_fluid_create", "gb_fluid_destroy", "gb_fluid_solve_device", "gb_fluid_solve_host",
            "gb_fluid_solve_levels_device", "gb_fluid_get_status", "gb_fluid_host_alloc", "gb_fluid_host_free",
            "gb_fluid_set_block_size", "gb_fluid_get_block_size", "gb_fluid_array_bytes", "gb_fluid_strerror",
            "gb_fluid_version", "gb_fluid_graph_create_levels", "gb_fluid_graph_set_dt", "gb_fluid_graph_launch",
            "gb_fluid_graph_destroy", "gb_fluid_get_config", "gb_fluid_adjoint_workspace_bytes",
            "gb_fluid_adjoint_step_device", "gb_box_gather_device", "gb_box_scatter_device",
            "gb_box_gather_adjoint_device", "gb_box_scatter_adjoint_device", "gb_fluid_set_mhd_chunk",
            "gb_dt_cfl_device", "gb_dt_cfl_from_output_device", "gb_fluid_correct_unphysical_device",
            "gb_flux_fixup_device", "gb_fluid_solve_host_async", "gb_fluid_synchronize",
            "gb_ctu_mhd_solve_static", "gb_ctu_mhd_static_capacity", "gb_interpolate_device",
            "gb_assemble_windows_device", "gb_fluid_correct_unphysical_mhd_device", "gb_flux_fixup_mhd_device",
            "gb_mhd_fixup_electric_device", "gb_fluid_set_launch", "gb_fluid_get_launch"]

_lib = None


def load_library(path: str | None = None):
    """Load the CUDA library (raises if it was not built: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built: run `python -m gamer_b200.build`")
    lib = ctypes.CDLL(path)
    vp, i, ip = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)
    lib.gb_fluid_create.argtypes = [ctypes.POINTER(_Config), ctypes.POINTER(vp)]
    lib.gb_fluid_destroy.argtypes = [vp]
    lib.gb_fluid_solve_device.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, i, ctypes.POINTER(_Params), vp]
    lib.gb_fluid_solve_host.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i, ctypes.POINTER(_Params)]
    lib.gb_fluid_solve_host_async.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i, ctypes.POINTER(_Params), vp]
    lib.gb_fluid_synchronize.argtypes = [vp]
    lib.gb_ctu_mhd_solve_static.argtypes = [ctypes.POINTER(_Config), vp, vp, vp, vp, vp, vp, i,
                                            ctypes.POINTER(_Params), vp]
    lib.gb_ctu_mhd_static_capacity.argtypes = [i, ip]
    lib.gb_interpolate_device.argtypes = [ctypes.POINTER(_InterpParams), vp, vp, i, vp]
    lib.gb_assemble_windows_device.argtypes = [vp, vp, vp, vp, i, i, i, i, vp]
    lib.gb_fluid_solve_levels_device.argtypes = [vp, vp, vp, vp, vp, vp, i, ip, ctypes.POINTER(ctypes.c_double),
                                                 ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_Params), vp]
    lib.gb_fluid_get_status.argtypes = [vp, ip]
    lib.gb_fluid_host_alloc.argtypes = [ctypes.POINTER(vp), ctypes.c_ulonglong]
    lib.gb_fluid_host_free.argtypes = [vp]
    lib.gb_fluid_set_block_size.argtypes = [vp, i]
    lib.gb_fluid_get_block_size.argtypes = [vp, ip]
    lib.gb_fluid_set_mhd_chunk.argtypes = [vp, i]
    lib.gb_fluid_set_launch.argtypes = [vp, i, i, i]
    lib.gb_fluid_get_launch.argtypes = [vp, ip, ip, ip]
    d = ctypes.c_double
    lib.gb_dt_cfl_device.argtypes = [ctypes.POINTER(_Config), vp, vp, vp, i, d, d, d, vp]
    lib.gb_flux_fixup_device.argtypes = [ctypes.POINTER(_Config), vp, vp, vp, vp, i, ctypes.POINTER(_Params),
                                         ctypes.c_long, vp]
    lib.gb_fluid_correct_unphysical_device.argtypes = [vp, vp, vp, vp, vp, i, ctypes.POINTER(_Params),
                                                       ctypes.POINTER(_CloseParams), vp, vp]
    lib.gb_fluid_correct_unphysical_mhd_device.argtypes = [vp, vp, vp, vp, vp, vp, i, ctypes.POINTER(_Params),
                                                           ctypes.POINTER(_CloseParams), vp, vp]
    lib.gb_flux_fixup_mhd_device.argtypes = [ctypes.POINTER(_Config), vp, vp, vp, vp, i, ctypes.POINTER(_Params),
                                             ctypes.c_long, vp]
    lib.gb_mhd_fixup_electric_device.argtypes = [ctypes.POINTER(_Config), vp, vp, vp, vp, vp, i, d, vp]
    lib.gb_dt_cfl_from_output_device.argtypes = [ctypes.POINTER(_Config), vp, vp, vp, i, d, d, d, vp]
    lib.gb_fluid_array_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(ctypes.c_ulonglong),
                                         ctypes.POINTER(ctypes.c_ulonglong)]
    dp = ctypes.POINTER(ctypes.c_double)
    lib.gb_fluid_graph_create_levels.argtypes = [vp, vp, vp, vp, vp, vp, i, ip, dp, dp, ctypes.POINTER(_Params),
                                                 ctypes.POINTER(vp)]
    lib.gb_fluid_graph_set_dt.argtypes = [vp, dp]
    lib.gb_fluid_graph_launch.argtypes = [vp, vp]
    lib.gb_fluid_graph_destroy.argtypes = [vp]
    ull = ctypes.c_ulonglong
    lib.gb_fluid_get_config.argtypes = [vp, ctypes.POINTER(_Config)]
    lib.gb_fluid_adjoint_workspace_bytes.argtypes = [vp, i, ctypes.POINTER(ull)]
    lib.gb_fluid_adjoint_step_device.argtypes = [vp, vp, vp, vp, i, ctypes.POINTER(_Params), vp, ull, vp]
    lib.gb_box_gather_device.argtypes = [vp, vp, i, i, i, i, i, i, vp]
    lib.gb_box_scatter_device.argtypes = [vp, vp, i, i, i, i, i, vp]
    lib.gb_box_gather_adjoint_device.argtypes = [vp, vp, i, i, i, i, i, vp]
    lib.gb_box_scatter_adjoint_device.argtypes = [vp, vp, i, i, i, i, vp]
    lib.gb_fluid_strerror.restype = ctypes.c_char_p
    lib.gb_fluid_strerror.argtypes = [i]
    for name in EXPORTED:
        f = getattr(lib, name)
        if name != "gb_fluid_strerror":
            f.restype = ctypes.c_int
    _lib = lib
    return lib


def _check(rc, where):
    if rc != 0:
        raise FluidSolverError(rc, where)


def _dptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("device arrays must be contiguous CUDA tensors")
    return ctypes.c_void_p(t.data_ptr())


def _expect(t, shape, dtype, name):
    """Shape and dtype of an array handed to a device entry point: the C ABI takes bare pointers,
    so a mismatch here would become an out-of-bounds access on the device."""
    if t is None:
        return
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name}: shape {tuple(t.shape)}, expected {tuple(shape)}")
    if dtype is not None and t.dtype != dtype:
        raise ValueError(f"{name}: dtype {t.dtype}, expected {dtype}")


def _hptr(a):
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("host arrays must be C-contiguous")
    return a.ctypes.data_as(ctypes.c_void_p)


@dataclass
class SolverParams:
    """Run-time parameters of one solver call (names of CPU_FluidSolver's arguments).

    PassiveFloor: bit v floors variable v (v >= 5); None floors the dual-energy field, as GAMER
    registers it (src/Init/Init_Field.cpp).  NormIdx / FracIdx: passive-scalar indices (0 = first
    passive scalar) of NormPassive / FracPassive; an empty list turns the option off."""
    dt: float
    dh: float
    StoreFlux: bool = True
    LR_Limiter: str = "gminmod"
    MinMod_Coeff: float = 1.5
    MinMod_MaxIter: int = 0
    MinDens: float = 0.0
    MinPres: float = 0.0
    MinEint: float = 0.0
    DualEnergySwitch: float = 2e-2
    StoreElectric: bool = False
    PassiveFloor: int | None = None
    NormIdx: tuple = ()
    FracIdx: tuple = ()
    JeansMinPres: bool = False
    JeansMinPres_Coeff: float = 0.0

    def c(self, solver=None):
        """The C struct; ``solver`` (a FluidSolver) places the dual-energy bit of the default PassiveFloor."""
        floor = self.PassiveFloor
        if floor is None:
            floor = (1 << (solver.ncomp - 1)) if (solver is not None and solver.dual) else 0
        norm = list(self.NormIdx) + [0] * (MAX_PASSIVE - len(self.NormIdx))
        frac = list(self.FracIdx) + [0] * (MAX_PASSIVE - len(self.FracIdx))
        return _Params(self.dt, self.dh, int(self.StoreFlux), int(self.StoreElectric), LIMITER[self.LR_Limiter],
                       self.MinMod_Coeff,
                       self.MinMod_MaxIter, self.MinDens, self.MinPres, self.MinEint, self.DualEnergySwitch,
                       int(floor), int(len(self.NormIdx) > 0), len(self.NormIdx), (ctypes.c_int * 3)(*norm[:3]),
                       int(len(self.FracIdx) > 0), len(self.FracIdx), (ctypes.c_int * 3)(*frac[:3]),
                       int(self.JeansMinPres), self.JeansMinPres_Coeff)


class FluidSolver:
    """A configured solver (the reference's compile-time options are chosen here)."""

    def __init__(self, scheme="mhm", lr="plm", rsolver="hllc", precision="fp32", dual_energy=False,
                 flu_nxt=None, gamma=5.0 / 3.0, block_size=None, char_reconstruction=False, npassive_user=0):
        self.lib = load_library()
        if flu_nxt is None:
            # FLU_NXT of the scheme, 16 + 2 FLU_GHOST_SIZE (include/Macro.h:653-665): MHM and hydro CTU
            # 1 + LR ghost, CTU+MHD and MHM_RP 2 + LR ghost (LR ghost: PLM 1, PPM 2)
            if scheme == "mhm_rp":
                flu_nxt = 24 if lr == "ppm" else 22
            else:
                if scheme == "ctu" and rsolver == "hlld":
                    flu_nxt = 24 if lr == "ppm" else 22
                else:
                    flu_nxt = 22 if lr == "ppm" else 20
        self.cfg = _Config(SCHEME[scheme], LR[lr], RSOLVER[rsolver], PRECISION[precision],
                           1 if dual_energy else 0, flu_nxt, gamma, 1 if char_reconstruction else 0,
                           int(npassive_user))
        h = ctypes.c_void_p()
        _check(self.lib.gb_fluid_create(ctypes.byref(self.cfg), ctypes.byref(h)), "gb_fluid_create")
        self.h = h
        self.precision = precision
        self.dual = bool(dual_energy)
        self.npassive_user = int(npassive_user)
        # NCOMP_TOTAL: the fluid, the user passive scalars, the dual-energy field (last)
        self.ncomp = 5 + self.npassive_user + (1 if dual_energy else 0)
        self.flu_nxt = flu_nxt
        # HLLD is the MHD solver (CTU or MHM_RP): the calls take the magnetic arrays
        self.mhd = rsolver == "hlld"
        self.np_dtype = np.float64 if precision == "fp64" else np.float32
        # block_size="auto": the launch gamer_b200.autotune recorded for this GPU, configuration and
        # the batch size of each call (threads, CTAs per SM, register variant)
        self._auto = None
        self._applied = None
        if block_size == "auto":
            self._auto = (scheme, lr, rsolver, precision, bool(dual_energy), flu_nxt)
        elif block_size:
            self.set_block_size(block_size)

    def _apply_tuned(self, npg):
        """With block_size="auto", set the tuned launch for a batch of npg patch groups."""
        if self._auto is None:
            return
        try:
            import torch
            from gamer_b200 import autotune
            name = torch.cuda.get_device_name(torch.cuda.current_device())
            t = autotune.lookup_launch(name, *self._auto, npg=npg)
        except Exception:
            t = None
        t = t or (0, 0, 0)
        if t != self._applied:
            self.set_launch(*t)
            self._applied = t

    @property
    def torch_dtype(self):
        import torch
        return torch.float64 if self.precision == "fp64" else torch.float32

    def close(self):
        if getattr(self, "h", None):
            self.lib.gb_fluid_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_block_size(self, threads):
        _check(self.lib.gb_fluid_set_block_size(self.h, int(threads)), "gb_fluid_set_block_size")

    def set_launch(self, threads=0, ctas_per_sm=0, max_registers=0):
        """gb_fluid_set_launch: threads per CTA, a cap on CTAs per SM, the register variant (0 each:
        the defaults)."""
        _check(self.lib.gb_fluid_set_launch(self.h, int(threads), int(ctas_per_sm), int(max_registers)),
               "gb_fluid_set_launch")

    def launch(self):
        """(threads, ctas_per_sm, max_registers) of the next MHM launch."""
        v = [ctypes.c_int() for _ in range(3)]
        _check(self.lib.gb_fluid_get_launch(self.h, *(ctypes.byref(x) for x in v)), "gb_fluid_get_launch")
        return tuple(x.value for x in v)

    def block_size(self):
        t = ctypes.c_int()
        _check(self.lib.gb_fluid_get_block_size(self.h, ctypes.byref(t)), "gb_fluid_get_block_size")
        return t.value

    def status(self):
        """Read and clear the device status word (bits STATUS_*)."""
        s = ctypes.c_int()
        _check(self.lib.gb_fluid_get_status(self.h, ctypes.byref(s)), "gb_fluid_get_status")
        return s.value

    # -- device arrays (torch CUDA tensors) ----------------------------------------------------
    def dt_cfl(self, flu, dh, mag=None, safety=0.5, min_pres=0.0, from_output=False, dt_out=None, stream=None):
        """CFL time step per patch (CUFLU_dtSolver_HydroCFL).  ``flu``: GAMER's dt arrays
        [npatch][5][8^3] (``mag`` [npatch][3][9*8*8] with MHD) or, with ``from_output``, this solver's
        outputs [npg][NCOMP][16^3] (``mag`` [npg][3][17*16*16]); returns dt [npatch] / [8*npg]
        (torch CUDA tensors)."""
        import torch
        if stream is None:
            stream = torch.cuda.current_stream(flu.device)
        n = flu.shape[0] * (8 if from_output else 1)
        if dt_out is None:
            dt_out = torch.empty(n, dtype=flu.dtype, device=flu.device)
        fn = self.lib.gb_dt_cfl_from_output_device if from_output else self.lib.gb_dt_cfl_device
        rc = fn(ctypes.byref(self.cfg), _dptr(flu), _dptr(mag), _dptr(dt_out), flu.shape[0], dh, safety, min_pres,
                ctypes.c_void_p(stream.cuda_stream))
        _check(rc, fn.__name__)
        return dt_out

    def set_mhd_chunk(self, npg):
        _check(self.lib.gb_fluid_set_mhd_chunk(self.h, int(npg)), "gb_fluid_set_mhd_chunk")

    def solve_device(self, flu_in, flu_out, params: SolverParams, flux=None, de_out=None, pg_fail=None,
                     stream=None, mag_in=None, mag_out=None, ele=None):
        """Asynchronous on ``stream`` (a torch.cuda.Stream; default: torch's current stream).  MHD (CTU)
        takes mag_in [NPG][3][(FLU_NXT+1)*FLU_NXT^2], mag_out [NPG][3][17*16*16] and, with
        StoreElectric, ele [NPG][9][2][17*16]."""
        import torch
        npg = flu_in.shape[0]
        if stream is None:
            stream = torch.cuda.current_stream(flu_in.device)
        self._apply_tuned(npg)
        p = params.c(self)
        rc = self.lib.gb_fluid_solve_device(self.h, _dptr(flu_in), _dptr(flu_out), _dptr(mag_in), _dptr(mag_out),
                                            _dptr(de_out), _dptr(flux), _dptr(ele), _dptr(pg_fail), npg,
                                            ctypes.byref(p), ctypes.c_void_p(stream.cuda_stream))
        _check(rc, "gb_fluid_solve_device")

    def correct_unphysical_device(self, flu_in, flu_out, params: SolverParams, flux=None, de_out=None,
                                  counts=None, OPT__1ST_FLUX_CORR="3d", OPT__1ST_FLUX_CORR_SCHEME="hlle",
                                  OPT__LAST_RESORT_FLOOR=True, AutoReduceDt_Continue=False,
                                  OPT__CHECK_PRES_AFTER_FLU=False, stream=None, mag_in=None, mag_out=None):
        """CorrectUnphysical() of Flu_Close (src/Fluid/Flu_Close.cpp:542) in place on the arrays of a
        solve_device call; an MHD solver also takes the call's mag_in and mag_out (its MHD branch).
        counts: a device int32[2] the corrected / still-unphysical cell counts are added to
        (allocated and zeroed if None); returned, not synchronised."""
        import torch
        npg, nc, nx, fd = flu_out.shape[0], self.ncomp, self.flu_nxt, self.torch_dtype
        _expect(flu_in, (npg, nc, nx, nx, nx), fd, "flu_in")
        _expect(flu_out, (npg, nc, 16, 16, 16), fd, "flu_out")
        _expect(flux, (npg, 9, nc, 16, 16), fd, "flux")
        _expect(de_out, (npg, 16, 16, 16), torch.int8, "de_out")
        if self.mhd:
            if mag_in is None or mag_out is None:
                raise ValueError("an MHD solver corrects with mag_in and mag_out")
            _expect(mag_in, (npg, 3, (nx + 1) * nx * nx), fd, "mag_in")
            _expect(mag_out, (npg, 3, 17 * 16 * 16), fd, "mag_out")
        if counts is not None and ( counts.dtype != torch.int32 or counts.numel() < 2 ):
            raise ValueError("counts: a device int32 array of at least 2 elements")
        if stream is None:
            stream = torch.cuda.current_stream(flu_in.device)
        if counts is None:
            counts = torch.zeros(2, dtype=torch.int32, device=flu_in.device)
        cp = _CloseParams(FIRST_FLUX_CORR[OPT__1ST_FLUX_CORR], RSOLVER_1ST[OPT__1ST_FLUX_CORR_SCHEME],
                          int(OPT__LAST_RESORT_FLOOR), int(AutoReduceDt_Continue), int(OPT__CHECK_PRES_AFTER_FLU))
        p = params.c(self)
        if self.mhd:
            rc = self.lib.gb_fluid_correct_unphysical_mhd_device(
                self.h, _dptr(flu_in), _dptr(mag_in), _dptr(flu_out), _dptr(mag_out), _dptr(flux), npg,
                ctypes.byref(p), ctypes.byref(cp), _dptr(counts), ctypes.c_void_p(stream.cuda_stream))
            _check(rc, "gb_fluid_correct_unphysical_mhd_device")
            return counts
        rc = self.lib.gb_fluid_correct_unphysical_device(
            self.h, _dptr(flu_in), _dptr(flu_out), _dptr(de_out), _dptr(flux), flu_out.shape[0], ctypes.byref(p),
            ctypes.byref(cp), _dptr(counts), ctypes.c_void_p(stream.cuda_stream))
        _check(rc, "gb_fluid_correct_unphysical_device")
        return counts

    def flux_fixup_device(self, fluid, flux, has_flux, params: SolverParams, de_status=None, tvar=None,
                          stream=None, magnetic=None):
        """Flu_FixUp_Flux() (src/Fluid/Flu_FixUp_Flux.cpp:23) in place on device patches of one level:
        fluid [NP][NCOMP][8][8][8], flux [NP][6][NCOMP][8][8] (coarse minus fine flux of each face),
        has_flux uint8 [NP][6], de_status int8 [NP][8][8][8] with dual energy, magnetic
        [NP][3][9*8*8] (the patches' face-centred B) with MHD; params.dh and the floors are used;
        tvar = FixUpVar_Flux (all variables by default)."""
        import torch
        npatch, nc, fd = fluid.shape[0], self.ncomp, self.torch_dtype
        _expect(fluid, (npatch, nc, 8, 8, 8), fd, "fluid")
        _expect(flux, (npatch, 6, nc, 8, 8), fd, "flux")
        _expect(has_flux, (npatch, 6), torch.uint8, "has_flux")
        _expect(de_status, (npatch, 8, 8, 8), torch.int8, "de_status")
        if stream is None:
            stream = torch.cuda.current_stream(fluid.device)
        if tvar is None:
            tvar = (1 << self.ncomp) - 1
        p = params.c(self)
        if self.mhd:
            if magnetic is None:
                raise ValueError("an MHD fix-up needs the patches' magnetic field")
            _expect(magnetic, (npatch, 3, 9 * 8 * 8), fd, "magnetic")
            rc = self.lib.gb_flux_fixup_mhd_device(ctypes.byref(self.cfg), _dptr(fluid), _dptr(magnetic), _dptr(flux),
                                                   _dptr(has_flux), npatch, ctypes.byref(p), tvar,
                                                   ctypes.c_void_p(stream.cuda_stream))
            _check(rc, "gb_flux_fixup_mhd_device")
            return
        rc = self.lib.gb_flux_fixup_device(ctypes.byref(self.cfg), _dptr(fluid), _dptr(de_status), _dptr(flux),
                                           _dptr(has_flux), fluid.shape[0], ctypes.byref(p), tvar,
                                           ctypes.c_void_p(stream.cuda_stream))
        _check(rc, "gb_flux_fixup_device")

    def fixup_electric_device(self, magnetic, electric, electric_bitrep, has_ele, sib_leaf, dh, stream=None):
        """MHD_FixUp_Electric() (src/Model_Hydro/MHD_FixUp_Electric.cpp:22) in place on device patches
        of one level: magnetic [NP][3][9*8*8] corrected; electric and electric_bitrep
        [NP][ELE_PER_PATCH] (the 18 sides packed) zeroed on the patches with a listed side;
        has_ele uint8 [NP][18]; sib_leaf uint8
        [NP][6] (1 where the sibling across the face is a leaf or the non-periodic boundary)."""
        import torch
        npatch, fd = magnetic.shape[0], self.torch_dtype
        _expect(magnetic, (npatch, 3, 9 * 8 * 8), fd, "magnetic")
        _expect(electric, (npatch, ELE_PER_PATCH), fd, "electric")
        _expect(electric_bitrep, (npatch, ELE_PER_PATCH), fd, "electric_bitrep")
        _expect(has_ele, (npatch, 18), torch.uint8, "has_ele")
        _expect(sib_leaf, (npatch, 6), torch.uint8, "sib_leaf")
        if stream is None:
            stream = torch.cuda.current_stream(magnetic.device)
        rc = self.lib.gb_mhd_fixup_electric_device(ctypes.byref(self.cfg), _dptr(magnetic), _dptr(electric),
                                                   _dptr(electric_bitrep), _dptr(has_ele), _dptr(sib_leaf), npatch,
                                                   float(dh), ctypes.c_void_p(stream.cuda_stream))
        _check(rc, "gb_mhd_fixup_electric_device")

    def solve_levels_device(self, flu_in, flu_out, level_npg, level_dt, level_dh, params: SolverParams,
                            flux=None, de_out=None, pg_fail=None, stream=None):
        import torch
        if stream is None:
            stream = torch.cuda.current_stream(flu_in.device)
        n = len(level_npg)
        self._apply_tuned(sum(level_npg))
        npg = (ctypes.c_int * n)(*level_npg)
        dt = (ctypes.c_double * n)(*level_dt)
        dh = (ctypes.c_double * n)(*level_dh)
        p = params.c(self)
        rc = self.lib.gb_fluid_solve_levels_device(self.h, _dptr(flu_in), _dptr(flu_out), _dptr(de_out), _dptr(flux),
                                                   _dptr(pg_fail), n, npg, dt, dh, ctypes.byref(p),
                                                   ctypes.c_void_p(stream.cuda_stream))
        _check(rc, "gb_fluid_solve_levels_device")

    def capture_levels(self, flu_in, flu_out, level_npg, level_dt, level_dh, params: SolverParams, flux=None,
                       de_out=None, pg_fail=None):
        """Capture the multi-level launch into a CUDA graph (see LevelsGraph)."""
        return LevelsGraph(self, flu_in, flu_out, level_npg, level_dt, level_dh, params, flux, de_out, pg_fail)

    # -- host arrays (numpy), the CPU_FluidSolver form --------------------------------------------
    def solve_host(self, flu_in, params: SolverParams, flu_out=None, flux=None, de_out=None, mag_in=None,
                   mag_out=None, ele=None):
        """Synchronous; returns (flu_out, flux, de_out), and for MHD (flu_out, flux, de_out, mag_out, ele)."""
        flu_in = np.ascontiguousarray(flu_in, dtype=self.np_dtype)
        npg = flu_in.shape[0]
        if flu_out is None:
            flu_out = np.empty((npg, self.ncomp, 16, 16, 16), self.np_dtype)
        if params.StoreFlux and flux is None:
            flux = np.empty((npg, 9, self.ncomp, 16, 16), self.np_dtype)
        if self.dual and de_out is None:
            de_out = np.zeros((npg, 16, 16, 16), np.int8)
        if self.mhd:
            if mag_in is None:
                raise ValueError("MHD needs mag_in")
            mag_in = np.ascontiguousarray(mag_in, dtype=self.np_dtype)
            if mag_out is None:
                mag_out = np.empty((npg, 3, 17 * 16 * 16), self.np_dtype)
            if params.StoreElectric and ele is None:
                ele = np.empty((npg, 9, 2, 17 * 16), self.np_dtype)
        self._apply_tuned(min(npg, HOST_CHUNK))
        p = params.c(self)
        rc = self.lib.gb_fluid_solve_host(self.h, _hptr(flu_in), _hptr(flu_out), _hptr(mag_in), _hptr(mag_out),
                                          _hptr(de_out), _hptr(flux) if params.StoreFlux else None,
                                          _hptr(ele) if params.StoreElectric else None, npg, ctypes.byref(p))
        _check(rc, "gb_fluid_solve_host")
        if self.mhd:
            return flu_out, flux, de_out, mag_out, ele
        return flu_out, flux, de_out

    def solve_host_async(self, flu_in, flu_out, params: SolverParams, flux=None, de_out=None, mag_in=None,
                         mag_out=None, ele=None, stream=None):
        """CUAPI_Asyn_FluidSolver: enqueue H2D, solve and D2H of host (preferably pinned) arrays and
        return at once; ``synchronize()`` (CUAPI_Synchronize) ends the call.  Every array must be
        given, C-contiguous and of the solver's dtype, and must stay untouched until then.  ``stream``
        (a torch.cuda.Stream) orders the call after the stream's earlier work and the stream's later
        work after the call; None orders it only after this solver's earlier host-array calls."""
        for name, a in (("flu_in", flu_in), ("flu_out", flu_out), ("flux", flux), ("mag_in", mag_in),
                        ("mag_out", mag_out), ("ele", ele)):
            if a is not None and a.dtype != self.np_dtype:
                raise ValueError(f"{name}: dtype {a.dtype}, expected {np.dtype(self.np_dtype)}")
        npg = flu_in.shape[0]
        self._apply_tuned(min(npg, HOST_CHUNK))
        p = params.c(self)
        st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        rc = self.lib.gb_fluid_solve_host_async(self.h, _hptr(flu_in), _hptr(flu_out), _hptr(mag_in), _hptr(mag_out),
                                                _hptr(de_out), _hptr(flux) if params.StoreFlux else None,
                                                _hptr(ele) if params.StoreElectric else None, npg, ctypes.byref(p), st)
        _check(rc, "gb_fluid_solve_host_async")

    def synchronize(self):
        """Wait for this solver's host-array calls (CUAPI_Synchronize)."""
        _check(self.lib.gb_fluid_synchronize(self.h), "gb_fluid_synchronize")


class LevelsGraph:
    """A captured multi-level solver launch (gb_fluid_graph_*); replay with launch()."""

    def __init__(self, solver, flu_in, flu_out, level_npg, level_dt, level_dh, params, flux, de_out, pg_fail):
        self.solver = solver
        self.lib = solver.lib
        self.n = len(level_npg)
        self._keep = (flu_in, flu_out, flux, de_out, pg_fail)       # the graph holds raw pointers
        npg = (ctypes.c_int * self.n)(*level_npg)
        dt = (ctypes.c_double * self.n)(*level_dt)
        dh = (ctypes.c_double * self.n)(*level_dh)
        p = params.c(solver)
        h = ctypes.c_void_p()
        _check(self.lib.gb_fluid_graph_create_levels(solver.h, _dptr(flu_in), _dptr(flu_out), _dptr(de_out),
                                                     _dptr(flux), _dptr(pg_fail), self.n, npg, dt, dh,
                                                     ctypes.byref(p), ctypes.byref(h)), "gb_fluid_graph_create_levels")
        self.h = h

    def set_dt(self, level_dt):
        dt = (ctypes.c_double * self.n)(*level_dt)
        _check(self.lib.gb_fluid_graph_set_dt(self.h, dt), "gb_fluid_graph_set_dt")

    def launch(self, stream=None):
        import torch
        if stream is None:
            stream = torch.cuda.current_stream()
        _check(self.lib.gb_fluid_graph_launch(self.h, ctypes.c_void_p(stream.cuda_stream)), "gb_fluid_graph_launch")

    def close(self):
        if getattr(self, "h", None):
            self.lib.gb_fluid_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PinnedArray:
    """numpy view of pinned host memory from gb_fluid_host_alloc (the reference pins its solver
    arrays with cudaMallocHost, src/GPU_API/CUAPI_MemAllocate_Fluid.cu:288-322)."""

    def __init__(self, shape, dtype):
        self.lib = load_library()
        dtype = np.dtype(dtype)
        nbytes = int(np.prod(shape)) * dtype.itemsize
        p = ctypes.c_void_p()
        _check(self.lib.gb_fluid_host_alloc(ctypes.byref(p), max(nbytes, 16)), "gb_fluid_host_alloc")
        self.ptr = p
        buf = (ctypes.c_char * max(nbytes, 16)).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)

    def free(self):
        if self.ptr:
            self.array = None
            self.lib.gb_fluid_host_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def interpolate_device(cdata, fdata, scheme, cstart, crange, fstart=(0, 0, 0), monotonic=True, mono_coeff=2.0,
                       opp_sign_0th_order=False, iterate=False, int_prim=True, mono_max_iter=10, gamma=5.0 / 3.0,
                       min_pres=0.0, status=None, stream=None):
    """Interpolate() of the reference (src/Interpolation/Interpolate.cpp:90) on a batch of regions:
    cdata [nbatch][ncomp][cz][cy][cx] and fdata [nbatch][ncomp][fz][fy][fx] (contiguous CUDA tensors,
    float32 or float64); cstart / crange / fstart are (x, y, z).  ``monotonic``: a bool for every
    component or a sequence of ncomp bools.  ``iterate`` selects Interpolate_Iterate (the five conserved
    hydro variables; OPT__INT_PRIM = int_prim, MONO_MAX_ITER = mono_max_iter) and needs ``status``, a
    device int32 tensor that receives INTERP_FAILED where a parent still fails.  Asynchronous."""
    import torch
    lib = load_library()
    nb, nc = cdata.shape[0], cdata.shape[1]
    if fdata.shape[:2] != cdata.shape[:2] or cdata.dtype != fdata.dtype:
        raise ValueError("cdata and fdata need the same batch, components and dtype")
    if cdata.dtype not in (torch.float32, torch.float64):
        raise ValueError("float32 or float64 arrays")
    mono = [bool(monotonic)] * nc if isinstance(monotonic, bool) else [bool(m) for m in monotonic]
    if len(mono) != nc:
        raise ValueError("monotonic: one flag per component")
    if iterate and (status is None or status.dtype != torch.int32):
        raise ValueError("iterate needs a device int32 status tensor")
    p = _InterpParams()
    p.scheme = INT_SCHEME[scheme] if isinstance(scheme, str) else int(scheme)
    p.precision = PRECISION["fp64"] if cdata.dtype == torch.float64 else PRECISION["fp32"]
    p.ncomp = nc
    p.csize[:] = [cdata.shape[4], cdata.shape[3], cdata.shape[2]]
    p.fsize[:] = [fdata.shape[4], fdata.shape[3], fdata.shape[2]]
    p.cstart[:], p.crange[:], p.fstart[:] = list(cstart), list(crange), list(fstart)
    p.monotonic = sum(1 << v for v, m in enumerate(mono) if m)
    p.mono_coeff, p.opp_sign_0th_order = mono_coeff, int(opp_sign_0th_order)
    p.mode = 1 if iterate else 0
    p.int_prim, p.mono_max_iter, p.gamma, p.min_pres = int(int_prim), int(mono_max_iter), gamma, min_pres
    p.status = status.data_ptr() if status is not None else None
    if stream is None:
        stream = torch.cuda.current_stream(cdata.device)
    _check(lib.gb_interpolate_device(ctypes.byref(p), _dptr(cdata), _dptr(fdata), nb,
                                     ctypes.c_void_p(stream.cuda_stream)), "gb_interpolate_device")


def assemble_windows_device(fine, nbr, cint, windows, stream=None):
    """Ghost-zone fill of one level (gb_assemble_windows_device): windows [npg][ncomp][nxt^3] from the
    patch groups' interiors fine [npg][ncomp][16^3], the same-level neighbours nbr (int32 [npg][27],
    side s = (dz+1)*9 + (dy+1)*3 + (dx+1), -1 = coarse) and the coarse-interpolated windows cint (same
    shape as windows, or None).  Contiguous CUDA tensors of one dtype."""
    import torch
    lib = load_library()
    npg, nc, nxt = windows.shape[0], windows.shape[1], windows.shape[2]
    _expect(fine, (npg, nc, 16, 16, 16), windows.dtype, "fine")
    _expect(nbr, (npg, 27), torch.int32, "nbr")
    _expect(cint, tuple(windows.shape), windows.dtype, "cint")
    prec = PRECISION["fp64"] if windows.dtype == torch.float64 else PRECISION["fp32"]
    if stream is None:
        stream = torch.cuda.current_stream(windows.device)
    _check(lib.gb_assemble_windows_device(_dptr(fine), _dptr(nbr), _dptr(cint), _dptr(windows), npg, nc, nxt, prec,
                                          ctypes.c_void_p(stream.cuda_stream)), "gb_assemble_windows_device")
