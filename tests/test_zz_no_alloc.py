"""The allocation-free CTU+MHD entry point gb_ctu_mhd_solve_static (for callers that cannot call
cudaMalloc, e.g. codes whose device memory belongs to their own pool allocator) against the
solver-object entry point gb_fluid_solve_device, on two calls in a row.  Collected last and
independent of the other test files, so it passes alone and after them."""
import ctypes

import numpy as np
import pytest

from gamer_b200.fluid import FluidSolver, SolverParams, _Config, _Params, _dptr, load_library
from parity import GAMMA, gpu_solve_mhd, mhd_case

pytestmark = pytest.mark.gpu

PREC = {"fp32": 0, "mixed": 1, "fp64": 2}


def _lib():
    lib = load_library()
    vp = ctypes.c_void_p
    lib.gb_ctu_mhd_solve_static.argtypes = [ctypes.POINTER(_Config), vp, vp, vp, vp, vp, vp, ctypes.c_int,
                                            ctypes.POINTER(_Params), vp]
    lib.gb_ctu_mhd_solve_static.restype = ctypes.c_int
    lib.gb_ctu_mhd_static_capacity.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.gb_ctu_mhd_static_capacity.restype = ctypes.c_int
    return lib


def capacity(precision):
    """Patch groups one call takes (the fixed scratch over the pipeline's scratch per patch group),
    as the library reports it."""
    n = ctypes.c_int(0)
    assert _lib().gb_ctu_mhd_static_capacity(PREC[precision], ctypes.byref(n)) == 0
    return n.value


def _static_solve(precision, x, b, prm):
    import torch
    lib = _lib()
    cfg = _Config(5, 1, 5, PREC[precision], 0, 22, GAMMA)
    dt = torch.float64 if precision == "fp64" else torch.float32
    npg = x.shape[0]
    t_in = torch.from_numpy(x).to("cuda", dt)
    t_b = torch.from_numpy(b).to("cuda", dt)
    # garbage-filled outputs: the call must write everything it returns
    t_out = torch.full((npg, 5, 16, 16, 16), float("nan"), dtype=dt, device="cuda")
    t_bo = torch.full((npg, 3, 17 * 256), float("nan"), dtype=dt, device="cuda")
    t_f = torch.zeros((npg, 9, 5, 16, 16), dtype=dt, device="cuda")
    t_e = torch.zeros((npg, 9, 2, 17 * 16), dtype=dt, device="cuda")
    p = prm.c()
    rc = lib.gb_ctu_mhd_solve_static(ctypes.byref(cfg), _dptr(t_in), _dptr(t_b), _dptr(t_out), _dptr(t_bo),
                                     _dptr(t_f), _dptr(t_e), npg, ctypes.byref(p),
                                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return rc, {"out": t_out.cpu().numpy(), "mag_out": t_bo.cpu().numpy(), "flux": t_f.cpu().numpy(),
                "ele": t_e.cpu().numpy()}


@pytest.mark.parametrize("precision", ["fp32", "mixed", "fp64"])
def test_static_entry_point_matches_solver_entry_point(cuda_device, precision):
    s = FluidSolver(scheme="ctu", lr="plm", rsolver="hlld", precision=precision, gamma=GAMMA)
    npg = capacity(precision)
    assert 1 <= npg <= 27
    # two consecutive calls on different states: the second must not see the first's scratch
    for seed in (1, 2):
        x, b, dt, dh = mhd_case(npd=3, seed=seed)
        x, b = x[:npg], b[:npg]
        prm = SolverParams(dt=dt, dh=dh, StoreFlux=True, StoreElectric=True)
        want = gpu_solve_mhd(s, x, b, prm)
        rc, got = _static_solve(precision, x, b, prm)
        assert rc == 0
        for k in ("out", "mag_out", "flux", "ele"):
            assert np.array_equal(got[k], want[k]), k


def test_static_entry_point_rejects_batches_beyond_its_scratch(cuda_device):
    x, b, dt, dh = mhd_case(npd=3, seed=3)
    prm = SolverParams(dt=dt, dh=dh, StoreFlux=False)
    n64, n32 = capacity("fp64"), capacity("fp32")
    assert n64 < n32 < x.shape[0]
    rc, _ = _static_solve("fp64", x[:n64 + 1], b[:n64 + 1], prm)
    assert rc == -1
    rc, _ = _static_solve("fp32", x[:n32 + 1], b[:n32 + 1], prm)
    assert rc == -1
    rc, _ = _static_solve("fp32", x[:n32], b[:n32], prm)
    assert rc == 0
