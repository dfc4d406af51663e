"""The reference's own GPU kernel CUFLU_FluidSolver_MHM (src/Model_Hydro/CPU_Hydro/CPU_FluidSolver_MHM.cpp:265),
built unmodified for sm_100a by oracle/build_ref_gpu.sh: checked against the reference CPU solver (so
that the bench's reference-GPU leg times a correct launch), and this repository's kernels checked
against it on the same device arrays."""
import numpy as np
import pytest

import pyoracle as po
from gamer_b200.fluid import FluidSolver, SolverParams
from parity import RTOL32, RTOL64, gpu_solve, kh_case, lognormal_case, scaled_err

pytestmark = pytest.mark.gpu

TOL = {"fp32": RTOL32, "fp64": RTOL64}


def _ref_gpu(variant, prec, x, dt, dh, **kw):
    import torch
    r = po.RefGpuSolver(variant, prec)
    dt_t = torch.float64 if prec == "fp64" else torch.float32
    t_in = torch.from_numpy(np.ascontiguousarray(x)).to("cuda", dt_t)
    t_out = torch.full((x.shape[0], 5, 16, 16, 16), float("nan"), dtype=dt_t, device="cuda")
    t_flux = torch.full((x.shape[0], 9, 5, 16, 16), float("nan"), dtype=dt_t, device="cuda")
    r.solve_device(t_in, t_out, dt, dh, t_flux, **kw)
    torch.cuda.synchronize()
    return {"out": t_out.cpu().numpy(), "flux": t_flux.cpu().numpy()}


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("variant,nxt", [("mhm_plm_hllc", 20), ("mhm_ppm_roe", 22)])
def test_reference_gpu_kernel_matches_reference_cpu(cuda_device, variant, nxt, prec):
    x, dt, dh = lognormal_case(npd=2, seed=101, nxt=nxt)
    cpu = po.RefSolver(variant, prec).solve(x, dt, dh)
    gpu = _ref_gpu(variant, prec, x, dt, dh)
    assert scaled_err(gpu["out"], cpu["out"]) <= TOL[prec]
    assert scaled_err(gpu["flux"], cpu["flux"], axis_var=2) <= TOL[prec]


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
@pytest.mark.parametrize("variant,nxt", [("mhm_plm_hllc", 20), ("mhm_ppm_roe", 22)])
def test_this_solver_matches_reference_gpu_kernel(cuda_device, variant, nxt, prec):
    """Same Kelvin-Helmholtz input on both GPU kernels: the mixed policy against the reference's FP32
    build (its storage type)."""
    _, lr, rs = variant.split("_")
    x, dt, dh = kh_case(npd=2, seed=102, nxt=nxt)
    rprec = "fp64" if prec == "fp64" else "fp32"
    ref = _ref_gpu(variant, rprec, x, dt, dh)
    g = gpu_solve(FluidSolver(lr=lr, rsolver=rs, precision=prec, flu_nxt=nxt), x, SolverParams(dt=dt, dh=dh))
    assert scaled_err(g["out"], ref["out"]) <= TOL[rprec]
    assert scaled_err(g["flux"], ref["flux"], axis_var=2) <= TOL[rprec]
