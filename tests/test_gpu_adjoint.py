"""GPU tests of the periodic-box kernels and of the hand-written adjoint of the MHM+PLM+HLLC step
(through the C ABI)."""
import numpy as np
import pytest

import pyoracle as po
from gamer_b200 import ic
from gamer_b200.fluid import FluidSolver, SolverParams
from parity import GAMMA

pytestmark = pytest.mark.gpu


def _box(npd, seed, smooth=True):
    b = ic.smooth_box(npd, seed, gamma=GAMMA) if smooth else ic.lognormal_box(npd, seed, gamma=GAMMA)
    dh = 1.0 / (npd * 16)
    return b, dh, ic.cfl_dt(b, GAMMA, dh, cfl=0.5)


def test_box_gather_scatter_match_host_cut(cuda_device):
    import torch
    from gamer_b200 import adjoint
    b, dh, dt = _box(2, 1, smooth=False)
    s = FluidSolver(precision="fp64")
    tb = torch.from_numpy(ic.to_device_layout(b)).cuda()
    win = adjoint.gather(s, tb)
    assert np.array_equal(win.cpu().numpy(), ic.cut_patch_groups(b, 20))
    back = adjoint.scatter(s, win[:, :, 2:18, 2:18, 2:18].contiguous(), tb)
    assert np.array_equal(back.cpu().numpy(), ic.to_device_layout(b))


@pytest.mark.parametrize("npd", [1, 2, 3])
def test_gather_adjoint_is_the_transpose(cuda_device, npd):
    """<gather(b), w> == <b, gather_adjoint(w)>, also when a window wraps onto itself (npd = 1)."""
    import ctypes
    import torch
    from gamer_b200 import adjoint
    from gamer_b200.fluid import _dptr
    s = FluidSolver(precision="fp64")
    rng = np.random.default_rng(npd)
    n = 16 * npd
    b = torch.from_numpy(rng.standard_normal((5, n, n, n))).cuda()
    w = torch.from_numpy(rng.standard_normal((npd ** 3, 5, 20, 20, 20))).cuda()
    gb = adjoint.gather(s, b)
    wt = torch.empty_like(b)
    s.lib.gb_box_gather_adjoint_device(_dptr(w), _dptr(wt), npd, npd, npd, 20, 5,
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    lhs = float((gb * w).sum())
    rhs = float((b * wt).sum())
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def _loss_weights(shape, seed=99):
    return np.random.default_rng(seed).standard_normal(shape[1:])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_adjoint_one_step_vs_central_difference(cuda_device, precision):
    import torch
    from gamer_b200.adjoint import mhm_steps
    b, dh, dt = _box(2, 5)
    s = FluidSolver(precision=precision)
    prm = SolverParams(dt=dt, dh=dh)
    dtype = torch.float64 if precision == "fp64" else torch.float32
    x = torch.from_numpy(ic.to_device_layout(b)).to(device="cuda", dtype=dtype).requires_grad_(True)
    w = torch.from_numpy(_loss_weights(x.shape)).cuda()
    y = mhm_steps(x, 1, s, prm)
    loss = (y[0].double() * w).sum()
    loss.backward()
    grad = x.grad.double()
    rng = np.random.default_rng(7)
    v = torch.from_numpy(rng.standard_normal(x.shape) * np.array([1.0, 0.2, 0.2, 0.2, 1.0])[:, None, None, None]).cuda()
    eps = 1e-3
    s64 = FluidSolver(precision="fp64")
    x64 = x.detach().double()
    lp = float((mhm_steps(x64 + eps * v, 1, s64, prm)[0] * w).sum())
    lm = float((mhm_steps(x64 - eps * v, 1, s64, prm)[0] * w).sum())
    fd = (lp - lm) / (2 * eps)
    ad = float((grad * v).sum())
    assert abs(ad - fd) <= 1e-4 * abs(fd), (ad, fd)


def _ref_k_steps(b, K, dt, dh):
    """K steps of the reference FP64 CPU solver on a periodic box (host ghost-zone refill)."""
    ref = po.RefSolver("mhm_plm_hllc", "fp64")
    npd = b.shape[1] // 16
    cur = b
    for _ in range(K):
        out = ref.solve(ic.cut_patch_groups(cur, 20), dt, dh, store_flux=False)["out"]
        cur = ic.assemble_box(out, npd)
    return cur


def test_adjoint_k8_fp32_vs_fp64_reference_gradient(cuda_device):
    """K = 8 steps: the FP32 hand-written adjoint against central differences of the reference FP64
    CPU solver (the 'FP64 reference gradient'), loss = sum w * rho_final, eps = 1e-3."""
    import torch
    from gamer_b200.adjoint import mhm_steps
    K = 8
    b, dh, dt = _box(2, 11)
    s = FluidSolver(precision="fp32")
    prm = SolverParams(dt=dt, dh=dh)
    x = torch.from_numpy(ic.to_device_layout(b)).to(device="cuda", dtype=torch.float32).requires_grad_(True)
    w = _loss_weights(x.shape, seed=5)
    y = mhm_steps(x, K, s, prm)
    loss = (y[0].double() * torch.from_numpy(w).cuda()).sum()
    loss.backward()
    grad = ic.from_device_layout(x.grad.double().cpu().numpy())
    rng = np.random.default_rng(3)
    v = rng.standard_normal(b.shape) * np.array([1.0, 0.2, 0.2, 0.2, 1.0])[:, None, None, None]
    eps = 1e-3
    wb = ic.from_device_layout(w[None])[0]
    lp = float((_ref_k_steps(b + eps * v, K, dt, dh)[0] * wb).sum())
    lm = float((_ref_k_steps(b - eps * v, K, dt, dh)[0] * wb).sum())
    fd = (lp - lm) / (2 * eps)
    ad = float((grad * v).sum())
    assert abs(ad - fd) <= 1e-4 * abs(fd), (ad, fd)
