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
    # smooth = the branch-free state of ic.supersonic_separable_box (finite differences across a
    # limiter or wave-speed switch would not converge to the derivative)
    b = ic.supersonic_separable_box(npd, gamma=GAMMA, seed=seed) if smooth else ic.lognormal_box(npd, seed, gamma=GAMMA)
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


def _direction(shape, seed):
    """Smooth perturbation direction (long-wavelength modes, O(0.1) of each variable's scale)."""
    rng = np.random.default_rng(seed)
    n = shape[1]
    d = np.stack([ic._smooth_gaussian(rng, n, 0.1, kmax=2) for _ in range(shape[0])])
    return ic.to_device_layout(d) * np.array([1.0, 1.0, 1.0, 1.0, 3.0])[:, None, None, None]


@pytest.mark.parametrize("rs", ["hllc", "hlle", "roe", "exact"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_adjoint_one_step_vs_central_difference(cuda_device, precision, rs):
    """One step, every Riemann solver the adjoint differentiates (the exact solver's star pressure
    through the implicit function theorem at its root)."""
    import torch
    from gamer_b200.adjoint import mhm_steps
    b, dh, dt = _box(2, 5)
    s = FluidSolver(precision=precision, rsolver=rs)
    prm = SolverParams(dt=dt, dh=dh)
    dtype = torch.float64 if precision == "fp64" else torch.float32
    x = torch.from_numpy(ic.to_device_layout(b)).to(device="cuda", dtype=dtype).requires_grad_(True)
    w = torch.from_numpy(_loss_weights(x.shape)).cuda()
    y = mhm_steps(x, 1, s, prm)
    loss = (y[0].double() * w).sum()
    loss.backward()
    grad = x.grad.double()
    # direction of size ~1e-2 of the state: eps = 1e-3 stays inside the branch-free neighbourhood
    v = 0.1 * torch.from_numpy(_direction(x.shape, 7)).cuda()
    eps = 1e-3
    s64 = FluidSolver(precision="fp64", rsolver=rs)
    x64 = x.detach().double()
    lp = float((mhm_steps(x64 + eps * v, 1, s64, prm)[0] * w).sum())
    lm = float((mhm_steps(x64 - eps * v, 1, s64, prm)[0] * w).sum())
    fd = (lp - lm) / (2 * eps)
    ad = float((grad * v).sum())
    assert abs(ad - fd) <= 1e-4 * abs(fd), (ad, fd)


def test_adjoint_single_cell_perturbation_converges(cuda_device):
    """On generic (lognormal, branch-rich) data the adjoint still matches central differences of a
    single-cell perturbation once eps is below the distance to the nearest branch switch."""
    import torch
    from gamer_b200.adjoint import mhm_steps
    b, dh, dt = _box(2, 21, smooth=False)
    s = FluidSolver(precision="fp64")
    prm = SolverParams(dt=dt, dh=dh)
    x = torch.from_numpy(ic.to_device_layout(b)).cuda().requires_grad_(True)
    w = torch.from_numpy(_loss_weights(x.shape)).cuda()
    (mhm_steps(x, 2, s, prm)[0] * w).sum().backward()
    v = torch.zeros_like(x)
    v[:, 10, 9, 12] = torch.tensor([1.0, 0.3, -0.2, 0.1, 2.0], dtype=torch.float64)
    ad = float((x.grad * v).sum())
    eps = 1e-6
    lp = float((mhm_steps(x.detach() + eps * v, 2, s, prm)[0] * w).sum())
    lm = float((mhm_steps(x.detach() - eps * v, 2, s, prm)[0] * w).sum())
    fd = (lp - lm) / (2 * eps)
    assert abs(ad - fd) <= 1e-6 * abs(fd), (ad, fd)


def _ref_k_steps(b, K, dt, dh, variant="mhm_plm_hllc"):
    """K steps of the reference FP64 CPU solver on a periodic box (host ghost-zone refill)."""
    ref = po.RefSolver(variant, "fp64")
    npd = b.shape[1] // 16
    cur = b
    for _ in range(K):
        out = ref.solve(ic.cut_patch_groups(cur, 20), dt, dh, store_flux=False)["out"]
        cur = ic.assemble_box(out, npd)
    return cur


def _oblique_direction(n, seed):
    """Perturbation that is, like the oblique-wave state, a function of i + j + k only."""
    rng = np.random.default_rng(seed)
    i = np.arange(n)
    s = (i[:, None, None] + i[None, :, None] + i[None, None, :]).astype(np.float64)
    v = np.stack([0.1 * np.sin(2.0 * np.pi * s / n + rng.uniform(0.0, 2.0 * np.pi)) for _ in range(5)])
    return v * np.array([1.0, 1.0, 1.0, 1.0, 3.0])[:, None, None, None]


def test_adjoint_k8_fp32_vs_fp64_reference_gradient(cuda_device):
    """K = 8 steps: the FP32 hand-written adjoint against central differences of the reference FP64
    CPU solver (the 'FP64 reference gradient'), loss = sum w * rho_final.

    A generic 3-D state evolved for several steps has limiter branch switches at every scale, and a
    finite difference across a switch does not converge.  The state is therefore the oblique wave
    (every field a function of i + j + k, kept so by the scheme), perturbed along a direction of the
    same form, and the finite difference is accepted only if two perturbation sizes agree."""
    import torch
    from gamer_b200.adjoint import mhm_steps
    K = 8
    npd, n = 2, 32
    b = ic.oblique_wave_box(npd, gamma=GAMMA, seed=11)
    dh = 1.0 / n
    dt = ic.cfl_dt(b, GAMMA, dh, cfl=0.5)
    s = FluidSolver(precision="fp32")
    prm = SolverParams(dt=dt, dh=dh)
    x = torch.from_numpy(ic.to_device_layout(b)).to(device="cuda", dtype=torch.float32).requires_grad_(True)
    w = _loss_weights(x.shape, seed=5)
    y = mhm_steps(x, K, s, prm)
    loss = (y[0].double() * torch.from_numpy(w).cuda()).sum()
    loss.backward()
    grad = ic.from_device_layout(x.grad.double().cpu().numpy())
    v = _oblique_direction(n, 3)
    wb = ic.from_device_layout(w[None])[0]
    b64 = ic.from_device_layout(x.detach().double().cpu().numpy())     # the float-rounded state

    def fd(eps):
        lp = float((_ref_k_steps(b64 + eps * v, K, dt, dh)[0] * wb).sum())
        lm = float((_ref_k_steps(b64 - eps * v, K, dt, dh)[0] * wb).sum())
        return (lp - lm) / (2 * eps)

    fd1, fd2 = fd(1e-5), fd(5e-6)
    assert abs(fd1 - fd2) <= 1e-6 * abs(fd1), ("finite difference crossed a branch switch", fd1, fd2)
    ad = float((grad * v).sum())
    assert abs(ad - fd1) <= 1e-4 * abs(fd1), (ad, fd1)


def test_adjoint_k4_exact_solver_vs_fp64_reference_gradient(cuda_device):
    """K = 4 steps with the exact Riemann solver: the FP64 adjoint against central differences of
    the reference's FP64 exact-solver build on the oblique wave, loss = sum w * rho_final."""
    import torch
    from gamer_b200.adjoint import mhm_steps
    K = 4
    npd, n = 2, 32
    b = ic.oblique_wave_box(npd, gamma=GAMMA, seed=12)
    dh = 1.0 / n
    dt = ic.cfl_dt(b, GAMMA, dh, cfl=0.5)
    s = FluidSolver(precision="fp64", rsolver="exact")
    prm = SolverParams(dt=dt, dh=dh)
    x = torch.from_numpy(ic.to_device_layout(b)).to(device="cuda", dtype=torch.float64).requires_grad_(True)
    w = _loss_weights(x.shape, seed=6)
    y = mhm_steps(x, K, s, prm)
    (y[0] * torch.from_numpy(w).cuda()).sum().backward()
    grad = ic.from_device_layout(x.grad.cpu().numpy())
    v = _oblique_direction(n, 4)
    wb = ic.from_device_layout(w[None])[0]

    def fd(eps):
        lp = float((_ref_k_steps(b + eps * v, K, dt, dh, "mhm_plm_exact")[0] * wb).sum())
        lm = float((_ref_k_steps(b - eps * v, K, dt, dh, "mhm_plm_exact")[0] * wb).sum())
        return (lp - lm) / (2 * eps)

    fd1, fd2 = fd(1e-5), fd(5e-6)
    assert abs(fd1 - fd2) <= 1e-6 * abs(fd1), ("finite difference crossed a branch switch", fd1, fd2)
    ad = float((grad * v).sum())
    assert abs(ad - fd1) <= 1e-5 * abs(fd1), (ad, fd1)
