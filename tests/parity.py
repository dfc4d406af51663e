"""Shared helpers of the parity tests: seeded inputs, GPU runs through the C ABI, error metrics."""
from __future__ import annotations

import numpy as np

from gamer_b200 import ic

GAMMA = 5.0 / 3.0

# FP32 GPU vs FP32 reference: |g - r| <= RTOL32*|r| + RTOL32*rms(r_v) for each variable v.
# The second term keeps momenta that cross zero from turning a round-off difference into an
# unbounded relative error.
RTOL32 = 1e-5
# FP64 GPU vs FP64 reference (same algorithm, FMA contraction and operation order differ)
RTOL64 = 1e-11


def lognormal_case(npd=4, seed=1234, nxt=20, dual=False):
    box = ic.lognormal_box(npd, seed=seed, gamma=GAMMA, dual=dual)
    dh = 1.0 / (npd * 16)
    dt = ic.cfl_dt(box, GAMMA, dh, cfl=0.5)
    return ic.cut_patch_groups(box, nxt), dt, dh


def blast_case(npd=2, seed=7, nxt=20, dual=True):
    box = ic.blast_box(npd, seed=seed, gamma=GAMMA, dual=dual)
    dh = 1.0 / (npd * 16)
    dt = ic.cfl_dt(box, GAMMA, dh, cfl=0.5)
    return ic.cut_patch_groups(box, nxt), dt, dh


def kh_case(npd=2, seed=3, nxt=22, dual=False):
    box = ic.kelvin_helmholtz_box(npd, seed=seed, gamma=GAMMA, dual=dual)
    dh = 1.0 / (npd * 16)
    dt = ic.cfl_dt(box, GAMMA, dh, cfl=0.5)
    return ic.cut_patch_groups(box, nxt), dt, dh


def with_passive(x, dual, seed, npass=2):
    """Append npass passive scalars (positive fractions of the density) after the fluid variables
    and before the dual-energy field, the reference's order (include/Macro.h:290-305)."""
    rng = np.random.default_rng(seed)
    rho = x[:, 0]
    p = np.stack([rho * (0.2 + 0.6 * rng.random(rho.shape)) for _ in range(npass)], axis=1)
    return np.concatenate([x[:, :5], p, x[:, 5:6]], axis=1) if dual else np.concatenate([x, p], axis=1)


def scaled_err(g, r, axis_var=1):
    """max over cells of |g-r| / (|r| + s_v): s_v is the rms of variable v, floored at 1e-2 of the
    largest variable rms so that a component that is zero up to round-off (e.g. m_z of a 2-D shear
    layer) is judged against the flow's scale, not its own noise."""
    g = np.asarray(g, np.float64)
    r = np.asarray(r, np.float64)
    red = tuple(a for a in range(r.ndim) if a != axis_var)
    rms = np.sqrt(np.mean(r * r, axis=red, keepdims=True))
    rms = np.maximum(rms, 1e-2 * rms.max())
    return float(np.max(np.abs(g - r) / (np.abs(r) + rms + 1e-300)))


def reference_spread(ref_solver, x, dt, dh, eps, seeds=(0, 1, 2), nvar=None, key="out", axis_var=1, **solve_kw):
    """The reference's own round-off spread on a case: the largest scaled_err of result `key` between
    its solve of x and of x with every input value multiplied by (1 + eps * N(0,1)), over a few seeds.

    At strong shocks a limiter branch or an entropy/energy switch can flip on a last-bit difference,
    and characteristic projections amplify rounding, so two correct builds that contract FMAs
    differently disagree by far more than their epsilon; this measures by how much for the reference
    itself.  nvar: the leading input variables that get the noise (the dual-energy field is exactly
    reconstructed from them); solve_kw go to every solve (e.g. mag_in, limiter)."""
    base = ref_solver.solve(x, dt, dh, **solve_kw)[key]
    worst = 0.0
    for s in seeds:
        xp = np.array(x, copy=True)
        v = slice(None) if nvar is None else slice(0, nvar)
        noise = np.random.default_rng(s).standard_normal(xp[:, v].shape)
        xp[:, v] = xp[:, v] * (1.0 + eps * noise)
        worst = max(worst, scaled_err(ref_solver.solve(xp, dt, dh, **solve_kw)[key], base, axis_var=axis_var))
    return worst


def frac_rel_within(g, r, tol):
    g = np.asarray(g, np.float64)
    r = np.asarray(r, np.float64)
    return float(np.mean(np.abs(g - r) <= tol * np.abs(r)))


def l1_rel(g, r):
    g = np.asarray(g, np.float64)
    r = np.asarray(r, np.float64)
    return float(np.sum(np.abs(g - r)) / np.sum(np.abs(r)))


def gpu_solve(solver, x, params, device="cuda:0", want_flux=True, de=None, pg_fail=False):
    """Run FluidSolver.solve_device on numpy input; returns numpy outputs."""
    import torch
    npg = x.shape[0]
    t_in = torch.from_numpy(np.ascontiguousarray(x, dtype=solver.np_dtype)).to(device)
    t_out = torch.zeros((npg, solver.ncomp, 16, 16, 16), dtype=solver.torch_dtype, device=device)
    t_flux = torch.zeros((npg, 9, solver.ncomp, 16, 16), dtype=solver.torch_dtype, device=device) \
        if want_flux else None
    t_de = None
    if solver.dual:
        t_de = torch.zeros((npg, 16, 16, 16), dtype=torch.int8, device=device) if de is None else \
            torch.from_numpy(de).to(device)
    t_fail = torch.full((npg,), -1, dtype=torch.int32, device=device) if pg_fail else None
    solver.solve_device(t_in, t_out, params, flux=t_flux, de_out=t_de, pg_fail=t_fail)
    torch.cuda.synchronize()
    res = {"out": t_out.cpu().numpy(), "flux": t_flux.cpu().numpy() if want_flux else None,
           "de": t_de.cpu().numpy() if t_de is not None else None,
           "pg_fail": t_fail.cpu().numpy() if pg_fail else None}
    return res


def mhd_case(npd=2, seed=1, nxt=22, cfl=0.3, **box):
    """Magnetised state (divergence-free face B) cut into Flu/Mag input windows; dt from the fast
    magnetosonic CFL bound |v| + c_f <= |v| + sqrt(c_s^2 + B^2/rho).  ``box`` goes to ic.mhd_box
    (b0, db, mach)."""
    cons, faces = ic.mhd_box(npd, seed=seed, gamma=GAMMA, **box)
    dh = 1.0 / (npd * 16)
    rho = cons[0]
    v = cons[1:4] / rho
    b2 = sum(f * f for f in faces)
    ek = 0.5 * rho * (v ** 2).sum(0)
    p = (GAMMA - 1.0) * (cons[4] - ek - 0.5 * b2)
    cf = np.sqrt(GAMMA * np.abs(p) / rho + b2 / rho)
    dt = cfl * dh / float((np.abs(v).max(0) + cf).max())
    return ic.cut_patch_groups(cons, nxt), ic.cut_mag_windows(faces, nxt), dt, dh


def gpu_solve_mhd(solver, x, b, params, device="cuda:0"):
    """CTU+MHD through FluidSolver.solve_device; returns numpy out/flux/mag_out/ele."""
    import torch
    npg = x.shape[0]
    dt = solver.torch_dtype
    t_in = torch.from_numpy(np.ascontiguousarray(x, dtype=solver.np_dtype)).to(device)
    t_b = torch.from_numpy(np.ascontiguousarray(b, dtype=solver.np_dtype)).to(device)
    t_out = torch.zeros((npg, 5, 16, 16, 16), dtype=dt, device=device)
    t_bout = torch.zeros((npg, 3, 17 * 16 * 16), dtype=dt, device=device)
    t_flux = torch.zeros((npg, 9, 5, 16, 16), dtype=dt, device=device) if params.StoreFlux else None
    t_ele = torch.zeros((npg, 9, 2, 17 * 16), dtype=dt, device=device) if params.StoreElectric else None
    solver.solve_device(t_in, t_out, params, flux=t_flux, mag_in=t_b, mag_out=t_bout, ele=t_ele)
    torch.cuda.synchronize()
    return {"out": t_out.cpu().numpy(), "mag_out": t_bout.cpu().numpy(),
            "flux": None if t_flux is None else t_flux.cpu().numpy(),
            "ele": None if t_ele is None else t_ele.cpu().numpy()}
