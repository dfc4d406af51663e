"""GPU parity of the coarse-to-fine interpolation of the AMR ghost-zone fill (gb_interpolate_device)
against the reference's own Interpolate() (src/Interpolation/Interpolate.cpp:90, Int_*.cpp and
Interpolate_Iterate), compiled from source into oracle/_ref, and of the window assembly of a two-level
layout (gb_assemble_windows_device) against the reference's side-by-side interpolation.

Every comparison is bit for bit: the device evaluates each operation of the reference, explicitly
rounded (no FMA contraction, IEEE division)."""
import zlib

import numpy as np
import pytest

import pyoracle as po
from gamer_b200 import ic
from gamer_b200.fluid import INTERP_FAILED, assemble_windows_device, interpolate_device

pytestmark = pytest.mark.gpu

SCHEMES = ["minmod3d", "minmod1d", "vanleer", "cquad", "quad", "cquar", "quar"]
GHOST = {"cquar": 2, "quar": 2}


def _to_dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("mono,opp", [(True, False), (False, False), (True, True)])
def test_interpolate_matches_reference(cuda_device, scheme, prec, mono, opp):
    """Random regions (smooth positive fields with bumps, and a signed component for the
    opposite-sign rule) on a batch of 3, a range away from the array origin on both sides; cells of
    the fine array outside the range stay as they were."""
    import torch
    dt = np.float64 if prec == "fp64" else np.float32
    g = GHOST.get(scheme, 1)
    rng = np.random.default_rng(zlib.crc32(f"{scheme}{prec}{mono}{opp}".encode()))
    nb, nc = 3, 3
    csize = (11 + 2 * g, 9 + 2 * g, 8 + 2 * g)                           # (x, y, z)
    cstart, crange = (g, g + 1, g), (9, 6, 7)
    fstart, fsize = (1, 0, 2), (20, 14, 17)
    c = np.empty((nb, nc, csize[2], csize[1], csize[0]), dt)
    c[:, 0] = np.exp(rng.normal(0, 0.5, c[:, 0].shape))
    c[:, 1] = 1.0 + 0.3 * np.sin(np.arange(csize[0]) * 0.9)[None, None, None, :] * rng.random(c[:, 1].shape)
    c[:, 2] = rng.normal(0, 1, c[:, 2].shape)                          # changes sign
    f0 = np.full((nb, nc, fsize[2], fsize[1], fsize[0]), -7.25, dt)
    fr = f0.copy()
    assert po.ref_interpolate(c, fr, scheme, cstart, crange, fstart, monotonic=mono, opp_sign_0th_order=opp) == 0
    tf = _to_dev(f0)
    interpolate_device(_to_dev(c), tf, scheme, cstart, crange, fstart, monotonic=mono, opp_sign_0th_order=opp)
    torch.cuda.synchronize()
    gf = tf.cpu().numpy()
    assert np.array_equal(gf, fr), float(np.nanmax(np.abs(gf - fr)))
    assert np.count_nonzero(gf != -7.25) == nb * nc * 8 * np.prod(crange)


def _hydro_coarse(nb, csize, seed, jump):
    """Conserved hydro states with steep density / pressure steps (a factor `jump`) and fast flow, so
    that interpolated children of some parents are unphysical in conserved variables."""
    n = csize[0]
    rng = np.random.default_rng(seed)
    out = []
    for b in range(nb):
        x = np.arange(n)
        X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
        r = np.sqrt((X - n / 2 + rng.random()) ** 2 + (Y - n / 2) ** 2 + (Z - n / 2) ** 2)
        rho = np.where(r < n / 4, jump, 1.0) * np.exp(rng.normal(0, 0.05, r.shape))
        p = np.where(r < n / 4 + 0.7, jump, 1e-3) * np.exp(rng.normal(0, 0.05, r.shape))
        v = rng.normal(0, 3.0, (3,) + r.shape)
        u = ic.prim2cons(rho, v[0], v[1], v[2], p, 5.0 / 3.0)           # [5][x][y][z]
        out.append(np.transpose(u, (0, 3, 2, 1)))                       # [5][z][y][x]
    return np.stack(out)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("scheme,int_prim,mono_iter", [("cquad", True, 10), ("quad", True, 10), ("cquar", True, 10),
                                                        ("quar", True, 10), ("cquad", False, 10), ("cquar", False, 4),
                                                        ("cquad", True, 0), ("minmod3d", True, 0)])
def test_interpolate_iterate_matches_reference(cuda_device, prec, scheme, int_prim, mono_iter):
    """Interpolate_Iterate (the hydro ghost-zone path): parents with an unphysical child are redone in
    primitive variables and with a reduced monotonicity coefficient, each on its own (INTERP_MASK);
    the result equals the reference's bit for bit and differs from the single plain attempt."""
    import torch
    dt = np.float64 if prec == "fp64" else np.float32
    g = GHOST.get(scheme, 1)
    n = 12 + 2 * g
    c = _hydro_coarse(2, (n, n, n), seed=5, jump=1e3).astype(dt)
    crange = (12, 12, 12)
    f0 = np.zeros((2, 5, 24, 24, 24), dt)
    fr = f0.copy()
    kw = dict(iterate=True, int_prim=int_prim, mono_max_iter=mono_iter, min_pres=1e-8)
    assert po.ref_interpolate(c, fr, scheme, (g, g, g), crange, **kw) == 0
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    tf = _to_dev(f0)
    interpolate_device(_to_dev(c), tf, scheme, (g, g, g), crange, status=st, **kw)
    torch.cuda.synchronize()
    assert st.item() == 0
    assert np.array_equal(tf.cpu().numpy(), fr)
    # the iterations acted: a single conserved-variable attempt differs
    fp = f0.copy()
    po.ref_interpolate(c, fp, scheme, (g, g, g), crange)
    assert not np.array_equal(fp, fr)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_interpolate_iterate_reports_failure(cuda_device, prec):
    """Parents whose children stay unphysical after every attempt (conserved variables only, the
    coefficient reduced to zero): the reference aborts the run; the device sets GB_INTERP_FAILED."""
    import torch
    dt = np.float64 if prec == "fp64" else np.float32
    c = _hydro_coarse(2, (14, 14, 14), seed=5, jump=1e3).astype(dt)
    fr = np.zeros((2, 5, 24, 24, 24), dt)
    kw = dict(iterate=True, int_prim=False, mono_max_iter=10, min_pres=1e-8)
    assert po.ref_interpolate(c, fr, "quad", (1, 1, 1), (12, 12, 12), **kw) == 2
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    interpolate_device(_to_dev(c), _to_dev(np.zeros_like(fr)), "quad", (1, 1, 1), (12, 12, 12), status=st, **kw)
    torch.cuda.synchronize()
    assert st.item() & INTERP_FAILED


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_two_level_ghost_fill_matches_reference_side_by_side(cuda_device, prec):
    """A two-level layout: a 2x2x2 block of fine patch groups inside a coarse box.  Each fine window
    (FLU_NXT = 20) takes its interior and the sides towards the other fine patch groups at the fine
    level, and every other side from the coarse level.  Device: the whole window interpolated from its
    parents (gb_interpolate_device, Interpolate_Iterate), then assembled (gb_assemble_windows_device).
    Reference: Interpolate() called on each of the 26 sides separately, as InterpolateGhostZone does,
    and the same-level copies done on the host -- equal bit for bit."""
    import torch
    dt = np.float64 if prec == "fp64" else np.float32
    nxt, gh = 20, 2
    cg = 1                                                               # CQuad's CGhost
    coarse = ic.lognormal_box(2, seed=11)                                # [5][x][y][z] 32^3 coarse cells
    coarse = np.transpose(coarse, (0, 3, 2, 1)).astype(dt)               # [5][z][y][x]
    fine_box = ic.lognormal_box(2, seed=12)                              # the 2x2x2 fine patch groups
    fine_box = np.transpose(fine_box, (0, 3, 2, 1)).astype(dt)
    origin = np.array([8, 8, 8])                                         # coarse cell under fine cell 0 (z, y, x)
    pgs = [(pz, py, px) for pz in range(2) for py in range(2) for px in range(2)]
    npg = len(pgs)
    fine = np.stack([fine_box[:, 16 * pz:16 * pz + 16, 16 * py:16 * py + 16, 16 * px:16 * px + 16]
                     for pz, py, px in pgs])
    nbr = np.full((npg, 27), -1, np.int32)
    for p, (pz, py, px) in enumerate(pgs):
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    q = (pz + dz, py + dy, px + dx)
                    if q in pgs:
                        nbr[p, (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)] = pgs.index(q)
    # coarse region of each window: its 10^3 parents plus CGhost
    nw = nxt // 2
    creg = np.stack([coarse[:, origin[0] + 8 * pz - 1 - cg: origin[0] + 8 * pz - 1 + nw + cg,
                            origin[1] + 8 * py - 1 - cg: origin[1] + 8 * py - 1 + nw + cg,
                            origin[2] + 8 * px - 1 - cg: origin[2] + 8 * px - 1 + nw + cg] for pz, py, px in pgs])
    kw = dict(iterate=True, int_prim=True, mono_max_iter=10, min_pres=0.0)
    # device
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    tcint = torch.zeros((npg, 5, nxt, nxt, nxt), dtype=torch.float64 if prec == "fp64" else torch.float32,
                        device="cuda")
    interpolate_device(_to_dev(creg), tcint, "cquad", (cg, cg, cg), (nw, nw, nw), status=st, **kw)
    twin = torch.empty_like(tcint)
    assemble_windows_device(_to_dev(fine), _to_dev(nbr), tcint, twin)
    torch.cuda.synchronize()
    assert st.item() == 0
    got = twin.cpu().numpy()
    # reference: side by side
    want = np.empty_like(got)
    for p in range(npg):
        want[p, :, gh:gh + 16, gh:gh + 16, gh:gh + 16] = fine[p]
        for s in range(27):
            if s == 13:
                continue
            dz, dy, dx = s // 9 - 1, (s // 3) % 3 - 1, s % 3 - 1
            sl = [slice(0, gh) if d < 0 else slice(gh + 16, nxt) if d > 0 else slice(gh, gh + 16) for d in (dz, dy, dx)]
            q = nbr[p, s]
            if q >= 0:
                src = [slice(16 - gh, 16) if d < 0 else slice(0, gh) if d > 0 else slice(0, 16) for d in (dz, dy, dx)]
                want[p][(slice(None), *sl)] = fine[q][(slice(None), *src)]
                continue
            # the side's parents (coarse cells of the window, by fine index // 2) and their fine block
            lo = [x.start // 2 for x in sl]
            hi = [(x.stop - 1) // 2 + 1 for x in sl]
            cs = [h - l for l, h in zip(lo, hi)]
            reg = creg[p][:, lo[0]:hi[0] + 2 * cg, lo[1]:hi[1] + 2 * cg, lo[2]:hi[2] + 2 * cg]
            fblk = np.zeros((1, 5, 2 * cs[0], 2 * cs[1], 2 * cs[2]), dt)
            assert po.ref_interpolate(reg[None], fblk, "cquad", (cg, cg, cg), cs[::-1], **kw) == 0
            off = [x.start - 2 * l for x, l in zip(sl, lo)]
            want[p][(slice(None), *sl)] = fblk[0][:, off[0]:off[0] + sl[0].stop - sl[0].start,
                                                    off[1]:off[1] + sl[1].stop - sl[1].start,
                                                    off[2]:off[2] + sl[2].stop - sl[2].start]
    assert np.array_equal(got, want)
