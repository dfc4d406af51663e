"""Seeded synthetic initial conditions on a periodic uniform grid, cut into patch-group windows.

The reference benchmarks its solver only inside whole simulations (test problems under
``example/test_problem/Hydro``).  These generators produce the same kinds of states — a lognormal
turbulent-like field, a Kelvin-Helmholtz shear layer
(src/TestProblem/Hydro/KelvinHelmholtzInstability/Init_TestProb_Hydro_KelvinHelmholtzInstability.cpp),
a blast wave on a lognormal background, a linear acoustic wave
(src/TestProblem/Hydro/AcousticWave) — on a periodic box of ``pg_per_dim**3`` patch groups, and
:func:`cut_patch_groups` builds the ``[NPG][NCOMP][FLU_NXT^3]`` input windows exactly as GAMER's
ghost-zone preparation would for a single refinement level with periodic boundaries.

All arrays are float64 numpy; callers cast to the solver precision.
"""
from __future__ import annotations

import numpy as np

PS2 = 16


def _smooth_gaussian(rng, n, std, kmax=3):
    """White noise low-passed to the Fourier modes |k_i| <= kmax, rescaled to the given std."""
    w = rng.standard_normal((n, n, n))
    f = np.fft.fftn(w)
    k = np.fft.fftfreq(n, d=1.0 / n)
    kx, ky, kz = np.meshgrid(k, k, k, indexing="ij")
    mask = (np.abs(kx) <= kmax) & (np.abs(ky) <= kmax) & (np.abs(kz) <= kmax)
    g = np.real(np.fft.ifftn(f * mask))
    g -= g.mean()
    s = g.std()
    return g * (std / s) if s > 0 else g


def prim2cons(rho, vx, vy, vz, p, gamma, dual=False):
    """Primitive -> conserved [5(+1), ...]; the dual variable is DE_ENPY's P*rho^(1-gamma)."""
    e = p / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    u = [rho, rho * vx, rho * vy, rho * vz, e]
    if dual:
        u.append(p * rho ** (1.0 - gamma))
    return np.stack(u)


def lognormal_box(pg_per_dim, seed, gamma=5.0 / 3.0, dual=False):
    """rho = exp(N(0,0.3)) smoothed to |k|<=3, v ~ U(-1,1)*c_s per component, P = exp(N(0,0.2))."""
    rng = np.random.default_rng(seed)
    n = pg_per_dim * PS2
    rho = np.exp(_smooth_gaussian(rng, n, 0.3))
    p = np.exp(rng.normal(0.0, 0.2, (n, n, n)))
    cs = np.sqrt(gamma * p / rho)
    v = rng.uniform(-1.0, 1.0, (3, n, n, n)) * cs
    return prim2cons(rho, v[0], v[1], v[2], p, gamma, dual)


def kelvin_helmholtz_box(pg_per_dim, seed, gamma=5.0 / 3.0, dual=False):
    """Shear layer: rho 2 in |y-1/2|<1/4 else 1, v_x +-0.5, v_y = 0.01 sin(4 pi x) (+ seeded noise
    of 1e-4 to break symmetry), P = 2.5."""
    rng = np.random.default_rng(seed)
    n = pg_per_dim * PS2
    x = (np.arange(n) + 0.5) / n
    X, Y, _ = np.meshgrid(x, x, x, indexing="ij")
    inner = np.abs(Y - 0.5) < 0.25
    rho = np.where(inner, 2.0, 1.0)
    vx = np.where(inner, 0.5, -0.5)
    vy = 0.01 * np.sin(4.0 * np.pi * X) + 1e-4 * rng.standard_normal((n, n, n))
    vz = np.zeros_like(vx)
    p = np.full_like(rho, 2.5)
    return prim2cons(rho, vx, vy, vz, p, gamma, dual)


def blast_box(pg_per_dim, seed, gamma=5.0 / 3.0, dual=True, jump=1.0e3):
    """Lognormal background with a central sphere of density and pressure raised by ``jump``;
    background velocities at Mach ~10 relative to the background sound speed."""
    rng = np.random.default_rng(seed)
    n = pg_per_dim * PS2
    rho = np.exp(_smooth_gaussian(rng, n, 0.3))
    p = np.exp(rng.normal(0.0, 0.2, (n, n, n))) * 1e-2
    x = (np.arange(n) + 0.5) / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    r = np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2 + (Z - 0.5) ** 2)
    inside = r < 0.1
    rho = np.where(inside, rho * jump, rho)
    p = np.where(inside, p * jump * 1e2, p)
    cs = np.sqrt(gamma * p / rho)
    v = rng.uniform(-1.0, 1.0, (3, n, n, n)) * 10.0 * np.sqrt(gamma * 1e-2)
    v = np.where(inside[None], 0.0, v)
    return prim2cons(rho, v[0], v[1], v[2], p, gamma, dual)


def acoustic_wave_box(pg_per_dim, amp=1e-4, gamma=5.0 / 3.0, rho0=1.0, p0=None, direction=0):
    """Linear acoustic wave along ``direction``: one wavelength across the box
    (src/TestProblem/Hydro/AcousticWave; rho0 = 1, c_s = 1)."""
    n = pg_per_dim * PS2
    if p0 is None:
        p0 = rho0 / gamma  # c_s = 1
    cs = np.sqrt(gamma * p0 / rho0)
    x = (np.arange(n) + 0.5) / n
    grids = np.meshgrid(x, x, x, indexing="ij")
    phase = np.sin(2.0 * np.pi * grids[direction])
    rho = rho0 * (1.0 + amp * phase)
    v = [np.zeros_like(rho) for _ in range(3)]
    v[direction] = cs * amp * phase
    p = p0 * (1.0 + gamma * amp * phase)
    return prim2cons(rho, v[0], v[1], v[2], p, gamma)


def smooth_box(pg_per_dim, seed, gamma=5.0 / 3.0, amp=0.1):
    """Smooth state for gradient checks: density, velocity and pressure made of a few random
    long-wavelength Fourier modes (|k| <= 2) around rho = P = 1."""
    rng = np.random.default_rng(seed)
    n = pg_per_dim * PS2
    rho = 1.0 + amp * _smooth_gaussian(rng, n, 1.0, kmax=2)
    p = 1.0 + amp * _smooth_gaussian(rng, n, 1.0, kmax=2)
    v = [2.0 * amp * _smooth_gaussian(rng, n, 1.0, kmax=2) for _ in range(3)]
    return prim2cons(rho, v[0], v[1], v[2], p, gamma)


def supersonic_separable_box(pg_per_dim, gamma=5.0 / 3.0, amp=0.1, mach=2.0, seed=0):
    """Smooth state whose MHM+PLM+HLLC update is free of branch switches under small perturbations
    (for finite-difference checks of the adjoint): a uniform flow at Mach ``mach`` along every axis
    (all faces supersonic, so HLLC returns the upwind flux whatever the wave-speed estimates) plus
    separable sinusoids in rho, v and P whose extrema sit at cell centres (generalized MinMod keeps
    a margin of >= 10% to its branch changes)."""
    rng = np.random.default_rng(seed)
    n = pg_per_dim * PS2
    xc = (np.arange(n) + 0.5) / n
    # sin(2 pi x + phi) has extrema at cell centres when phi = pi/2 - 2 pi (c + 1/2)/n, c integer
    def mode(c):
        return np.sin(2.0 * np.pi * xc + np.pi / 2 - 2.0 * np.pi * (c + 0.5) / n)
    def field(base, a):
        cs = rng.integers(0, n, size=3)
        X, Y, Z = np.meshgrid(mode(cs[0]), mode(cs[1]), mode(cs[2]), indexing="ij")
        return base + a * (X + Y + Z) / 3.0
    rho = field(1.0, amp)
    p = field(1.0, amp)
    c0 = np.sqrt(gamma)
    v = [field(mach * c0, amp * c0) for _ in range(3)]
    return prim2cons(rho, v[0], v[1], v[2], p, gamma)


def oblique_wave_box(pg_per_dim, gamma=5.0 / 3.0, amp=0.1, mach=2.0, seed=0):
    """Supersonic flow plus sinusoids that depend on s = i + j + k only (a plane wave along the box
    diagonal).  A translation-invariant scheme keeps every field a function of s to the last bit,
    so a step evaluates only ~3n distinct limiter cases per axis instead of n^3: over several steps
    the branch switches stay far from the state, which finite-difference checks need."""
    rng = np.random.default_rng(seed)
    n = pg_per_dim * PS2
    i = np.arange(n)
    s = (i[:, None, None] + i[None, :, None] + i[None, None, :]).astype(np.float64)

    def field(base, a):
        m = rng.integers(1, 3, size=2)
        ph = rng.uniform(0.0, 2.0 * np.pi, size=2)
        return base + a * 0.5 * (np.sin(2.0 * np.pi * m[0] * s / n + ph[0]) +
                                 np.sin(2.0 * np.pi * m[1] * s / n + ph[1]))
    rho = field(1.0, amp)
    p = field(1.0, amp)
    c0 = np.sqrt(gamma)
    v = [field(mach * c0, amp * c0) for _ in range(3)]
    return prim2cons(rho, v[0], v[1], v[2], p, gamma)


def mhd_box(pg_per_dim, seed, gamma=5.0 / 3.0, b0=(0.8, 0.6, 0.5), db=0.6, mach=0.5, kmax=4):
    """Magnetised lognormal-like state (plasma beta ~ 1) with a divergence-free face-centred field.

    Returns (cons [5][n][n][n], (bx, by, bz)) with bx[i][j][k] the x-field on the left x-face of cell
    (i, j, k) (likewise by, bz), all indexed [x][y][z].  B is a uniform field b0 plus the discrete curl
    of a random smooth edge-centred vector potential, so the discrete divergence of every cell vanishes
    to round-off.  Total energy includes 1/2 |B_cc|^2 with B_cc the mean of the two faces (the
    reference's MHD_GetCellCenteredBField)."""
    rng = np.random.default_rng(seed)
    n = pg_per_dim * PS2
    rho = np.exp(_smooth_gaussian(rng, n, 0.3))
    p = np.exp(_smooth_gaussian(rng, n, 0.2))
    cs = np.sqrt(gamma * p / rho)
    v = [mach * cs * _smooth_gaussian(rng, n, 1.0) for _ in range(3)]
    # modes |k_i| <= kmax: a forward difference of A is ~ 2 pi kmax / n of A, so dB ~ db
    a = [db * n / (2.0 * np.pi * kmax) * _smooth_gaussian(rng, n, 1.0, kmax=kmax) for _ in range(3)]
    ax, ay, az = a

    def d(f, axis):      # forward difference f[i+1] - f[i] along axis (periodic)
        return np.roll(f, -1, axis=axis) - f
    # the dh factors of the discrete curl cancel against A's scaling; B = curl A in cell units
    bx = b0[0] + d(az, 1) - d(ay, 2)
    by = b0[1] + d(ax, 2) - d(az, 0)
    bz = b0[2] + d(ay, 0) - d(ax, 1)
    bcc = [0.5 * (bx + np.roll(bx, -1, 0)), 0.5 * (by + np.roll(by, -1, 1)), 0.5 * (bz + np.roll(bz, -1, 2))]
    cons = prim2cons(rho, v[0], v[1], v[2], p, gamma)
    cons[4] += 0.5 * (bcc[0] ** 2 + bcc[1] ** 2 + bcc[2] ** 2)
    return cons, (bx, by, bz)


def cut_mag_windows(faces, nxt):
    """(bx, by, bz) of a periodic box -> Mag_Array_In [NPG][3][(nxt+1)*nxt*nxt] in GAMER's layout
    (IDX321_BX/BY/BZ: x fastest; the component's own axis has nxt+1 faces), patch groups in the order
    of :func:`cut_patch_groups`."""
    n = faces[0].shape[0]
    npd = n // PS2
    g = (nxt - PS2) // 2
    pads = [np.pad(f, ((g, g + 1), (g, g + 1), (g, g + 1)), mode="wrap") for f in faces]
    out = np.empty((npd ** 3, 3, (nxt + 1) * nxt * nxt), faces[0].dtype)
    p = 0
    for pz in range(npd):
        for py in range(npd):
            for px in range(npd):
                o = (px * PS2, py * PS2, pz * PS2)
                for c in range(3):
                    ext = [nxt, nxt, nxt]
                    ext[c] += 1
                    w = pads[c][o[0]:o[0] + ext[0], o[1]:o[1] + ext[1], o[2]:o[2] + ext[2]]
                    out[p, c] = np.transpose(w, (2, 1, 0)).reshape(-1)
                p += 1
    return out


def mag_out_faces(mag_out):
    """Mag_Array_Out [NPG][3][17*16*16] -> list of three arrays [NPG][nz][ny][nx] per component
    (the component's own axis has 17 faces)."""
    npg = mag_out.shape[0]
    shapes = [(PS2, PS2, PS2 + 1), (PS2, PS2 + 1, PS2), (PS2 + 1, PS2, PS2)]
    return [mag_out[:, c].reshape((npg,) + shapes[c]) for c in range(3)]


def div_b(mag_out):
    """Per-cell discrete divergence (in cell units) of each patch group's output field: [NPG][16][16][16]."""
    fx, fy, fz = mag_out_faces(mag_out)
    return (fx[..., 1:] - fx[..., :-1]) + (fy[:, :, 1:, :] - fy[:, :, :-1, :]) + (fz[:, 1:] - fz[:, :-1])


# offsets (x, y, z) in patch units of the eight patches of a patch group, by LocalID
# (TABLE_02, src/Tables/Table_02.cpp)
LOCAL_ID_OFFSET = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (0, 1, 1), (1, 0, 1), (1, 1, 1)]


def patches_from_output(flu_out, mag_out=None):
    """Solver outputs [NPG][NCOMP][16][16][16] (and Mag_Array_Out [NPG][3][17*16*16]) -> the dt solver's
    patch arrays [8*NPG][5][8^3] (and [8*NPG][3][9*8*8]), patches in LocalID order, as dt_Prepare_Flu
    lays them out (src/Miscellaneous/dt_Prepare_Flu.cpp:23-49)."""
    npg = flu_out.shape[0]
    flu = np.empty((8 * npg, 5, 8, 8, 8), flu_out.dtype)
    mag = None if mag_out is None else np.empty((8 * npg, 3, 9 * 8 * 8), mag_out.dtype)
    faces = None if mag_out is None else mag_out_faces(mag_out)
    for lid, (ox, oy, oz) in enumerate(LOCAL_ID_OFFSET):
        x, y, z = 8 * ox, 8 * oy, 8 * oz
        flu[lid::8] = flu_out[:, :5, z:z + 8, y:y + 8, x:x + 8]
        if faces is not None:
            mag[lid::8, 0] = faces[0][:, z:z + 8, y:y + 8, x:x + 9].reshape(npg, -1)
            mag[lid::8, 1] = faces[1][:, z:z + 8, y:y + 9, x:x + 8].reshape(npg, -1)
            mag[lid::8, 2] = faces[2][:, z:z + 9, y:y + 8, x:x + 8].reshape(npg, -1)
    return flu.reshape(8 * npg, 5, 512), mag


def to_device_layout(box):
    """numpy box [v][x][y][z] -> [v][z][y][x] (x fastest), the layout of gb_box_* and gamer_b200.adjoint."""
    return np.ascontiguousarray(np.transpose(box, (0, 3, 2, 1)))


def from_device_layout(box):
    return np.ascontiguousarray(np.transpose(box, (0, 3, 2, 1)))


def cut_patch_groups(box, nxt):
    """[NCOMP][n][n][n] periodic box -> [NPG][NCOMP][nxt][nxt][nxt] input windows, patch groups in
    x-fastest order (PG index = (pz*npd + py)*npd + px)."""
    nc, n = box.shape[0], box.shape[1]
    npd = n // PS2
    g = (nxt - PS2) // 2
    padded = np.pad(box, ((0, 0), (g, g), (g, g), (g, g)), mode="wrap")
    out = np.empty((npd ** 3, nc, nxt, nxt, nxt), box.dtype)
    p = 0
    # box arrays are indexed [var][x][y][z]; the solver layout is [var][z][y][x] (x fastest)
    for pz in range(npd):
        for py in range(npd):
            for px in range(npd):
                w = padded[:, px * PS2:px * PS2 + nxt, py * PS2:py * PS2 + nxt, pz * PS2:pz * PS2 + nxt]
                out[p] = np.transpose(w, (0, 3, 2, 1))
                p += 1
    return out


def assemble_box(pg_out, npd):
    """Inverse of the interior part of :func:`cut_patch_groups`: [NPG][NCOMP][16][16][16] (z,y,x)
    -> [NCOMP][n][n][n] (x,y,z)."""
    nc = pg_out.shape[1]
    n = npd * PS2
    box = np.empty((nc, n, n, n), pg_out.dtype)
    p = 0
    for pz in range(npd):
        for py in range(npd):
            for px in range(npd):
                box[:, px * PS2:(px + 1) * PS2, py * PS2:(py + 1) * PS2, pz * PS2:(pz + 1) * PS2] = \
                    np.transpose(pg_out[p], (0, 3, 2, 1))
                p += 1
    return box


def cfl_dt(box, gamma, dh, cfl=0.5):
    """dt = cfl * dh / max_d max_cells(|v_d| + c_s) (src/Model_Hydro/CPU_Hydro/CPU_dtSolver_HydroCFL.cpp:205-207)."""
    rho = box[0]
    v = box[1:4] / rho
    ek = 0.5 * rho * (v ** 2).sum(0)
    p = (gamma - 1.0) * (box[4] - ek)
    cs = np.sqrt(gamma * p / rho)
    smax = max(float((np.abs(v[d]) + cs).max()) for d in range(3))
    return cfl * dh / smax
