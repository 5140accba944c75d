"""Initial conditions on the host (primitive variables of the global field).

These are the harness inputs of the benchmark configurations.  ``blast``
restates setup_problem_blast (src/problems.F90:355-794); the turbulence and
smooth states are seeded synthetic inputs with the shapes, spectra and
amplitudes of the benchmark configurations (the reference has no public
dataset).  Fields are (NZ, NY, NX, nv) float64.
"""
from __future__ import annotations

import math

import numpy as np

HD_NV, MHD_NV = 5, 9
DN, VX, VY, VZ = 0, 1, 2, 3
BX, BY, BZ, BP = 4, 5, 6, 7


def nvars(eqsys: str) -> int:
    return MHD_NV if eqsys.lower().startswith("mhd") or "magneto" in eqsys.lower() else HD_NV


def uniform(mesh, nv: int, dens=1.0, pres=1.0, vel=(0.0, 0.0, 0.0), mag=(0.0, 0.0, 0.0)) -> np.ndarray:
    q = np.zeros(mesh.shape + (nv,))
    q[..., DN] = dens
    q[..., nv - 1] = pres
    q[..., VX], q[..., VY], q[..., VZ] = vel
    if nv == MHD_NV:
        q[..., BX], q[..., BY], q[..., BZ] = mag
    return q


def blast(mesh, nv: int, gamma: float, dens=1.0, ratio=100.0, radius=0.1, csnd=0.40824829046386301635,
          buni=1.0, angle=45.0, nsubgrid=10) -> np.ndarray:
    """setup_problem_blast, src/problems.F90:355-794 (adiabatic: the pressure
    is raised by `ratio` inside `radius`; edge cells get the covered area
    (2D) or sub-grid volume (3D) fraction)."""
    dn_amb = dens
    dn_ovr = dn_amb
    pr_amb = dens * csnd * csnd / gamma
    pr_ovr = pr_amb * ratio
    r2 = radius * radius
    dx, dy, dz = mesh.dx, mesh.dy, mesh.dz
    dxh, dyh = 0.5 * dx, 0.5 * dy
    dzh = 0.5 * dz if mesh.ndims == 3 else 1.0
    dvol = dx * dy * dz
    x, y, z = mesh.cell_centres()
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    xl, xu = np.abs(X) - dxh, np.abs(X) + dxh
    yl, yu = np.abs(Y) - dyh, np.abs(Y) + dyh
    if mesh.ndims == 3:
        zl, zu = np.abs(Z) - dzh, np.abs(Z) + dzh
        rl = xl * xl + yl * yl + zl * zl
        ru = xu * xu + yu * yu + zu * zu
    else:
        rl = xl * xl + yl * yl
        ru = xu * xu + yu * yu
    fc = np.zeros(mesh.shape)
    inside = ru <= r2
    outside = (~inside) & (rl >= r2)
    edge = ~(inside | outside)
    fc[inside] = 1.0
    idx = np.argwhere(edge)
    if mesh.ndims == 3:
        # sub-cells fully inside count 1, cut ones 1/2 (src/problems.F90:
        # 620-657); counted at once rather than accumulated one by one, for
        # a batch of edge cells at a time
        n = max(1, int(nsubgrid))
        fm = (np.arange(n) * 1.0) / n
        fp = (np.arange(1, n + 1) * 1.0) / n
        for s0 in range(0, len(idx), 2048):
            kk, jj, ii = idx[s0:s0 + 2048].T
            a_xl, a_yl, a_zl = xl[kk, jj, ii][:, None], yl[kk, jj, ii][:, None], zl[kk, jj, ii][:, None]
            xb, xt = (a_xl + fm * dx) ** 2, (a_xl + fp * dx) ** 2
            yb, yt = (a_yl + fm * dy) ** 2, (a_yl + fp * dy) ** 2
            zb, zt = (a_zl + fm * dz) ** 2, (a_zl + fp * dz) ** 2
            top = zt[:, :, None, None] + yt[:, None, :, None] + xt[:, None, None, :]
            bot = zb[:, :, None, None] + yb[:, None, :, None] + xb[:, None, None, :]
            full = top <= r2
            half = (~full) & (bot < r2)
            nf = full.reshape(len(kk), -1).sum(axis=1)
            nh = half.reshape(len(kk), -1).sum(axis=1)
            f = (dvol / n ** 3) * (nf + 0.5 * nh)
            fc[kk, jj, ii] = f / dvol
    else:
        for (kk, jj, ii) in idx:
            a_xl, a_xu, a_yl, a_yu = xl[kk, jj, ii], xu[kk, jj, ii], yl[kk, jj, ii], yu[kk, jj, ii]
            rlu = a_xl * a_xl + a_yu * a_yu
            rul = a_xu * a_xu + a_yl * a_yl
            if min(rlu, rul) >= r2:
                xb = math.sqrt(r2 - a_yl ** 2) - a_xl
                yb = math.sqrt(r2 - a_xl ** 2) - a_yl
                sn = 0.5 * math.sqrt(xb ** 2 + yb ** 2) / radius
                ph = 2.0 * math.asin(sn)
                sn = math.sin(ph)
                f = 0.5 * (xb * yb + (ph - sn) * r2)
            elif rlu >= r2:
                yb = math.sqrt(r2 - a_xl ** 2) - a_yl
                yt = math.sqrt(r2 - a_xu ** 2) - a_yl
                sn = 0.5 * math.sqrt(dx ** 2 + (yt - yb) ** 2) / radius
                ph = 2.0 * math.asin(sn)
                sn = math.sin(ph)
                f = 0.5 * ((yt + yb) * dx + (ph - sn) * r2)
            elif rul >= r2:
                xb = math.sqrt(r2 - a_yl ** 2) - a_xl
                xt = math.sqrt(r2 - a_yu ** 2) - a_xl
                sn = 0.5 * math.sqrt((xt - xb) ** 2 + dy ** 2) / radius
                ph = 2.0 * math.asin(sn)
                sn = math.sin(ph)
                f = 0.5 * ((xt + xb) * dy + (ph - sn) * r2)
            else:
                xt = a_xu - math.sqrt(r2 - a_yu ** 2)
                yt = a_yu - math.sqrt(r2 - a_xu ** 2)
                sn = 0.5 * math.sqrt(xt ** 2 + yt ** 2) / radius
                ph = 2.0 * math.asin(sn)
                sn = math.sin(ph)
                f = dvol - 0.5 * (xt * yt - (ph - sn) * r2)
            fc[kk, jj, ii] = f / dvol
    q = np.zeros(mesh.shape + (nv,))
    fa = 1.0 - fc
    q[..., DN] = np.where(inside, dn_ovr, np.where(outside, dn_amb, fc * dn_ovr + fa * dn_amb))
    q[..., nv - 1] = np.where(inside, pr_ovr, np.where(outside, pr_amb, fc * pr_ovr + fa * pr_amb))
    if nv == MHD_NV:
        sn = math.sin(math.pi / 180.0 * angle)
        q[..., BX] = buni * math.sqrt(1.0 - sn * sn)
        q[..., BY] = buni * sn
    return q


def random_phase_field(shape, seed: int, kmin: float = 1.0, kmax: float = 4.0, ncomp: int = 3) -> np.ndarray:
    """Gaussian random-phase field: independent components, mode amplitude^2
    proportional to |k|^-2 on integer wave vectors kmin <= |k| <= kmax of the
    periodic box, phases from numpy's PCG64(seed).  Returns (*shape, ncomp)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    axes = [np.fft.fftfreq(n, d=1.0 / n) for n in shape]
    K = np.meshgrid(*axes, indexing="ij")
    kk = np.sqrt(sum(k * k for k in K))
    shell = (kk >= kmin) & (kk <= kmax)
    amp = np.zeros(shape)
    amp[shell] = 1.0 / kk[shell]
    out = np.empty(tuple(shape) + (ncomp,))
    for c in range(ncomp):
        ph = rng.uniform(0.0, 2.0 * np.pi, size=shape)
        spec = amp * np.exp(1j * ph)
        out[..., c] = np.real(np.fft.ifftn(spec)) * np.prod(shape)
    return out


def turbulence(mesh, gamma: float, seed: int = 0, mach: float = 1.0) -> np.ndarray:
    """Adiabatic MHD box: rho=1, p=1, B=(1,0,0)/sqrt(4 pi), psi=0, velocity a
    random-phase field (|k|^-2 on 1<=|k|<=4) scaled to rms Mach `mach`."""
    q = uniform(mesh, MHD_NV, 1.0, 1.0, mag=(1.0 / math.sqrt(4.0 * math.pi), 0.0, 0.0))
    shp = mesh.shape if mesh.ndims == 3 else mesh.shape[1:]
    v = random_phase_field(shp, seed)
    if mesh.ndims == 2:
        v = v[None]
    cs = math.sqrt(gamma * 1.0 / 1.0)
    vrms = math.sqrt(np.mean(np.sum(v * v, axis=-1)))
    v *= mach * cs / vrms
    q[..., VX:VZ + 1] = v
    return q


def srmhd_turbulence(mesh, seed: int = 0, lorentz_max: float = 10.0) -> np.ndarray:
    """Relativistic MHD box: rho=1, p=1, B=(0.5,0,0), psi=0; velocity the
    random-phase field of `turbulence` rescaled so the largest Lorentz factor
    is `lorentz_max` (max |v|^2 = 1 - 1/lorentz_max^2)."""
    q = uniform(mesh, MHD_NV, 1.0, 1.0, mag=(0.5, 0.0, 0.0))
    shp = mesh.shape if mesh.ndims == 3 else mesh.shape[1:]
    v = random_phase_field(shp, seed)
    if mesh.ndims == 2:
        v = v[None]
    vmax = math.sqrt(1.0 - 1.0 / lorentz_max ** 2)
    v *= vmax / math.sqrt(np.max(np.sum(v * v, axis=-1)))
    q[..., VX:VZ + 1] = v
    return q


def smooth_mhd(mesh, seed: int = 0) -> np.ndarray:
    """2D smooth MHD state: rho = 1 + 0.01 * (random Fourier modes with
    integer 1<=|k|<=4, normalised to max 1), p = 1,
    v = 0.1 (-sin 2 pi y, sin 2 pi x, 0), B = 0.1 (-sin 2 pi y, sin 4 pi x, 0)."""
    q = uniform(mesh, MHD_NV)
    x, y, _ = mesh.cell_centres()
    Y, X = np.meshgrid(y, x, indexing="ij")
    f = random_phase_field(mesh.shape[1:], seed, ncomp=1)[..., 0]
    f = f / np.max(np.abs(f))
    q[0, ..., DN] = 1.0 + 0.01 * f
    q[0, ..., VX] = -0.1 * np.sin(2 * np.pi * Y)
    q[0, ..., VY] = 0.1 * np.sin(2 * np.pi * X)
    q[0, ..., BX] = -0.1 * np.sin(2 * np.pi * Y)
    q[0, ..., BY] = 0.1 * np.sin(4 * np.pi * X)
    return q
