"""FP64 tape of the forward stage update (test infrastructure, CPU only).

A differentiable restatement, in torch FP64 on the host, of the stage update
whose discrete adjoint the GPU library implements: adiabatic HD or GLM-MHD,
WENO-Z reconstruction (src/interpolations.F90:1937-2083) or TVD with the
positivity halving (729-848) and the limiters of 4684-4877, the HLL solver
(and for HD the HLLC solver, src/schemes.F90:1366-1513)
(src/schemes.F90:1248-1341, 3163-3274 with the GLM averaging), the flux
difference (src/evolution.F90:1898-1977), the SSPRK stage combinations of
src/evolution.F90 (628-770 rk2, 1005-1208 rk3) and the psi decay
(src/evolution.F90:749), on a uniform periodic mesh.  torch.autograd over it
gives the reference gradient that the adjoint kernels are checked against.

Per step the time step and the GLM speed cmax come from the state at the
start of the step (new_time_step, src/evolution.F90:379-493) and are held
constant in the derivative, as the adjoint does.  Branches follow the GPU
kernels' selections: min/max pick the second operand on ties, |x| has
derivative sign(x).

Only tests import this module; it is not part of the library.
"""
from __future__ import annotations

import math

import torch

DN, VX, VY, VZ = 0, 1, 2, 3
BX, BY, BZ, BP = 4, 5, 6, 7

_ROT = {0: (0, 1, 2), 1: (1, 2, 0), 2: (2, 0, 1)}


class Scheme:
    def __init__(self, nv: int, ndims: int, gamma: float, cfl: float, dx, alpha: float = 2.0,
                 eps: float = 2.220446049250313e-16, time_advance: str = "rk3", reconstruction: str = "weno5z",
                 limiter: str = "mc", riemann: str = "hll"):
        self.nv, self.ndims = nv, ndims
        self.mhd = nv == 9
        self.gamma = gamma
        self.gammam1 = gamma - 1.0
        self.gammam1i = 1.0 / (gamma - 1.0)
        self.cfl = cfl
        self.dx = list(dx)  # per direction x, y, z
        self.dx_min = min(self.dx[:ndims])
        self.eps = eps
        self.decay = math.exp(-alpha * cfl)
        self.ta = time_advance
        self.pr = nv - 1
        self.rec = reconstruction
        self.lim = limiter
        if riemann == "hllc" and self.mhd:
            raise ValueError("the tape has HLLC for HD only")
        self.rs = riemann

    # ---- equations -------------------------------------------------------------
    def prim2cons(self, q):
        rho, vx, vy, vz, p = q[DN], q[VX], q[VY], q[VZ], q[self.pr]
        mx, my, mz = rho * vx, rho * vy, rho * vz
        ek = 0.5 * (mx * vx + my * vy + mz * vz)
        ei = self.gammam1i * p
        if not self.mhd:
            return [rho, mx, my, mz, ei + ek]
        bx, by, bz, bp = q[BX], q[BY], q[BZ], q[BP]
        em = 0.5 * (bx * bx + by * by + bz * bz)
        return [rho, mx, my, mz, bx, by, bz, bp, ei + ek + em]

    def cons2prim(self, u):
        rho = u[DN]
        vx, vy, vz = u[VX] / rho, u[VY] / rho, u[VZ] / rho
        ek = 0.5 * (u[VX] * vx + u[VY] * vy + u[VZ] * vz)
        if not self.mhd:
            return [rho, vx, vy, vz, self.gammam1 * (u[4] - ek)]
        bx, by, bz, bp = u[BX], u[BY], u[BZ], u[BP]
        em = 0.5 * (bx * bx + by * by + bz * bz)
        return [rho, vx, vy, vz, bx, by, bz, bp, self.gammam1 * (u[8] - (ek + em))]

    def fluxspeed(self, q, u, cmax2):
        vx, p, rho = q[VX], q[self.pr], q[DN]
        if not self.mhd:
            f = [u[VX], vx * u[VX] + p, vx * u[VY], vx * u[VZ], vx * (u[4] + p)]
            cs = torch.sqrt(self.gamma * p / rho)
            return f, vx - cs, vx + cs
        bx, by, bz = q[BX], q[BY], q[BZ]
        bx2, by2, bz2 = bx * bx, by * by, bz * bz
        bb = bx2 + by2 + bz2
        vb = vx * bx + q[VY] * by + q[VZ] * bz
        pt = p + 0.5 * bb
        f = [u[VX], vx * u[VX] - bx2 + pt, vx * u[VY] - bx * by, vx * u[VZ] - bx * bz, q[BP],
             vx * by - bx * q[VY], vx * bz - bx * q[VZ], cmax2 * bx, vx * (u[8] + pt) - bx * vb]
        fa = self.gamma * p
        fb = fa + bb
        fc = fb * fb - 4.0 * fa * bx2
        pos = fc > 0
        fcs = torch.where(pos, fc, torch.ones_like(fc))
        cf = torch.where(pos, torch.sqrt(0.5 * (fb + torch.sqrt(fcs)) / rho), torch.sqrt(0.5 * fb / rho))
        return f, vx - cf, vx + cf

    def cell_speed(self, q):
        vv = q[VX] ** 2 + q[VY] ** 2 + q[VZ] ** 2
        if not self.mhd:
            c = torch.sqrt(self.gamma * q[self.pr] / q[DN])
        else:
            bb = q[BX] ** 2 + q[BY] ** 2 + q[BZ] ** 2
            c = torch.sqrt((self.gamma * q[self.pr] + bb) / q[DN])
        return torch.sqrt(vv) + c

    def hll(self, ql, qr, cmax, cmax2):
        ql, qr = list(ql), list(qr)
        if self.mhd:
            bx = 0.5 * ((qr[BX] + ql[BX]) - (qr[BP] - ql[BP]) / cmax)
            bp = 0.5 * ((qr[BP] + ql[BP]) - (qr[BX] - ql[BX]) * cmax)
            ql[BX] = qr[BX] = bx
            ql[BP] = qr[BP] = bp
        ul, ur = self.prim2cons(ql), self.prim2cons(qr)
        fl, clm, clp = self.fluxspeed(ql, ul, cmax2)
        fr, crm, crp = self.fluxspeed(qr, ur, cmax2)
        sl = torch.where(clm < crm, clm, crm)
        sr = torch.where(clp > crp, clp, crp)
        left, right = sl >= 0, sr <= 0
        mid = ~(left | right)
        srml = torch.where(mid, sr - sl, torch.ones_like(sl))
        out = []
        for v in range(self.nv):
            wl = sl * ul[v] - fl[v]
            wr = sr * ur[v] - fr[v]
            fm = (sl * wr - sr * wl) / srml
            out.append(torch.where(left, fl[v], torch.where(right, fr[v], fm)))
        return out

    def hllc(self, ql, qr, cmax, cmax2):
        """HD HLLC (src/schemes.F90:1366-1513) in the GPU solver's operation
        order: the HLL speeds, the contact speed sm and pressure from the
        HLL fluxes w = s u - f, the star state of the side sm points away
        from (the flux -w_x of the momentum only when sm = 0).  Unused
        branches divide by 1 so their zero gradients stay finite."""
        ul, ur = self.prim2cons(ql), self.prim2cons(qr)
        fl, clm, clp = self.fluxspeed(ql, ul, cmax2)
        fr, crm, crp = self.fluxspeed(qr, ur, cmax2)
        sl = torch.where(clm < crm, clm, crm)
        sr = torch.where(clp > crp, clp, crp)
        left, right = sl >= 0, sr <= 0
        mid = ~(left | right)
        one = torch.ones_like(sl)
        wl = [sl * ul[v] - fl[v] for v in range(self.nv)]
        wr = [sr * ur[v] - fr[v] for v in range(self.nv)]
        dn = torch.where(mid, wr[DN] - wl[DN], one)
        sm = (wr[VX] - wl[VX]) / dn
        pr = (wl[DN] * wr[VX] - wr[DN] * wl[VX]) / dn
        pos, neg = mid & (sm > 0), mid & (sm < 0)
        slmm = torch.where(pos, sl - sm, one)
        srmm = torch.where(neg, sr - sm, one)
        en = self.pr
        dl = wl[DN] / slmm
        uil = [dl, dl * sm, dl * ql[VY], dl * ql[VZ], (wl[en] + sm * pr) / slmm]
        dr = wr[DN] / srmm
        uir = [dr, dr * sm, dr * qr[VY], dr * qr[VZ], (wr[en] + sm * pr) / srmm]
        zero = torch.zeros_like(sl)
        out = []
        for v in range(self.nv):
            f0 = -wl[VX] if v == VX else zero
            fs = torch.where(pos, sl * uil[v] - wl[v], torch.where(neg, sr * uir[v] - wr[v], f0))
            out.append(torch.where(left, fl[v], torch.where(right, fr[v], fs)))
        return out

    # ---- reconstruction ----------------------------------------------------------
    def weno_right(self, fm2, fm1, f0, fp1, fp2):
        c1, c2 = 13.0 / 12.0, 0.25
        dm1, d0m, d0p, dp1 = fm1 - fm2, f0 - fm1, fp1 - f0, fp2 - fp1
        bl = c1 * (d0m - dm1) ** 2 + c2 * (3.0 * d0m - dm1) ** 2
        bc = c1 * (d0p - d0m) ** 2 + c2 * (d0p + d0m) ** 2
        br = c1 * (dp1 - d0p) ** 2 + c2 * (3.0 * d0p - dp1) ** 2
        tt = torch.abs(br - bl)
        al = 1.0 + tt / (bl + self.eps)
        ac = 1.0 + tt / (bc + self.eps)
        ar = 1.0 + tt / (br + self.eps)
        wl, wc, wr = 0.1 * al, 0.6 * ac, 0.3 * ar
        ww = (wl + wr) + wc
        wl, wr = wl / ww, wr / ww
        wc = 1.0 - (wl + wr)
        ql = (2.0 / 6.0) * fm2 + (-7.0 / 6.0) * fm1 + (11.0 / 6.0) * f0
        qc = (-1.0 / 6.0) * fm1 + (5.0 / 6.0) * f0 + (2.0 / 6.0) * fp1
        qr = (2.0 / 6.0) * f0 + (5.0 / 6.0) * fp1 + (-1.0 / 6.0) * fp2
        return (wl * ql + wr * qr) + wc * qc

    def limiter(self, x, a, b):
        """limiter_{mm,mc,sb,vl,va} (src/interpolations.F90:4684-4877) with the
        GPU kernels' branch choices (min/max return the second operand on ties;
        SIGN(x, a) follows the sign bit of a)."""
        def dmin(p, q):
            return torch.where(p < q, p, q)

        def dmax(p, q):
            return torch.where(p > q, p, q)

        sa = torch.copysign(torch.full_like(a, abs(x)), a)
        sb = torch.copysign(torch.full_like(b, abs(x)), b)
        if self.lim == "mm":
            return 0.5 * (sa + sb) * dmin(torch.abs(a), torch.abs(b))
        if self.lim == "mc":
            return (sa + sb) * dmin(dmin(torch.abs(a), torch.abs(b)), 0.25 * torch.abs(a + b))
        if self.lim == "sb":
            return 0.5 * (sa + sb) * dmax(dmin(2.0 * torch.abs(a), torch.abs(b)), dmin(torch.abs(a), 2.0 * torch.abs(b)))
        if self.lim == "vl":
            c = a * b
            pos = c > 0.0
            den = torch.where(pos, a + b, torch.ones_like(a))
            return torch.where(pos, 2.0 * x * c / den, torch.zeros_like(a))
        if self.lim == "va":
            return x * a * b * (a + b) / dmax(torch.full_like(a, self.eps), a * a + b * b)
        raise ValueError(self.lim)

    def tvd_slopes(self, q):
        """interfaces_tvd (src/interpolations.F90:729-848) on the periodic
        field: per variable and direction the half-slope limiter(0.5, q -
        q(-1), q(+1) - q); density and pressure have the slopes of every
        direction halved together while q <= the sum of their magnitudes, and
        zeroed where q <= 0."""
        nd = self.ndims
        out = []
        for v, c in enumerate(q):
            sl = []
            for d in range(nd):
                axis = c.dim() - 1 - d
                sl.append(self.limiter(0.5, c - torch.roll(c, 1, axis), torch.roll(c, -1, axis) - c))
            if v == DN or v == self.pr:
                for _ in range(4096):
                    t = torch.abs(sl[0]) + torch.abs(sl[1])
                    if nd == 3:
                        t = t + torch.abs(sl[2])
                    m = (c > 0.0) & (c <= t)
                    if not bool(m.any()):
                        break
                    sl = [torch.where(m, 0.5 * x, x) for x in sl]
                sl = [torch.where(c > 0.0, x, torch.zeros_like(x)) for x in sl]
            out.append(sl)
        return out

    # ---- one stage operator L(q) ---------------------------------------------------
    def increment(self, q, cmax, cmax2):
        """du for interior cells from the primitive field q (list of nv
        tensors, spatial shape (NZ,)NY,NX, periodic)."""
        du = [torch.zeros_like(q[0]) for _ in range(self.nv)]
        nd = self.ndims
        slopes = self.tvd_slopes(q) if self.rec == "tvd" else None
        for d in range(nd):
            axis = q[0].dim() - 1 - d  # x is the last axis
            n = q[0].shape[axis]
            # periodic padding of 3 cells along the axis, moved last
            pads = [torch.cat([c.narrow(axis, n - 3, 3), c, c.narrow(axis, 0, 3)], dim=axis).movedim(axis, -1)
                    for c in q]
            # interfaces i+1/2 for i = -1..n-1: left state = right face of cell i,
            # right state = left face of cell i+1 (mirror stencil)
            ql, qr = [], []
            if slopes is not None:
                # faces of the TVD cells: q_i + dq_i and q_{i+1} - dq_{i+1}
                for v, c in enumerate(q):
                    fr = c + slopes[v][d]
                    fl = c - slopes[v][d]
                    fr = torch.cat([fr.narrow(axis, n - 1, 1), fr], dim=axis).movedim(axis, -1)
                    fl = torch.cat([fl, fl.narrow(axis, 0, 1)], dim=axis).movedim(axis, -1)
                    ql.append(fr)
                    qr.append(fl)
            for c in pads if slopes is None else ():
                s = [c[..., k:k + n + 1] for k in range(6)]  # cells i-2 .. i+3
                ql.append(self.weno_right(s[0], s[1], s[2], s[3], s[4]))
                qr.append(self.weno_right(s[5], s[4], s[3], s[2], s[1]))
            rot = _ROT[d]

            def rotate(st):
                st = list(st)
                vel = [st[VX + r] for r in rot]
                st[VX:VZ + 1] = vel
                if self.mhd:
                    mag = [st[BX + r] for r in rot]
                    st[BX:BZ + 1] = mag
                return st

            F = (self.hllc if self.rs == "hllc" else self.hll)(rotate(ql), rotate(qr), cmax, cmax2)
            Fu = list(F)
            for m, r in enumerate(rot):
                Fu[VX + r] = F[VX + m]
                if self.mhd:
                    Fu[BX + r] = F[BX + m]
            dxi = 1.0 / self.dx[d]
            for v in range(self.nv):
                diff = (Fu[v][..., 1:] - Fu[v][..., :-1]).movedim(-1, axis)
                du[v] = du[v] - dxi * diff
        return du

    # ---- time step -----------------------------------------------------------------
    def stages(self):
        if self.ta == "rk3":
            return [(0, 0, 0, 1, 0.0, 0.0, 1.0, False), (1, 0, 1, 1, 0.75, 0.25, 0.25, False),
                    (1, 0, 1, 0, 1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0, True)]
        if self.ta == "rk2":
            return [(0, 0, 0, 1, 0.0, 0.0, 1.0, False), (2, 0, 1, 0, 0.0, 0.0, 1.0, True)]
        raise ValueError(self.ta)

    def step(self, U, q, dtnext=1.0e30, fixed=None):
        """One full step from conserved U and primitive q (lists of nv
        tensors); returns (U, q, dt, cmax).  fixed = (dt, cmax) replays a
        recorded step instead of computing them from q."""
        if fixed is not None:
            dt, cmax = fixed
        else:
            with torch.no_grad():
                ms = float(torch.max(self.cell_speed([c.detach() for c in q])))
                cmax = max(ms, 1.0e-300)
                dt = min(self.cfl * self.dx_min / cmax, dtnext)
        cmax2 = cmax * cmax
        slots = [list(U), list(U)]
        qs = q
        for form, a, b, out, ca, cb, dscoef, fin in self.stages():
            du = self.increment(qs, cmax, cmax2)
            ds = dscoef * dt
            A, B = slots[a], slots[b]
            res = []
            for v in range(self.nv):
                if form == 0:
                    r = A[v] + ds * du[v]
                elif form == 1:
                    r = (ca * A[v] + cb * B[v]) + ds * du[v]
                elif form == 2:
                    r = 0.5 * ((A[v] + B[v]) + ds * du[v])
                else:
                    r = ca * A[v] + cb * (B[v] + ds * du[v])
                if fin and self.mhd and v == BP:
                    r = self.decay * r
                res.append(r)
            slots[out] = res
            qs = self.cons2prim(res)
        return slots[0], qs, dt, cmax


def split(field: torch.Tensor):
    """(..., nv) field -> list of nv tensors."""
    return [field[..., v] for v in range(field.shape[-1])]


def join(comps):
    return torch.stack(comps, dim=-1)


def evolve(scheme: Scheme, q0: torch.Tensor, nsteps: int, dtnext: float = 1.0e30, record=None, schedule=None):
    """Primitive field q0 ((NZ,)NY,NX,nv) -> conserved field after nsteps.
    record (a list) receives each step's (dt, cmax); schedule replays them."""
    q = split(q0)
    U = scheme.prim2cons(q)
    for n in range(nsteps):
        U, q, dt, cmax = scheme.step(U, q, dtnext, None if schedule is None else schedule[n])
        if record is not None:
            record.append((dt, cmax))
    return join(U)
