"""Pure-torch FP64 restatement of the DNS channel step, differentiable with
torch.autograd (test infrastructure only: the reference gradient that the
hand-written adjoint of libdiablo_gpu is checked against).

The step is for/channel.f90:rk_chan_1 (:10-917) with rem_div_chan
(:946-1023) for velocities and scalars (no LES, no 'Front' forcing), written
in Fourier space the way the CUDA path runs it: the Crank-Nicolson operator
and the wall rows act along y only, so the reference's physical-space solves
per (x, z) column equal solves per (kx, kz) column.  The nonlinear products
are formed in physical space with the reference's dealiased transforms
(for/fft.f90:247-382, float32 pi in the wavenumbers).  Scalars follow
:156-249 (buoyancy grav_y I(th) into cf2 outside the (0,0) mode, grav_x th
and grav_z th into cf1 and cf3, -nu/Pr k^2b th, the background gradients
-u1 dTHdX - u3 dTHdZ) and :553-710 (products th u1, th u3, the y-flux of
th u2, the implicit solve with apply_bc_th's wall rows, :1797-1876).

State: complex128 tensors u1, u2, u3, p, th_0 .. th_{N_th-1} of shape
(Ny+2, 2Nkz+1, Nkx+1) (plane j, packed kz index, kx index) -- the
significant Fourier box.
"""
from __future__ import annotations

import numpy as np
import torch

from oracle.channel import PI_REF, BETA_BAR, ZETA_BAR, H_FRAC, grid_metrics


class TorchChannel:
    def __init__(self, p, gy_file, device="cpu"):
        if p.use_les or getattr(p, "flavor", "Basic") == "Front":
            raise NotImplementedError("DNS without the 'Front' forcing")
        self.nth = p.n_th
        self.jst = [p.jstart_th(n) for n in range(p.n_th)]
        self.p = p
        self.dev = device
        self.Nx, self.Ny, self.Nz = p.nx, p.ny, p.nz
        self.Nyp = p.ny
        self.n = p.ny + 2
        self.Nkx, self.Nkz = p.nx // 3, p.nz // 3
        self.nk2 = 2 * self.Nkz + 1
        gy, gyf, dy, dyf = grid_metrics(gy_file)
        self.dy_np, self.dyf_np = dy, dyf
        t = lambda a: torch.tensor(a, dtype=torch.float64, device=device)
        # dy(0) is not a spacing (zero); 1 there keeps masked-out rows finite
        dys = dy.copy()
        dys[0] = 1.0
        self.dy, self.dyf = t(dys), t(dyf)
        kx = np.array([m * (2.0 * PI_REF) / p.lx for m in range(self.Nkx + 1)])
        kz = np.zeros(self.nk2)
        for k in range(self.Nkz + 1):
            kz[k] = k * (2.0 * PI_REF) / p.lz
        for k in range(1, self.Nkz + 1):
            kz[self.nk2 - k] = -k * (2.0 * PI_REF) / p.lz
        self.kx = t(kx)[None, None, :]
        self.kz = t(kz)[None, :, None]
        self.kk = (self.kx ** 2 + self.kz ** 2) ** p.beta
        self.nu = 1.0 / p.re
        self.roinvd = (0.0 if np.isinf(p.ro) else 1.0 / p.ro) / p.delta
        self.jstart = 1 if p.u_bc_ymin == 1 else 2
        self.jend = self.Nyp
        zidx = [k if k <= self.Nkz else k - self.nk2 + self.Nz for k in range(self.nk2)]
        self.zidx = torch.tensor(zidx, device=device)
        m00 = torch.zeros(1, self.nk2, self.Nkx + 1, dtype=torch.float64, device=device)
        m00[0, 0, 0] = 1.0
        self.m00 = m00

    # -- transforms (for/fft.f90:247-382) ------------------------------
    def to_physical(self, c):
        full = torch.zeros(c.shape[0], self.Nz, self.Nx // 2 + 1, dtype=torch.complex128, device=self.dev)
        full = full.index_copy(1, self.zidx, torch.nn.functional.pad(c, (0, self.Nx // 2 - self.Nkx)))
        return torch.fft.irfft2(full, s=(self.Nz, self.Nx), norm="forward")

    def to_fourier(self, v):
        full = torch.fft.rfft2(v, norm="forward")
        return full.index_select(1, self.zidx)[:, :, :self.Nkx + 1]

    # -- tridiagonal solves (for/channel.f90:1335-1540) ----------------
    @staticmethod
    def thomas(a, b, c, g, j0, j1):
        """Rows j0..j1 of a tridiagonal system (coefficients broadcast against
        g); forward elimination then back substitution, as the reference."""
        a = [a[j] for j in range(len(g))]
        b = [b[j] for j in range(len(g))]
        g = [g[j] for j in range(len(g))]
        for j in range(j0 + 1, j1 + 1):
            f = -a[j] / b[j - 1]
            b[j] = b[j] + f * c[j - 1]
            g[j] = g[j] + f * g[j - 1]
        x = [None] * len(g)
        x[j1] = g[j1] / b[j1]
        for j in range(j1 - 1, j0 - 1, -1):
            x[j] = (g[j] - c[j] * x[j + 1]) / b[j]
        return x

    def _solve_rows(self, kind, r, rk, pr=1.0, j0=None):
        """The implicit CN system of u1/u3 or a scalar (kind 0; the scalar's
        diffusivity is nu/pr and its rows start at j0, :657-707) or u2
        (kind 1) with its wall rows (for/channel.f90:716-877, 1545-1792),
        solved per column."""
        p, Nyp, n = self.p, self.Nyp, self.n
        dy, dyf = self.dy_np, self.dyf_np
        h = H_FRAC[rk - 1] * p.delta_t
        tc = 0.5 * self.nu * h * p.nu_v_scale / pr
        A = np.zeros(n); B = np.ones(n); C = np.zeros(n)
        j0 = self.jstart if j0 is None else j0
        rows = range(j0, self.jend + 1) if kind == 0 else range(2, Nyp + 1)
        for j in rows:
            if kind == 0:
                A[j] = -tc / (dy[j] * dyf[j])
                B[j] = 1. - tc * (-1. / (dy[j + 1] * dyf[j]) - 1. / (dy[j] * dyf[j]))
                C[j] = -tc / (dy[j + 1] * dyf[j])
            else:
                A[j] = -tc / (dyf[j - 1] * dy[j])
                B[j] = 1. + tc / (dyf[j] * dy[j]) + tc / (dyf[j - 1] * dy[j])
                C[j] = -tc / (dyf[j] * dy[j])
        zero = torch.zeros_like(r[0])
        vec = [r[j] if j in rows else zero for j in range(n)]
        return A, B, C, vec

    def _bc13(self, A, B, C, vec, bmin, cmin, bmax, cmax):
        Nyp, dy = self.Nyp, self.dy_np
        z = torch.zeros_like(vec[0])
        m = self.m00[0].to(torch.complex128)
        A[0], B[0], C[0], vec[0] = 0., 1., 0., z
        if bmin == 0:
            A[1], B[1], C[1], vec[1] = 0., 1., 0., cmin * m
        else:
            A[1], B[1], C[1], vec[1] = 0., -1., 1., dy[2] * cmin * m
        A[Nyp + 1], B[Nyp + 1], C[Nyp + 1], vec[Nyp + 1] = 0., 1., 0., z
        if bmax == 0:
            A[Nyp], B[Nyp], C[Nyp], vec[Nyp] = 0., 1., 0., cmax * m
        else:
            A[Nyp], B[Nyp], C[Nyp], vec[Nyp] = -1., 1., 0., dy[Nyp] * cmax * m

    def _bc2(self, A, B, C, vec):
        p, Nyp, dyf = self.p, self.Nyp, self.dyf_np
        z = torch.zeros_like(vec[0])
        m = self.m00[0].to(torch.complex128)
        if p.v_bc_ymin == 0:
            for r in (1, 2):
                A[r], B[r], C[r], vec[r] = 0., 1., 0., p.v_bc_ymin_c1 * m
        else:
            A[1], B[1], C[1], vec[1] = 0., -1., 1., dyf[1] * p.v_bc_ymin_c1 * m
        A[0], B[0], C[0], vec[0] = 0., 1., 0., z
        if p.v_bc_ymax == 0:
            for r in (Nyp + 1, Nyp):
                A[r], B[r], C[r], vec[r] = 0., 1., 0., p.v_bc_ymax_c1 * m
        else:
            A[Nyp + 1], B[Nyp + 1], C[Nyp + 1], vec[Nyp + 1] = -1., 1., 0., dyf[Nyp] * p.v_bc_ymax_c1 * m

    # -- nonlinear terms (for/channel.f90:299-459) ----------------------
    def nonlinear(self, u1c, u2c, u3c, thc=()):
        """NL of u1, u2, u3 (:299-459) and of each scalar (:553-608); the
        scalars' rows are masked by the caller."""
        Nyp = self.Nyp
        u1, u2, u3 = self.to_physical(u1c), self.to_physical(u2c), self.to_physical(u3c)
        dy = self.dy[:, None, None]
        dyf = self.dyf[:, None, None]
        J = slice(1, Nyp + 1)
        Jp, Jm = slice(2, Nyp + 2), slice(0, Nyp)
        ikx, ikz = 1j * self.kx, 1j * self.kz
        F = self.to_fourier
        p13 = F(u1[J] * u3[J])
        p11 = F(u1[J] * u1[J])
        p33 = F(u3[J] * u3[J])
        y1 = F((u1[Jp] * u2[Jp] + u1[J] * u2[Jp] - u1[J] * u2[J] - u1[Jm] * u2[J]) / (2.0 * dyf[J]))
        y3 = F((u3[Jp] * u2[Jp] + u3[J] * u2[Jp] - u3[J] * u2[J] - u3[Jm] * u2[J]) / (2.0 * dyf[J]))
        i1 = (dyf[J] * u1[J] + dyf[Jm] * u1[Jm]) / (2.0 * dy[J])
        i3 = (dyf[J] * u3[J] + dyf[Jm] * u3[Jm]) / (2.0 * dy[J])
        q1 = F(i1 * u2[J])
        q3 = F(i3 * u2[J])
        v = F((0.25 * (u2[J] + u2[Jp]) ** 2 - 0.25 * (u2[J] + u2[Jm]) ** 2) / dy[J])
        z = torch.zeros_like(u1c[:1])
        nl1 = torch.cat([z, ikz * p13 + ikx * p11 + y1, z])
        nl3 = torch.cat([z, ikx * p13 + ikz * p33 + y3, z])
        nl2 = torch.cat([z, ikx * q1 + ikz * q3 + v, z])
        nlth = []
        for c in thc:
            th = self.to_physical(c)
            a1 = F(th[J] * u1[J])
            a3 = F(th[J] * u3[J])
            yt = F((th[Jp] * u2[Jp] + th[J] * u2[Jp] - th[J] * u2[J] - th[Jm] * u2[J]) / (2.0 * dyf[J]))
            nlth.append(torch.cat([z, ikx * a1 + ikz * a3 + yt, z]))
        return (nl1, nl2, nl3) + tuple(nlth)

    # -- one RK substep -------------------------------------------------
    def substep(self, st, fprev, rk):
        p, Nyp, n = self.p, self.Nyp, self.n
        u1, u2, u3, pr = st[:4]
        ths = st[4:]
        h = H_FRAC[rk - 1] * p.delta_t
        t3, t4, t5 = ZETA_BAR[rk - 1] * h, h, BETA_BAR[rk - 1] * h
        tc = 0.5 * self.nu * h * p.nu_v_scale
        ikx, ikz = 1j * self.kx, 1j * self.kz
        dy, dyf = self.dy[:, None, None], self.dyf[:, None, None]
        nls = self.nonlinear(u1, u2, u3, ths)
        nl1, nl2, nl3 = nls[:3]
        js, je = self.jstart, self.jend
        rows13 = torch.zeros(n, 1, 1, dtype=torch.float64, device=self.dev)
        rows13[js:je + 1] = 1.0
        rows2 = torch.zeros(n, 1, 1, dtype=torch.float64, device=self.dev)
        rows2[2:Nyp + 1] = 1.0
        pm = torch.cat([pr[:1], pr[:-1]])
        dp = (pr - pm) / dy
        cf1 = rows13 * (-self.nu * self.kk * u1 + self.roinvd * u3 - nl1)
        cf3 = rows13 * (-self.nu * self.kk * u3 - self.roinvd * u1 - nl3)
        cf2 = rows2 * (-self.nu * self.kk * u2 - nl2)
        # scalars' explicit terms (:156-249) and their products (:553-608)
        dyfm = torch.cat([self.dyf[:1], self.dyf[:-1]])[:, None, None]
        cfth = []
        for q, th in enumerate(ths):
            thm = torch.cat([th[:1], th[:-1]])
            buoy = p.grav_y * (th * dyfm + thm * dyf) / (2.0 * dy)
            cf2 = cf2 + rows2 * (1.0 - self.m00) * buoy
            cf1 = cf1 + rows13 * p.grav_x * th
            cf3 = cf3 + rows13 * p.grav_z * th
            rowst = torch.zeros(n, 1, 1, dtype=torch.float64, device=self.dev)
            rowst[self.jst[q]:je + 1] = 1.0
            cfth.append(rowst * (-(self.nu / p.pr[q]) * self.kk * th - u1 * p.dthdx[q]
                                 - u3 * p.dthdz[q] - nls[3 + q]))
        px = 0.0
        if p.f_type == 1:
            px = t4 * p.px0
        cr1 = u1 - t4 * ikx * pr - px * self.m00 + t5 * cf1
        cr3 = u3 - t4 * ikz * pr + t5 * cf3
        cr2 = u2 - t4 * dp + t5 * cf2
        if rk > 1:
            cr1 = cr1 + t3 * fprev[0]
            cr2 = cr2 + t3 * fprev[1]
            cr3 = cr3 + t3 * fprev[2]
        up = lambda u: torch.cat([u[1:], u[-1:]])
        um = lambda u: torch.cat([u[:1], u[:-1]])
        dyp = torch.cat([self.dy[1:], self.dy[-1:]])[:, None, None]
        r1 = cr1 + tc * (((up(u1) - u1) / dyp - (u1 - um(u1)) / dy) / dyf)
        r3 = cr3 + tc * (((up(u3) - u3) / dyp - (u3 - um(u3)) / dy) / dyf)
        r2 = cr2 + tc * (((up(u2) - u2) / dyf - (u2 - um(u2)) / dyfm) / dy)
        out = []
        for kind, r, u, bc in ((0, r1, u1, (p.u_bc_ymin, p.u_bc_ymin_c1, p.u_bc_ymax, p.u_bc_ymax_c1)),
                               (1, r2, u2, None),
                               (0, r3, u3, (p.w_bc_ymin, p.w_bc_ymin_c1, p.w_bc_ymax, p.w_bc_ymax_c1))):
            A, B, C, vec = self._solve_rows(kind, r, rk)
            if kind == 0:
                self._bc13(A, B, C, vec, *bc)
                w0 = js - 1
            else:
                self._bc2(A, B, C, vec)
                w0 = 1
            x = self.thomas(A, B, C, vec, 0, n - 1)
            out.append(torch.stack([u[j] if j < w0 else x[j] for j in range(n)]))
        u1s, u2s, u3s = out
        # scalars: cr, the CN half and the implicit solve (:553-710)
        thn = []
        for q, th in enumerate(ths):
            crt = th + t5 * cfth[q]
            if rk > 1:
                crt = crt + t3 * fprev[3 + q]
            rt = crt + (tc / p.pr[q]) * (((up(th) - th) / dyp - (th - um(th)) / dy) / dyf)
            A, B, C, vec = self._solve_rows(0, rt, rk, p.pr[q], self.jst[q])
            self._bc13(A, B, C, vec, p.th_bc_ymin[q], p.th_bc_ymin_c1[q],
                       p.th_bc_ymax[q], p.th_bc_ymax_c1[q])
            x = self.thomas(A, B, C, vec, 0, n - 1)
            w0 = self.jst[q] - 1
            thn.append(torch.stack([th[j] if j < w0 else x[j] for j in range(n)]))
        # projection (rem_div_chan, for/channel.f90:946-1023)
        kx2, kz2 = self.kx ** 2, self.kz ** 2
        zero = torch.zeros_like(u1s[0])
        A = [torch.zeros_like(kx2[0].expand(self.nk2, -1)) for _ in range(n)]
        B = [torch.ones_like(A[0]) for _ in range(n)]
        C = [torch.zeros_like(A[0]) for _ in range(n)]
        dyn, dyfn = self.dy_np, self.dyf_np
        vec = [zero] * n
        for j in range(1, Nyp + 1):
            A[j] = A[j] + 1. / (dyn[j] * dyfn[j])
            B[j] = -kx2[0] - kz2[0] - 1. / (dyn[j + 1] * dyfn[j]) - 1. / (dyn[j] * dyfn[j])
            C[j] = C[j] + 1. / (dyn[j + 1] * dyfn[j])
            vec[j] = ikx[0] * u1s[j] + (u2s[j + 1] - u2s[j]) / dyfn[j] + ikz[0] * u3s[j]
        A[1] = torch.zeros_like(A[1]); B[1] = torch.ones_like(B[1])
        c1 = -torch.ones_like(C[1])
        c1[0, 0] = 0.0
        C[1] = c1
        vec[1] = zero
        A[Nyp] = torch.ones_like(A[Nyp]); B[Nyp] = -torch.ones_like(B[Nyp]); C[Nyp] = torch.zeros_like(C[Nyp])
        vec[Nyp] = zero
        phi = self.thomas(A, B, C, vec, 1, Nyp)
        phi = torch.stack([zero] + phi[1:Nyp + 1] + [zero])
        J = torch.zeros(n, 1, 1, dtype=torch.float64, device=self.dev)
        J[1:Nyp + 1] = 1.0
        J2 = torch.zeros(n, 1, 1, dtype=torch.float64, device=self.dev)
        J2[2:Nyp + 1] = 1.0
        u1n = u1s - J * ikx * phi
        u3n = u3s - J * ikz * phi
        phim = torch.cat([phi[:1], phi[:-1]])
        u2n = u2s - J2 * (phi - phim) / dy
        prn = pr + rows13 * phi / t4
        return (u1n, u2n, u3n, prn) + tuple(thn), (cf1, cf2, cf3) + tuple(cfth)

    def step(self, st, nsteps=1):
        for _ in range(nsteps):
            f = None
            for rk in (1, 2, 3):
                st, f = self.substep(st, f, rk)
        return st

    @staticmethod
    def energy(st, p, dy, dyf):
        """J = 1/2 <u.u>: the volume average of the kinetic energy of the
        dealiased field, by Parseval over the stored half spectrum (weight 2
        for kx > 0), u1, u3 on GYF planes 1..Ny (weights dyf), u2 on GY planes
        2..Ny (weights dy).  Entries of st beyond the third (scalars) count
        like u1: 1/2 <th^2> on GYF planes."""
        u1, u2, u3 = st[0], st[1], st[2]
        w = torch.full((u1.shape[2],), 2.0, dtype=torch.float64, device=u1.device)
        w[0] = 1.0
        ny = p.ny
        e13 = ((u1.abs() ** 2 + u3.abs() ** 2) * w).sum(dim=(1, 2))
        for th in st[3:]:
            e13 = e13 + ((th.abs() ** 2) * w).sum(dim=(1, 2))
        e2 = ((u2.abs() ** 2) * w).sum(dim=(1, 2))
        ly = dyf[1:ny + 1].sum()
        return 0.5 * ((e13[1:ny + 1] * dyf[1:ny + 1]).sum() + (e2[2:ny + 1] * dy[2:ny + 1]).sum()) / ly
