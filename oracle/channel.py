"""numpy restatement of the reference channel step (test infrastructure only).

Every routine below follows one reference routine, cited by file:line, on
arrays in the reference's memory layout: a field is ONE float64 buffer that is
either physical, ``v(0:Nx+1, 0:Nzp+1, 0:Nyp+1)``, or Fourier,
``vv(0:Nxp, 0:Nz+1, 0:Nyp+1)`` complex (``for/fft.f90:72-99``).  In numpy the
buffer has shape ``(Ny+2, Nz+2, Nx+2)`` (index ``[j, k, i]``) and its complex
view shape ``(Ny+2, Nz+2, Nx/2+1)``.  One y-rank and one z-rank
(NprocY = NprocZ = 1), so the MPI exchanges reduce to local copies.

This module is the checker for the CUDA library and the CPU baseline; it is
never the product.  Parity status: unpinned against the Fortran (which cannot
be built here); pinned by analytic known-answer tests.
"""
from __future__ import annotations

import math

import numpy as np

try:  # scipy's pocketfft takes a thread count; numpy's does not
    import scipy.fft as _sfft
except Exception:  # pragma: no cover
    _sfft = None

# ``pi = 4.*atan(1.0)`` (for/fft.f90:152) is evaluated with default-real
# (single precision) literals -- the build has no -fdefault-real-8
# (for/Makefile_0:25-39) -- so every wavenumber uses float32(pi).
PI_REF = float(np.float32(4.0) * np.arctan(np.float32(1.0)))

# RK3 (Wray) coefficients, for/flow.f90:78-86
BETA_BAR = (1.0, 25.0 / 8.0, 9.0 / 4.0)
ZETA_BAR = (0.0, -17.0 / 8.0, -5.0 / 4.0)
H_FRAC = (8.0 / 15.0, 2.0 / 15.0, 5.0 / 15.0)


def grid_metrics(gy_file):
    """gy, gyf, dy, dyf at one y-rank (for/domain.f90:230-248,429-527)."""
    gy_file = np.asarray(gy_file, dtype=np.float64)
    ny = gy_file.size - 1
    gy = np.zeros(ny + 2)
    gy[1:ny + 2] = gy_file                     # h5dread into gy(1:Nyp+1)
    gyf = np.zeros(ny + 2)
    for j in range(1, ny + 1):
        gyf[j] = 0.5 * (gy[j] + gy[j + 1])
    gyf[0] = 2.0 * gyf[1] - gyf[2]
    gyf[ny + 1] = 2.0 * gyf[ny] - gyf[ny - 1]
    dy = np.zeros(ny + 2)
    for j in range(1, ny + 2):
        dy[j] = gyf[j] - gyf[j - 1]
    dyf = np.zeros(ny + 2)
    for j in range(1, ny + 1):
        dyf[j] = gy[j + 1] - gy[j]
    dyf[0] = dyf[1]
    dyf[ny + 1] = dyf[ny]
    return gy, gyf, dy, dyf


class Field:
    """One aliased real/complex buffer (alloc_array3D, for/fft.f90:72-99)."""

    def __init__(self, ny, nz, nx):
        self.buf = np.zeros((ny + 2, nz + 2, nx + 2), dtype=np.float64)

    @property
    def r(self):
        return self.buf

    @property
    def c(self):
        return self.buf.view(np.complex128)


class OracleChannel:
    """State and routines of one channel at NprocY = NprocZ = 1."""

    def __init__(self, p, gy_file, workers=1):
        self.p = p
        self.workers = workers
        self.Nx, self.Ny, self.Nz, self.Nth = p.nx, p.ny, p.nz, p.n_th
        self.Nyp = self.Ny
        self.Nxp = self.Nx // 2
        self.Nkx = self.Nx // 3
        self.Nkz = self.Nz // 3
        self.twoNkz = 2 * self.Nkz
        self.gy, self.gyf, self.dy, self.dyf = grid_metrics(gy_file)
        assert self.gy.size == self.Ny + 2
        self.nu = 1.0 / p.re                               # parameters.f90:101
        self.Ro_inv = 0.0 if math.isinf(p.ro) else 1.0 / p.ro
        self.delta = p.delta
        # init_chan_mpi at rankY == 0 == NprocY-1 (for/domain.f90:284-303)
        self.jstart = 1 if p.u_bc_ymin == 1 else 2
        self.jend = self.Nyp
        self.jstart_th = [1 if p.th_bc_ymin[n] == 1 else 2 for n in range(self.Nth)]
        self.jend_th = [self.Nyp] * self.Nth
        # init_fft wavenumbers (for/fft.f90:213-230)
        self.kx = np.zeros(self.Nxp + 1)
        for i in range(self.Nxp):
            self.kx[i] = i * (2.0 * PI_REF) / p.lx
        self.kz = np.zeros(self.twoNkz + 1)
        for k in range(self.Nkz + 1):
            self.kz[k] = k * (2.0 * PI_REF) / p.lz
        for k in range(1, self.Nkz + 1):
            self.kz[self.twoNkz + 1 - k] = -k * (2.0 * PI_REF) / p.lz
        self.kx2 = self.kx * self.kx
        self.kz2 = self.kz * self.kz
        self.cikx = 1j * self.kx
        self.cikz = 1j * self.kz
        # RK coefficients and time (for/flow.f90:68-86)
        self.delta_t = p.delta_t
        self.h_bar = [f * self.delta_t for f in H_FRAC]
        self.time = 0.0
        self.time_step = 0
        self.rk_step = 1
        self.w_BC_Ymax_c1_transient = p.w_bc_ymax_c1
        mk = lambda: Field(self.Ny, self.Nz, self.Nx)
        self.u1, self.u2, self.u3, self.p_ = mk(), mk(), mk(), mk()
        self.r1, self.r2, self.r3 = mk(), mk(), mk()
        self.f1, self.f2, self.f3, self.s1 = mk(), mk(), mk(), mk()
        self.th = [mk() for _ in range(self.Nth)]
        self.fth = [mk() for _ in range(self.Nth)]
        self.rth = [mk() for _ in range(self.Nth)]
        self.nu_t = np.zeros((self.Ny + 2, self.Nz + 2, self.Nx + 2))
        self.kappa_t = [np.zeros((self.Ny + 2, self.Nz + 2, self.Nx + 2))
                        for _ in range(self.Nth)]

    # ------------------------------------------------------------------
    # FFTs (for/fft.f90:247-382)
    def _fft(self, a, axis, inverse):
        if _sfft is not None:
            f = _sfft.ifft if inverse else _sfft.fft
            out = f(a, axis=axis, workers=self.workers)
        else:
            out = np.fft.ifft(a, axis=axis) if inverse else np.fft.fft(a, axis=axis)
        if inverse:
            out *= a.shape[axis]  # FFTW's backward transform is unnormalised
        return out

    def fft_xz_to_fourier(self, fld: Field):
        """for/fft.f90:247-315 on one aliased buffer."""
        Nx, Nz, Nkx, Nkz, Nxp = self.Nx, self.Nz, self.Nkx, self.Nkz, self.Nxp
        v = fld.r
        x = v[:, :Nz, :Nx]
        if _sfft is not None:
            temp = _sfft.rfft(x, axis=-1, workers=self.workers)   # :258
        else:
            temp = np.fft.rfft(x, axis=-1)
        temp[:, :, :Nkx + 1] /= Nx                                   # :259-263
        temp[:, :, Nkx + 1:Nx // 2 + 1] = 0.0                        # :264-266
        vv = fld.c
        vv[:, :Nz, :Nxp] = temp[:, :Nz, :Nxp]                        # :289 (1 rank)
        vv[:, :Nz, :Nxp] = self._fft(vv[:, :Nz, :Nxp], 1, False)    # :298
        vv[:, :Nkz + 1, :Nxp] /= Nz                                  # :302-306
        vv[:, Nkz + 1:2 * Nkz + 1, :Nxp] = vv[:, Nz - Nkz:Nz, :Nxp] / Nz   # :308-312

    def fft_xz_to_physical(self, fld: Field):
        """for/fft.f90:319-382 on one aliased buffer."""
        Nx, Nz, Nkx, Nkz, Nxp = self.Nx, self.Nz, self.Nkx, self.Nkz, self.Nxp
        vv = fld.c
        vv[:, Nz - Nkz:Nz, :Nxp] = vv[:, Nkz + 1:2 * Nkz + 1, :Nxp].copy()   # :331-335
        vv[:, Nkz + 1:Nz - Nkz, :Nxp] = 0.0                                  # :336-340
        vv[:, :Nz, :Nxp] = self._fft(vv[:, :Nz, :Nxp], 1, True)             # :345
        temp = np.zeros((self.Ny + 2, Nz, Nx // 2 + 1), dtype=np.complex128)
        temp[:, :, :Nxp] = vv[:, :Nz, :Nxp]                                  # :366 (1 rank)
        temp[:, :, Nkx + 1:Nx // 2 + 1] = 0.0                                # :372-378
        if _sfft is not None:
            out = _sfft.irfft(temp, n=Nx, axis=-1, workers=self.workers) * Nx   # :380
        else:
            out = np.fft.irfft(temp, n=Nx, axis=-1) * Nx
        fld.r[:, :Nz, :Nx] = out

    # ------------------------------------------------------------------
    # Thomas solvers at one y-rank (for/channel.f90:1335-1540)
    @staticmethod
    def thomas_real(a, b, c, g, Nyp):
        """thomas_forward_real_mpi + thomas_backward_real_mpi; arrays [j, ...]."""
        for j in range(1, Nyp + 2):                  # :1375-1381 and :1396-1401
            a[j] = -a[j] / b[j - 1]
            b[j] = b[j] + a[j] * c[j - 1]
            g[j] = g[j] + a[j] * g[j - 1]
        g[Nyp + 1] = g[Nyp + 1] / b[Nyp + 1]        # :1483
        for j in range(Nyp, -1, -1):                 # :1486-1488
            g[j] = (g[j] - c[j] * g[j + 1]) / b[j]

    @staticmethod
    def thomas_complex(a, b, c, g, Nyp):
        """thomas_forward_complex_mpi + thomas_backward_complex_mpi (rows 1..Nyp)."""
        for j in range(2, Nyp + 1):                  # :1439-1443
            a[j] = -a[j] / b[j - 1]
            b[j] = b[j] + a[j] * c[j - 1]
            g[j] = g[j] + a[j] * g[j - 1]
        g[Nyp] = g[Nyp] / b[Nyp]                     # :1525
        for j in range(Nyp - 1, 0, -1):              # :1528-1530
            g[j] = (g[j] - c[j] * g[j + 1]) / b[j]

    # ------------------------------------------------------------------
    # implicit-solve boundary rows (for/channel.f90:1545-1968)
    def _bc_rows_1or3(self, matl, matd, matu, vec, bmin, cmin, bmax, cmax):
        Nyp, dy = self.Nyp, self.dy
        if bmin == 0:
            matl[0] = 0.; matd[0] = 1.; matu[0] = 0.; vec[0] = 0.
            matl[1] = 0.; matd[1] = 1.; matu[1] = 0.; vec[1] = cmin
        else:
            matl[0] = 0.; matd[0] = 1.; matu[0] = 0.; vec[0] = 0.
            matl[1] = 0.; matd[1] = -1.; matu[1] = 1.; vec[1] = dy[2] * cmin
        if bmax == 0:
            matl[Nyp + 1] = 0.; matd[Nyp + 1] = 1.; matu[Nyp + 1] = 0.; vec[Nyp + 1] = 0.
            matl[Nyp] = 0.; matd[Nyp] = 1.; matu[Nyp] = 0.; vec[Nyp] = cmax
        else:
            matl[Nyp] = -1.; matd[Nyp] = 1.; matu[Nyp] = 0.; vec[Nyp] = dy[Nyp] * cmax
            matl[Nyp + 1] = 0.; matd[Nyp + 1] = 1.; matu[Nyp + 1] = 0.; vec[Nyp + 1] = 0.

    def apply_bc_u1(self, matl, matd, matu, vec):           # :1545-1626
        p = self.p
        self._bc_rows_1or3(matl, matd, matu, vec, p.u_bc_ymin, p.u_bc_ymin_c1,
                           p.u_bc_ymax, p.u_bc_ymax_c1)

    def apply_bc_u3(self, matl, matd, matu, vec):           # :1710-1792
        p = self.p
        if p.w_bc_ymax != 0 and p.f_type == 4:              # :1775
            self.w_BC_Ymax_c1_transient = p.w_bc_ymax_c1 + p.amp_omega0 * math.sin(
                p.omega0 * (self.Ro_inv / self.delta * self.time - p.force_start))
        cmax = p.w_bc_ymax_c1 if p.w_bc_ymax == 0 else self.w_BC_Ymax_c1_transient
        self._bc_rows_1or3(matl, matd, matu, vec, p.w_bc_ymin, p.w_bc_ymin_c1,
                           p.w_bc_ymax, cmax)

    def apply_bc_th(self, matl, matd, matu, vec, n):        # :1797-1876
        p = self.p
        self._bc_rows_1or3(matl, matd, matu, vec, p.th_bc_ymin[n], p.th_bc_ymin_c1[n],
                           p.th_bc_ymax[n], p.th_bc_ymax_c1[n])

    def apply_bc_u2(self, matl, matd, matu, vec):           # :1631-1705
        p, Nyp, dyf = self.p, self.Nyp, self.dyf
        if p.v_bc_ymin == 0:
            for r in (1, 2):
                matl[r] = 0.; matd[r] = 1.; matu[r] = 0.; vec[r] = p.v_bc_ymin_c1
        elif p.v_bc_ymin == 1:
            matd[1] = -1.; matu[1] = 1.; matl[1] = 0.; vec[1] = dyf[1] * p.v_bc_ymin_c1
        matl[0] = 0.; matd[0] = 1.; matu[0] = 0.; vec[0] = 0.
        if p.v_bc_ymax == 0:
            for r in (Nyp + 1, Nyp):
                matl[r] = 0.; matd[r] = 1.; matu[r] = 0.; vec[r] = p.v_bc_ymax_c1
        elif p.v_bc_ymax == 1:
            matl[Nyp + 1] = -1.; matd[Nyp + 1] = 1.; matu[Nyp + 1] = 0.
            vec[Nyp + 1] = dyf[Nyp] * p.v_bc_ymax_c1

    def apply_bc_rem_div(self, matl, matd, matu, vec, k):   # :1974-2015
        Nyp = self.Nyp
        matl[1] = 0.; matd[1] = 1.; matu[1] = -1.; vec[1] = 0.
        if k == 0:
            matu[1, 0] = 0.
        matl[Nyp] = 1.; matd[Nyp] = -1.; matu[Nyp] = 0.; vec[Nyp] = 0.

    def apply_bc_poisson(self, matl, matd, matu, vec, k):   # :2019-2055
        Nyp = self.Nyp
        matd[1] = 1.; matu[1] = -1.; vec[1] = 0.
        if k == 0:
            matu[1, 0] = 0.
        matd[Nyp] = -1.; matl[Nyp] = 1.; vec[Nyp] = 0.

    # ------------------------------------------------------------------
    # Fourier-space boundary values (for/boundary.f90:299-498,728-821)
    def apply_bc_vel_post(self):
        p, Nyp, K, I = self.p, self.Nyp, slice(0, self.twoNkz + 1), slice(0, self.Nxp)
        dy, dyf = self.dy, self.dyf
        cu1, cu2, cu3 = self.u1.c, self.u2.c, self.u3.c
        # lower (:299-396)
        for cu, b, c1 in ((cu1, p.u_bc_ymin, p.u_bc_ymin_c1), (cu3, p.w_bc_ymin, p.w_bc_ymin_c1)):
            if b == 0:
                cu[0, K, I] = 0.; cu[1, K, I] = 0.
                cu[1, 0, 0] = c1; cu[0, 0, 0] = c1
            else:
                cu[1, K, I] = cu[2, K, I]; cu[0, K, I] = cu[1, K, I]
                cu[1, 0, 0] = cu[2, 0, 0] - dy[2] * c1
                cu[0, 0, 0] = cu[1, 0, 0] - dy[1] * c1
        if p.v_bc_ymin == 0:
            cu2[1, K, I] = 2.0 * p.v_bc_ymin_c1 - cu2[2, K, I]
            cu2[0, K, I] = cu2[1, K, I]
        else:
            cu2[1, K, I] = cu2[2, K, I]; cu2[0, K, I] = cu2[1, K, I]
            cu2[1, 0, 0] = cu2[2, 0, 0] - dyf[1] * p.v_bc_ymin_c1
            cu2[0, 0, 0] = cu2[1, 0, 0] - dyf[1] * p.v_bc_ymin_c1
        # upper (:399-498)
        if p.u_bc_ymax == 0:
            cu1[Nyp, K, I] = 0.; cu1[Nyp + 1, K, I] = 0.
            cu1[Nyp, 0, 0] = p.u_bc_ymax_c1; cu1[Nyp + 1, 0, 0] = p.u_bc_ymax_c1
        else:
            cu1[Nyp, K, I] = cu1[Nyp - 1, K, I]; cu1[Nyp + 1, K, I] = cu1[Nyp, K, I]
            cu1[Nyp, 0, 0] = cu1[Nyp - 1, 0, 0] + dy[Nyp] * p.u_bc_ymax_c1
            cu1[Nyp + 1, 0, 0] = cu1[Nyp, 0, 0] + dy[Nyp] * p.u_bc_ymax_c1
        if p.w_bc_ymax == 0:
            cu3[Nyp, K, I] = 0.; cu3[Nyp + 1, K, I] = 0.
            cu3[Nyp, 0, 0] = p.w_bc_ymax_c1; cu3[Nyp + 1, 0, 0] = p.w_bc_ymax_c1
            cu3[Nyp + 1, 0, 0] = 0.                         # :454 ghost cell not used
        else:
            cu3[Nyp, K, I] = cu3[Nyp - 1, K, I]; cu3[Nyp + 1, K, I] = cu3[Nyp, K, I]
            if p.f_type == 4:
                self.w_BC_Ymax_c1_transient = p.w_bc_ymax_c1 + p.amp_omega0 * math.sin(
                    p.omega0 * (self.Ro_inv / self.delta * self.time - p.force_start))
            cu3[Nyp, 0, 0] = cu3[Nyp - 1, 0, 0] + dy[Nyp] * self.w_BC_Ymax_c1_transient
            cu3[Nyp + 1, 0, 0] = cu3[Nyp, 0, 0] + dy[Nyp] * self.w_BC_Ymax_c1_transient
        if p.v_bc_ymax == 0:
            cu2[Nyp + 1, 0, 0] = 2.0 * p.v_bc_ymax_c1 - cu2[Nyp, 0, 0]   # :476-480
        else:
            cu2[Nyp, K, I] = cu2[Nyp - 1, K, I]; cu2[Nyp + 1, K, I] = cu2[Nyp, K, I]
            cu2[Nyp + 1, 0, 0] = cu2[Nyp, 0, 0] + dy[Nyp] * p.v_bc_ymax_c1

    def apply_bc_th_post(self):
        p, Nyp, K, I = self.p, self.Nyp, slice(0, self.twoNkz + 1), slice(0, self.Nxp)
        dy = self.dy
        for n in range(self.Nth):
            cth = self.th[n].c
            if p.th_bc_ymin[n] == 0:                        # :739-752
                cth[0, K, I] = 0.; cth[1, K, I] = 0.
                cth[1, 0, 0] = p.th_bc_ymin_c1[n]; cth[0, 0, 0] = p.th_bc_ymin_c1[n]
            else:                                          # :753-765
                cth[1, K, I] = cth[2, K, I]; cth[0, K, I] = cth[1, K, I]
                cth[1, 0, 0] = cth[2, 0, 0] - dy[2] * p.th_bc_ymin_c1[n]
                cth[0, 0, 0] = cth[1, 0, 0] - dy[1] * p.th_bc_ymin_c1[n]
            if p.th_bc_ymax[n] == 0:                        # :787-800
                cth[Nyp, K, I] = 0.; cth[Nyp + 1, K, I] = 0.
                cth[Nyp, 0, 0] = p.th_bc_ymax_c1[n]; cth[Nyp + 1, 0, 0] = p.th_bc_ymax_c1[n]
            else:                                          # :801-813
                cth[Nyp, K, I] = cth[Nyp - 1, K, I]; cth[Nyp + 1, K, I] = cth[Nyp, K, I]
                cth[Nyp, 0, 0] = cth[Nyp - 1, 0, 0] + dy[Nyp] * p.th_bc_ymax_c1[n]
                cth[Nyp + 1, 0, 0] = cth[Nyp, 0, 0] + dy[Nyp] * p.th_bc_ymax_c1[n]

    # ------------------------------------------------------------------
    def rem_div_chan(self):
        """Projection onto divergence-free fields (for/channel.f90:946-1023)."""
        Nyp, Nxp, twoNkz = self.Nyp, self.Nxp, self.twoNkz
        dy, dyf = self.dy, self.dyf
        cu1, cu2, cu3, cr1 = self.u1.c, self.u2.c, self.u3.c, self.r1.c
        kx2, kz2, cikx, cikz = self.kx2[:Nxp], self.kz2, self.cikx[:Nxp], self.cikz
        for k in range(twoNkz + 1):
            matl = np.zeros((Nyp + 2, Nxp)); matd = np.ones((Nyp + 2, Nxp))
            matu = np.zeros((Nyp + 2, Nxp)); vec = np.zeros((Nyp + 2, Nxp), np.complex128)
            for j in range(1, Nyp + 1):
                matl[j] = 1. / (dy[j] * dyf[j])
                matd[j] = -kx2 - kz2[k] - 1. / (dy[j + 1] * dyf[j]) - 1. / (dy[j] * dyf[j])
                matu[j] = 1. / (dy[j + 1] * dyf[j])
                vec[j] = (cikx * cu1[j, k, :Nxp]
                          + (cu2[j + 1, k, :Nxp] - cu2[j, k, :Nxp]) / dyf[j]
                          + cikz[k] * cu3[j, k, :Nxp])
            self.apply_bc_rem_div(matl, matd, matu, vec, k)
            self.thomas_complex(matl, matd, matu, vec, Nyp)
            cr1[1:Nyp + 1, k, :Nxp] = vec[1:Nyp + 1]
        K, I = slice(0, twoNkz + 1), slice(0, Nxp)
        J = slice(1, Nyp + 1)
        cu1[J, K, I] = cu1[J, K, I] - cikx[None, None, :] * cr1[J, K, I]
        cu3[J, K, I] = cu3[J, K, I] - cikz[None, :, None] * cr1[J, K, I]
        J2 = slice(2, Nyp + 1)
        cu2[J2, K, I] = cu2[J2, K, I] - (cr1[J2, K, I] - cr1[1:Nyp, K, I]) / dy[2:Nyp + 1, None, None]

    def poisson_p_chan(self):
        """Initial pressure from the velocity field (for/channel.f90:1026-1234)."""
        Nyp, Nxp, twoNkz, Nx, Nz = self.Nyp, self.Nxp, self.twoNkz, self.Nx, self.Nz
        dy, dyf, gyf = self.dy, self.dyf, self.gyf
        cu1, cu2, cu3, cp = self.u1.c, self.u2.c, self.u3.c, self.p_.c
        f1, f2, f3 = self.f1, self.f2, self.f3
        cf1, cf2, cf3, cs1 = f1.c, f2.c, f3.c, self.s1.c
        K, I, J2 = slice(0, twoNkz + 1), slice(0, Nxp), slice(2, Nyp + 1)
        JP, JM = slice(3, Nyp + 2), slice(1, Nyp)
        cikx, cikz = self.cikx[None, None, :Nxp], self.cikz[None, :, None]
        dyf_ = dyf[J2, None, None]
        cf1[J2, K, I] = cikx * cu1[J2, K, I]
        cf2[J2, K, I] = (cu2[JP, K, I] - cu2[J2, K, I]) / dyf_
        cf3[J2, K, I] = cikz * cu3[J2, K, I]
        for f in (f1, f2, f3):
            self.fft_xz_to_physical(f)
        PX = (J2, slice(0, Nz), slice(0, Nx))
        for f in (f1, f2, f3):
            f.r[PX] = f.r[PX] ** 2.
        for f in (f1, f2, f3):
            self.fft_xz_to_fourier(f)
        cs1[J2, K, I] = cf1[J2, K, I] + cf2[J2, K, I] + cf3[J2, K, I]
        for pair in (("dy1", None), ("dy3", None), ("xz", None)):
            if pair[0] == "dy1":
                cf1[J2, K, I] = (cu1[JP, K, I] - cu1[JM, K, I]) / (2. * dyf_)
                cf2[J2, K, I] = cikx * 0.5 * (cu2[J2, K, I] + cu2[JP, K, I])
            elif pair[0] == "dy3":
                cf1[J2, K, I] = (cu3[JP, K, I] - cu3[JM, K, I]) / (2. * dyf_)
                cf2[J2, K, I] = cikz * 0.5 * (cu2[J2, K, I] + cu2[JP, K, I])
            else:
                cf1[J2, K, I] = cikz * cu1[J2, K, I]
                cf2[J2, K, I] = cikx * cu3[J2, K, I]
            self.fft_xz_to_physical(f1)
            self.fft_xz_to_physical(f2)
            f1.r[PX] = 2. * f1.r[PX] * f2.r[PX]
            self.fft_xz_to_fourier(f1)
            cs1[J2, K, I] = cs1[J2, K, I] + cf1[J2, K, I]
        for n in range(self.Nth):
            cth = self.th[n].c
            add = self.p.ri[n] * (cth[JP, K, I] - cth[JM, K, I]) / (gyf[JP] - gyf[JM])[:, None, None]
            add[:, 0, 0] = 0.0
            cs1[J2, K, I] = cs1[J2, K, I] + add
        for k in range(twoNkz + 1):
            matl = np.zeros((Nyp + 2, Nxp)); matd = np.ones((Nyp + 2, Nxp))
            matu = np.zeros((Nyp + 2, Nxp)); vec = np.zeros((Nyp + 2, Nxp), np.complex128)
            for j in range(2, Nyp + 1):
                matl[j] = 1. / (dy[j] * dyf[j])
                matd[j] = -self.kx2[:Nxp] - self.kz2[k] - 1. / (dy[j + 1] * dyf[j]) - 1. / (dy[j] * dyf[j])
                matu[j] = 1. / (dy[j + 1] * dyf[j])
                vec[j] = -1. * cs1[j, k, :Nxp]
            self.apply_bc_poisson(matl, matd, matu, vec, k)
            self.thomas_complex(matl, matd, matu, vec, Nyp)
            cp[1:Nyp + 1, k, :Nxp] = vec[1:Nyp + 1]

    def pre_first_step(self, compute_pressure=False):
        """for/advance.f90:17-44 (ghost_chan_mpi is a no-op at NprocY = 1)."""
        self.apply_bc_vel_post()
        self.rem_div_chan()
        if compute_pressure:
            self.poisson_p_chan()
        if self.p.variable_dt:
            for f in (self.u1, self.u2, self.u3):
                self.fft_xz_to_physical(f)
            self.courant()
            for f in (self.u1, self.u2, self.u3):
                self.fft_xz_to_fourier(f)

    def courant(self):
        """CFL time step, velocity in physical space (for/advance.f90:47-158),
        with the 'Front' thermal-wind branch (:76-89), without the output-event
        scheduling."""
        p = self.p
        dt = p.max_dt
        if self.Ro_inv != 0.0:
            dt = min(dt, 2.0 * PI_REF / abs(self.Ro_inv / self.delta) / 20.0)
        for n in range(self.Nth):
            nmax = math.sqrt(abs(p.th_bc_ymin_c1[n]))
            if nmax > 0:
                # the literal 0.1 is default (single-precision) REAL in the reference
                dt = min(dt, float(np.float32(0.1)) * 2.0 * PI_REF / nmax)
        dx = p.lx / self.Nx
        dz = p.lz / self.Nz
        if p.flavor == "Front":
            rd = self.Ro_inv / self.delta
            J = slice(self.jstart, self.jend + 1)
            gyf = self.gyf[J, None, None]
            with np.errstate(divide="ignore"):
                for n in range(self.Nth):
                    u1 = np.abs(self.u1.r[J, :self.Nz, :self.Nx] - p.dthdz[n] * gyf / rd)
                    u2 = np.abs(self.u2.r[J, :self.Nz, :self.Nx])
                    u3 = np.abs(self.u3.r[J, :self.Nz, :self.Nx]
                                + (1.0 / rd) * p.dthdx[n] * (gyf - 0.5 * p.ly))
                    dt = min(dt, np.min(p.cfl * dx / u1), np.min(p.cfl * self.dy[J, None, None] / u2),
                             np.min(p.cfl * dz / u3))
        else:
            J = slice(1, self.Nyp + 1)
            with np.errstate(divide="ignore"):
                u1 = np.abs(self.u1.r[J, :self.Nz, :self.Nx])
                u2 = np.abs(self.u2.r[J, :self.Nz, :self.Nx])
                u3 = np.abs(self.u3.r[J, :self.Nz, :self.Nx])
                dt_x = np.min(p.cfl * dx / u1)
                dt_y = np.min(p.cfl * self.dy[J, None, None] / u2)
                dt_z = np.min(p.cfl * dz / u3)
            dt = min(dt, dt_x, dt_y, dt_z)
        if dt <= 0:
            self.delta_t = 0.00001
        elif dt >= 1000.:
            self.delta_t = 1000.
        else:
            self.delta_t = dt
        self.h_bar = [f * self.delta_t for f in H_FRAC]

    # ------------------------------------------------------------------
    def user_rhs_chan_fourier(self):
        """Thermal-wind advection for flavor 'Front' (for/forcing.f90:37-113)."""
        p = self.p
        if not (p.flavor == "Front" and self.Ro_inv != 0.0):
            return
        Nyp, Nxp, twoNkz, Ly, d, ri = self.Nyp, self.Nxp, self.twoNkz, p.ly, self.delta, self.Ro_inv
        K, I = slice(0, twoNkz + 1), slice(0, Nxp)
        cikx, cikz = self.cikx[None, None, :Nxp], self.cikz[None, :, None]
        cu1, cu2, cu3 = self.u1.c, self.u2.c, self.u3.c
        cf1, cf2, cf3 = self.f1.c, self.f2.c, self.f3.c
        for n in range(self.Nth):
            dX, dZ = p.dthdx[n], p.dthdz[n]
            J = slice(self.jstart, self.jend + 1)
            JP = slice(self.jstart + 1, self.jend + 2)
            g = (self.gyf[J] - 0.5 * Ly)[:, None, None]
            cf1[J, K, I] = (cf1[J, K, I] - (dX * g * d / ri) * cikz * cu1[J, K, I]
                            - (-1. * dZ * g * d / ri) * cikx * cu1[J, K, I]
                            - (-1. * dZ * d / ri) * 0.5 * (cu2[J, K, I] + cu2[JP, K, I]))
            cf3[J, K, I] = (cf3[J, K, I] - (dX * g * d / ri) * cikz * cu3[J, K, I]
                            - (-1. * dZ * g * d / ri) * cikx * cu3[J, K, I]
                            - (dX * d / ri) * 0.5 * (cu2[J, K, I] + cu2[JP, K, I]))
            J2 = slice(2, Nyp + 1)
            g2 = (self.gy[J2] - 0.5 * Ly)[:, None, None]
            cf2[J2, K, I] = (cf2[J2, K, I] - (dX * g2 * d / ri) * cikz * cu2[J2, K, I]
                             - (-1. * dZ * g2 * d / ri) * cikx * cu2[J2, K, I])
            Jt = slice(self.jstart_th[n], self.jend_th[n] + 1)
            gt = (self.gyf[Jt] - 0.5 * Ly)[:, None, None]
            cth, cfth = self.th[n].c, self.fth[n].c
            cfth[Jt, K, I] = (cfth[Jt, K, I] - (d / ri) * dX * gt * cikz * cth[Jt, K, I]
                              - (d / ri) * (-1.) * dZ * gt * cikx * cth[Jt, K, I])

    def les_active(self):
        p = self.p
        return bool(p.use_les) and ((not p.create_new_flow) or self.time_step > 100)

    # ------------------------------------------------------------------
    def rk_chan_1(self):
        """One RK3/CN substep (for/channel.f90:10-917)."""
        p = self.p
        rk = self.rk_step
        Nyp, Nxp, twoNkz, Nx, Nz, nu = self.Nyp, self.Nxp, self.twoNkz, self.Nx, self.Nz, self.nu
        dy, dyf = self.dy, self.dyf
        h = self.h_bar[rk - 1]
        temp1 = 0.5 * nu * h
        temp2 = 0.5 * h
        temp3 = ZETA_BAR[rk - 1] * h
        temp4 = h
        temp5 = BETA_BAR[rk - 1] * h
        js, je = self.jstart, self.jend
        J, J2 = slice(js, je + 1), slice(2, Nyp + 1)
        K, I = slice(0, twoNkz + 1), slice(0, Nxp)
        cikx = self.cikx[None, None, :Nxp]
        cikz = self.cikz[None, :, None]
        kk = ((self.kx2[None, :Nxp] + self.kz2[:, None]) ** p.beta)[None]
        cu1, cu2, cu3, cp = self.u1.c, self.u2.c, self.u3.c, self.p_.c
        cr1, cr2, cr3 = self.r1.c, self.r2.c, self.r3.c
        cf1, cf2, cf3, cs1 = self.f1.c, self.f2.c, self.f3.c, self.s1.c

        cr1[J, K, I] = cu1[J, K, I]                                  # :40-54
        cr3[J, K, I] = cu3[J, K, I]
        cr2[J2, K, I] = cu2[J2, K, I]
        if rk > 1:                                                   # :57-73
            cr1[J, K, I] = cr1[J, K, I] + temp3 * cf1[J, K, I]
            cr3[J, K, I] = cr3[J, K, I] + temp3 * cf3[J, K, I]
            cr2[J2, K, I] = cr2[J2, K, I] + temp3 * cf2[J2, K, I]
        cs1[J2, K, I] = (cp[J2, K, I] - cp[1:Nyp, K, I]) / dy[J2, None, None]   # :76-82
        cr1[J, K, I] = cr1[J, K, I] - temp4 * (cikx * cp[J, K, I])   # :85-92
        cr3[J, K, I] = cr3[J, K, I] - temp4 * (cikz * cp[J, K, I])
        cr2[J2, K, I] = cr2[J2, K, I] - temp4 * cs1[J2, K, I]        # :94-100
        if p.f_type == 1:                                            # :108-120
            cr1[J, 0, 0] = cr1[J, 0, 0] - temp4 * p.px0
        elif p.f_type == 2:
            cr1[J, 0, 0] = cr1[J, 0, 0] - temp4 * (p.px0 + p.amp_omega0 * math.cos(p.omega0 * self.time))
        cf1[J, K, I] = -nu * kk * cu1[J, K, I]                       # :128-142
        cf3[J, K, I] = -nu * kk * cu3[J, K, I]
        cf2[J2, K, I] = -nu * kk * cu2[J2, K, I]
        cf1[J, K, I] = cf1[J, K, I] + (self.Ro_inv / self.delta) * cu3[J, K, I]   # :146-153
        cf3[J, K, I] = cf3[J, K, I] - (self.Ro_inv / self.delta) * cu1[J, K, I]
        for n in range(self.Nth):                                    # :156-249
            cth, cfth, crth = self.th[n].c, self.fth[n].c, self.rth[n].c
            buoy = p.grav_y * (cth[J2, K, I] * dyf[1:Nyp, None, None]
                               + cth[1:Nyp, K, I] * dyf[J2, None, None]) / (2.0 * dy[J2, None, None])
            buoy[:, 0, 0] = 0.0
            cf2[J2, K, I] = cf2[J2, K, I] + buoy
            cf1[J, K, I] = cf1[J, K, I] + p.grav_x * cth[J, K, I]
            cf3[J, K, I] = cf3[J, K, I] + p.grav_z * cth[J, K, I]
            Jt = slice(self.jstart_th[n], self.jend_th[n] + 1)
            crth[Jt, K, I] = cth[Jt, K, I]
            if rk > 1:
                crth[Jt, K, I] = crth[Jt, K, I] + temp3 * cfth[Jt, K, I]
            cfth[Jt, K, I] = -(nu / p.pr[n]) * kk * cth[Jt, K, I]
            cfth[Jt, K, I] = cfth[Jt, K, I] - cu1[Jt, K, I] * p.dthdx[n] - cu3[Jt, K, I] * p.dthdz[n]
        self.user_rhs_chan_fourier()                                 # :253

        if self.les_active():                                        # :259-289
            from oracle import les
            les.les_chan(self)
            les.les_chan_th(self)
        else:
            for f in (self.u1, self.u2, self.u3):
                self.fft_xz_to_physical(f)
            for n in range(self.Nth):
                self.fft_xz_to_physical(self.th[n])

        u1, u2, u3, s1 = self.u1.r, self.u2.r, self.u3.r, self.s1.r
        PX = (slice(0, Nz), slice(0, Nx))
        Jp = slice(js + 1, je + 2); Jm = slice(js - 1, je)
        J2p = slice(3, Nyp + 2); J2m = slice(1, Nyp)
        dyJ = dy[:, None, None]; dyfJ = dyf[:, None, None]
        # U1*U3 (:299-316)
        s1[(J,) + PX] = u3[(J,) + PX] * u1[(J,) + PX]
        self.fft_xz_to_fourier(self.s1)
        cf1[J, K, I] = cf1[J, K, I] - cikz * cs1[J, K, I]
        cf3[J, K, I] = cf3[J, K, I] - cikx * cs1[J, K, I]
        # U1*U1 (:318-335)
        s1[(J,) + PX] = u1[(J,) + PX] * u1[(J,) + PX]
        self.fft_xz_to_fourier(self.s1)
        cf1[J, K, I] = cf1[J, K, I] - cikx * cs1[J, K, I]
        # U3*U3 (:337-354)
        s1[(J,) + PX] = u3[(J,) + PX] * u3[(J,) + PX]
        self.fft_xz_to_fourier(self.s1)
        cf3[J, K, I] = cf3[J, K, I] - cikz * cs1[J, K, I]
        # U1*U2 (:356-375)
        s1[(J2,) + PX] = ((dyfJ[J2] * u1[(J2,) + PX] + dyfJ[1:Nyp] * u1[(J2m,) + PX])
                          / (2. * dyJ[J2])) * u2[(J2,) + PX]
        self.fft_xz_to_fourier(self.s1)
        cf2[J2, K, I] = cf2[J2, K, I] - cikx * cs1[J2, K, I]
        # U3*U2 (:377-396)
        s1[(J2,) + PX] = ((dyfJ[J2] * u3[(J2,) + PX] + dyfJ[1:Nyp] * u3[(J2m,) + PX])
                          / (2. * dyJ[J2])) * u2[(J2,) + PX]
        self.fft_xz_to_fourier(self.s1)
        cf2[J2, K, I] = cf2[J2, K, I] - cikz * cs1[J2, K, I]
        # d/dy(U1*U2) (:398-417)
        s1[(J,) + PX] = (u1[(Jp,) + PX] * u2[(Jp,) + PX] + u1[(J,) + PX] * u2[(Jp,) + PX]
                         - u1[(J,) + PX] * u2[(J,) + PX] - u1[(Jm,) + PX] * u2[(J,) + PX]) / (2.0 * dyfJ[J])
        self.fft_xz_to_fourier(self.s1)
        cf1[J, K, I] = cf1[J, K, I] - cs1[J, K, I]
        # d/dy(U3*U2) (:419-438)
        s1[(J,) + PX] = (u3[(Jp,) + PX] * u2[(Jp,) + PX] + u3[(J,) + PX] * u2[(Jp,) + PX]
                         - u3[(J,) + PX] * u2[(J,) + PX] - u3[(Jm,) + PX] * u2[(J,) + PX]) / (2.0 * dyfJ[J])
        self.fft_xz_to_fourier(self.s1)
        cf3[J, K, I] = cf3[J, K, I] - cs1[J, K, I]
        # d/dy(U2*U2) (:440-459)
        s1[(J2,) + PX] = (0.25 * (u2[(J2,) + PX] + u2[(J2p,) + PX]) ** 2.
                          - 0.25 * (u2[(J2,) + PX] + u2[(J2m,) + PX]) ** 2.) / dyJ[J2]
        self.fft_xz_to_fourier(self.s1)
        cf2[J2, K, I] = cf2[J2, K, I] - cs1[J2, K, I]

        # user_rhs_chan_physical is empty (for/forcing.f90:5-33)
        cr1[J, K, I] = cr1[J, K, I] + temp5 * cf1[J, K, I]            # :468-482
        cr3[J, K, I] = cr3[J, K, I] + temp5 * cf3[J, K, I]
        cr2[J2, K, I] = cr2[J2, K, I] + temp5 * cf2[J2, K, I]
        for f in (self.r1, self.r2, self.r3):                         # :485-487
            self.fft_xz_to_physical(f)
        r1, r2, r3 = self.r1.r, self.r2.r, self.r3.r
        c = temp1 * p.nu_v_scale                                      # :494-514
        for r, u in ((r1, u1), (r3, u3)):
            r[(J,) + PX] = r[(J,) + PX] + c * (((u[(Jp,) + PX] - u[(J,) + PX]) / dyJ[Jp]
                                                - (u[(J,) + PX] - u[(Jm,) + PX]) / dyJ[J]) / dyfJ[J])
        r2[(J2,) + PX] = r2[(J2,) + PX] + c * (((u2[(J2p,) + PX] - u2[(J2,) + PX]) / dyfJ[J2]
                                                - (u2[(J2,) + PX] - u2[(J2m,) + PX]) / dyfJ[1:Nyp]) / dyJ[J2])
        nt = self.nu_t
        if p.use_les:                                                 # :519-547
            for r, u in ((r1, u1), (r3, u3)):
                r[(J,) + PX] = r[(J,) + PX] + temp2 * (
                    (nt[(Jp,) + PX] * (u[(Jp,) + PX] - u[(J,) + PX]) / dyJ[Jp]
                     - nt[(J,) + PX] * (u[(J,) + PX] - u[(Jm,) + PX]) / dyJ[J]) / dyfJ[J])
            r2[(J2,) + PX] = r2[(J2,) + PX] + temp2 * (
                (0.5 * (nt[(J2,) + PX] + nt[(J2p,) + PX]) * (u2[(J2p,) + PX] - u2[(J2,) + PX]) / dyfJ[J2]
                 - 0.5 * (nt[(J2,) + PX] + nt[(J2m,) + PX]) * (u2[(J2,) + PX] - u2[(J2m,) + PX]) / dyfJ[1:Nyp])
                / dyJ[J2])

        for n in range(self.Nth):                                     # :553-710
            th, cfth, crth = self.th[n].r, self.fth[n].c, self.rth[n].c
            Jt = slice(self.jstart_th[n], self.jend_th[n] + 1)
            Jtp = slice(self.jstart_th[n] + 1, self.jend_th[n] + 2)
            Jtm = slice(self.jstart_th[n] - 1, self.jend_th[n])
            s1[(Jt,) + PX] = th[(Jt,) + PX] * u1[(Jt,) + PX]
            self.fft_xz_to_fourier(self.s1)
            cfth[Jt, K, I] = cfth[Jt, K, I] - cikx * cs1[Jt, K, I]
            s1[(Jt,) + PX] = th[(Jt,) + PX] * u3[(Jt,) + PX]
            self.fft_xz_to_fourier(self.s1)
            cfth[Jt, K, I] = cfth[Jt, K, I] - cikz * cs1[Jt, K, I]
            s1[(Jt,) + PX] = (th[(Jtp,) + PX] * u2[(Jtp,) + PX] + th[(Jt,) + PX] * u2[(Jtp,) + PX]
                              - th[(Jt,) + PX] * u2[(Jt,) + PX] - th[(Jtm,) + PX] * u2[(Jt,) + PX]) / (2.0 * dyfJ[Jt])
            self.fft_xz_to_fourier(self.s1)
            cfth[Jt, K, I] = cfth[Jt, K, I] - cs1[Jt, K, I]
            crth[Jt, K, I] = crth[Jt, K, I] + temp5 * cfth[Jt, K, I]
            self.fft_xz_to_physical(self.rth[n])
            rth = self.rth[n].r
            cth_ = (temp1 / p.pr[n]) * p.nu_v_scale
            rth[(Jt,) + PX] = rth[(Jt,) + PX] + cth_ * (
                ((th[(Jtp,) + PX] - th[(Jt,) + PX]) / dyJ[Jtp]
                 - (th[(Jt,) + PX] - th[(Jtm,) + PX]) / dyJ[Jt]) / dyfJ[Jt])
            kt = self.kappa_t[n]
            if p.use_les:
                rth[(Jt,) + PX] = rth[(Jt,) + PX] + temp2 * (
                    (kt[(Jtp,) + PX] * (th[(Jtp,) + PX] - th[(Jt,) + PX]) / dyJ[Jtp]
                     - kt[(Jt,) + PX] * (th[(Jt,) + PX] - th[(Jtm,) + PX]) / dyJ[Jt]) / dyfJ[Jt])
            # implicit solve (:657-707), vectorised over the k loop
            matl = np.zeros((Nyp + 2, Nz, Nx)); matd = np.ones((Nyp + 2, Nz, Nx))
            matu = np.zeros((Nyp + 2, Nz, Nx)); vec = np.zeros((Nyp + 2, Nz, Nx))
            for j in range(self.jstart_th[n], self.jend_th[n] + 1):
                matl[j] = -(temp1 / p.pr[n] * p.nu_v_scale) / (dy[j] * dyf[j])
                matd[j] = 1. + (temp1 / p.pr[n] * p.nu_v_scale) / (dy[j + 1] * dyf[j]) \
                    + (temp1 / p.pr[n] * p.nu_v_scale) / (dy[j] * dyf[j])
                matu[j] = -(temp1 / p.pr[n] * p.nu_v_scale) / (dy[j + 1] * dyf[j])
                vec[j] = rth[j, :Nz, :Nx]
            if p.use_les:
                for j in range(self.jstart_th[n], self.jend_th[n] + 1):
                    matl[j] = matl[j] - temp2 * kt[j, :Nz, :Nx] / (dy[j] * dyf[j])
                    matd[j] = matd[j] + temp2 * kt[j + 1, :Nz, :Nx] / (dy[j + 1] * dyf[j]) \
                        + temp2 * kt[j, :Nz, :Nx] / (dy[j] * dyf[j])
                    matu[j] = matu[j] - temp2 * kt[j + 1, :Nz, :Nx] / (dy[j + 1] * dyf[j])
            self.apply_bc_th(matl, matd, matu, vec, n)
            self.thomas_real(matl, matd, matu, vec, Nyp)
            th[self.jstart_th[n] - 1:self.jend_th[n] + 2, :Nz, :Nx] = \
                vec[self.jstart_th[n] - 1:self.jend_th[n] + 2]

        # U2 (:716-765)
        matl = np.zeros((Nyp + 2, Nz, Nx)); matd = np.ones((Nyp + 2, Nz, Nx))
        matu = np.zeros((Nyp + 2, Nz, Nx)); vec = np.zeros((Nyp + 2, Nz, Nx))
        for j in range(2, Nyp + 1):
            matl[j] = -temp1 * p.nu_v_scale / (dyf[j - 1] * dy[j])
            matd[j] = 1. + temp1 * p.nu_v_scale / (dyf[j] * dy[j]) + temp1 * p.nu_v_scale / (dyf[j - 1] * dy[j])
            matu[j] = -temp1 * p.nu_v_scale / (dyf[j] * dy[j])
            vec[j] = r2[j, :Nz, :Nx]
        if p.use_les:
            for j in range(2, Nyp + 1):
                matl[j] = matl[j] - temp2 * 0.5 * (nt[j, :Nz, :Nx] + nt[j - 1, :Nz, :Nx]) / (dyf[j - 1] * dy[j])
                matd[j] = matd[j] + temp2 * 0.5 * (nt[j, :Nz, :Nx] + nt[j + 1, :Nz, :Nx]) / (dyf[j] * dy[j]) \
                    + temp2 * 0.5 * (nt[j, :Nz, :Nx] + nt[j - 1, :Nz, :Nx]) / (dyf[j - 1] * dy[j])
                matu[j] = matu[j] - temp2 * 0.5 * (nt[j, :Nz, :Nx] + nt[j + 1, :Nz, :Nx]) / (dyf[j] * dy[j])
        self.apply_bc_u2(matl, matd, matu, vec)
        self.thomas_real(matl, matd, matu, vec, Nyp)
        u2[1:Nyp + 2, :Nz, :Nx] = vec[1:Nyp + 2]

        # U1 and U3 (:767-877)
        for u, r, bc in ((u1, r1, self.apply_bc_u1), (u3, r3, self.apply_bc_u3)):
            matl = np.zeros((Nyp + 2, Nz, Nx)); matd = np.ones((Nyp + 2, Nz, Nx))
            matu = np.zeros((Nyp + 2, Nz, Nx)); vec = np.zeros((Nyp + 2, Nz, Nx))
            for j in range(js, je + 1):
                matl[j] = -temp1 * p.nu_v_scale / (dy[j] * dyf[j])
                matd[j] = 1. - temp1 * p.nu_v_scale * (-1. / (dy[j + 1] * dyf[j]) - 1. / (dy[j] * dyf[j]))
                matu[j] = -temp1 * p.nu_v_scale / (dy[j + 1] * dyf[j])
                vec[j] = r[j, :Nz, :Nx]
            if p.use_les:
                for j in range(js, je + 1):
                    matl[j] = matl[j] - temp2 * nt[j, :Nz, :Nx] / (dy[j] * dyf[j])
                    matd[j] = matd[j] + temp2 * nt[j + 1, :Nz, :Nx] / (dy[j + 1] * dyf[j]) \
                        + temp2 * nt[j, :Nz, :Nx] / (dy[j] * dyf[j])
                    matu[j] = matu[j] - temp2 * nt[j + 1, :Nz, :Nx] / (dy[j + 1] * dyf[j])
            bc(matl, matd, matu, vec)
            self.thomas_real(matl, matd, matu, vec, Nyp)
            u[js - 1:je + 2, :Nz, :Nx] = vec[js - 1:je + 2]

        if p.variable_dt and rk == 3 and (self.time_step % p.update_dt == 0):   # :885-888
            self.courant()

        for f in (self.u1, self.u2, self.u3):                         # :891-896
            self.fft_xz_to_fourier(f)
        for n in range(self.Nth):
            self.fft_xz_to_fourier(self.th[n])
        self.rem_div_chan()                                           # :901
        cp[J, K, I] = cp[J, K, I] + cr1[J, K, I] / temp4              # :905-911

    def filter_chan(self, n):
        """Spectral filter of scalar n on rows jstart_th..jend_th
        (for/channel.f90:1241-1329)."""
        p = self.p
        Nxp, twoNkz = self.Nxp, self.twoNkz
        kx = self.kx[:Nxp][None, :]
        kz = self.kz[:twoNkz + 1][:, None]
        s0 = 0.5 * (1.0 + np.cos(np.sqrt((kx * p.lx * 1.0 / float(np.float32(self.Nx))) ** 2.0
                                         + (kz * p.lz * 1.0 / float(np.float32(self.Nz))) ** 2.0)))
        sigma = s0 ** 4.0 * (35.0 - 84.0 * s0 + 70.0 * s0 ** 2.0 - 20.0 * s0 ** 3.0)
        J = slice(self.jstart_th[n], self.jend_th[n] + 1)
        c = self.th[n].c
        c[J, :twoNkz + 1, :Nxp] = c[J, :twoNkz + 1, :Nxp] * sigma[None]

    def filter_scalars(self):
        """for/advance.f90:161-173."""
        p = self.p
        for n in range(self.Nth):
            if p.filter_th and p.filter_th[n] and p.filter_int[n] > 0 and self.time_step % p.filter_int[n] == 0:
                self.filter_chan(n)

    def step(self, nsteps=1):
        """Main-loop body without I/O (for/diablo.f90:98-111)."""
        for _ in range(nsteps):
            self.time_step += 1
            for rk in (1, 2, 3):
                self.rk_step = rk
                self.rk_chan_1()
            self.time += self.delta_t
            self.filter_scalars()
