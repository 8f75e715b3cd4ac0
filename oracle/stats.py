"""numpy restatement of the reference's plane statistics (test infrastructure
only): ``save_stats_chan`` (for/statistics.f90:44-712) with the routines it
calls -- compute_averages (:713-838), compute_TKE_diss (:839-1129),
compute_MKE_diss (:1130-1284), compute_TKE (:1285-1393),
compute_TKE_Production (:1394-1549), compute_Vorticity (:1550-1754),
integrate_y_var (:1974-1990) and compute_TKE_diss_les (:2054-2120) -- for the
x-homogeneous case (``homogeneousX``, for/parameters.f90:275-280: every IC type
but 5-8) and the non-homogeneous one, one y-rank and one z-rank.

Like the reference, every plane average is formed in PHYSICAL space: the
fields (and the spectral gradients the reference builds) are transformed with
``fft_xz_to_physical`` and summed over the Nx x Nz grid points.  The CUDA
library evaluates the same averages from the Fourier coefficients (Parseval),
so the two agree to round-off, not bit for bit.

Both branches of ``homogeneousX`` are restated, with compute_BPE and the y*
binning (Bin_Ystar_and_Write).  Not restated: HDF5/movie output.  The oracle is
the checker of the CUDA library, never the product.

Quirks kept from the reference:
  * pe_diss uses the wall-normal gradient of scalar 1 for every scalar
    (``crth(i, k, j +- 1, 1)``, :316).
  * In the homogeneous branch compute_MKE_diss returns before it fills
    dudx_m, dvdx_m, dwdx_m (:1147-1149), so uu_dudx, wu_dwdx and vu_dvdx are 0
    (the arrays are zero-initialised module storage) and epsilon_m is 0.
  * GY-grid profiles (uv, wv, epsilon, mke, the production terms) are 0 at
    j = 1, the first row their loops leave untouched.
  * compute_TKE_diss_les sums the work array ``temp`` over j = 1 too, whose
    row 1 it never writes; that row is reported as 0.

The thermal-wind shift ``(1/(Ro_inv/delta)) dTHdX(1)`` (:172, :1244, :1539,
:1587) is taken as 0 when dTHdX(1) = 0: the reference evaluates Inf * 0 = NaN
there when Ro_inv = 0 and reads past dTHdX when N_th = 0.
"""
from __future__ import annotations

import math

import numpy as np

from .channel import Field, OracleChannel

VEL_PROFILES = ("ume", "vme", "wme", "mke", "urms", "vrms", "wrms", "uv", "uw", "wv",
                "uu_dudx", "vv_dvdy", "wu_dwdx", "vu_dvdx", "uv_dudy", "wv_dwdy",
                "dudy", "dwdy", "cp", "shear", "omega_x", "omega_y", "omega_z",
                "epsilon", "epsilon_m", "nu_sgs", "eps_sgs2")
TH_PROFILES = ("thme", "dthdy", "thrms", "thv", "thv_m", "pe_diss", "kappa_sgs")
SCALARS = ("time", "dt", "ubulk", "urms_b", "vrms_b", "wrms_b", "u1y_left_b")


def thermal_wind_shear(p) -> float:
    """(1/(Ro_inv/delta)) * dTHdX(1) in IEEE arithmetic (a signed infinity
    when Ro_inv = 0), taken as 0 when dTHdX(1) = 0."""
    d = float(p.dthdx[0]) if p.n_th > 0 else 0.0
    if d == 0.0:
        return 0.0
    q = p.ro_inv / p.delta
    if q == 0.0:
        return math.copysign(math.inf, q) * d
    return (1.0 / q) * d


def integrate_y_var(o: OracleChannel, var) -> float:
    """for/statistics.f90:1974-1990 (one y-rank): trapezoid over GY, / Ly."""
    res = 0.0
    for j in range(2, o.Nyp + 1):
        res = res + 0.5 * (var[j] + var[j - 1]) * o.dy[j]
    return res / o.p.ly


def _phys(o: OracleChannel, c):
    """fft_xz_to_physical of a complex array laid out like Field.c; returns
    the physical values [j, k, i] on the Nz x Nx grid."""
    f = Field(o.Ny, o.Nz, o.Nx)
    f.c[:] = c
    o.fft_xz_to_physical(f)
    return f.r[:, :o.Nz, :o.Nx].copy()


def _krows(kfac, k0):
    """A wavenumber factor broadcast over [j, k, i], restricted to k >= k0."""
    return kfac if kfac.shape[1] == 1 else kfac[:, k0:, :]


def save_stats_chan(o: OracleChannel, nu_t=None, homogeneous_x: bool = True, kappa_t=None) -> dict:
    """Statistics of the oracle's current (Fourier) state.  Applies the
    velocity and scalar wall values first, as the reference does (:63-64),
    which changes the oracle's state the same way.  ``nu_t`` (reference
    physical layout) enables the LES rows nu_sgs and eps_sgs2; ``kappa_t`` (one
    such array per scalar) each scalar's kappa_sgs, the plane mean of its
    kappa_t (kappa_t_mean, for/les.f90:1420-1448).
    ``homogeneous_x = False`` is the branch of IC types 5-8: z-line averages
    ume_xy(x, y) etc. as the means (when Nz > 1), the x derivatives of epsilon
    without the kz = 0 row, compute_MKE_diss and the production terms that use
    its mean gradients."""
    p = o.p
    Nx, Nz, Nyp, Nxp, tk = o.Nx, o.Nz, o.Nyp, o.Nxp, o.twoNkz
    gy, gyf, dy, dyf = o.gy, o.gyf, o.dy, o.dyf
    NN = float(Nx * Nz)
    ny2 = Nyp + 2
    K, I = slice(0, tk + 1), slice(0, Nxp)
    tws = thermal_wind_shear(p)
    o.apply_bc_vel_post()
    o.apply_bc_th_post()
    cr1, cr2, cr3 = o.u1.c.copy(), o.u2.c.copy(), o.u3.c.copy()
    crth = [t.c.copy() for t in o.th]
    u1, u2, u3 = _phys(o, cr1), _phys(o, cr2), _phys(o, cr3)
    th = [_phys(o, c) for c in crth]
    cikx = o.cikx[None, None, :Nxp]
    cikz = o.cikz[None, :tk + 1, None]
    out = {k: np.zeros(ny2) for k in VEL_PROFILES}

    # compute_averages (:733-746, :749-836): plane means, and the z-line means
    # ume_xy(i, j) etc. that every fluctuation below is taken about
    ume, vme, wme = cr1[:, 0, 0].real.copy(), cr2[:, 0, 0].real.copy(), cr3[:, 0, 0].real.copy()
    thme = [c[:, 0, 0].real.copy() for c in crth]
    out["ume"][:], out["vme"][:], out["wme"][:] = ume, vme, wme
    ubulk = integrate_y_var(o, ume)
    ume_xy, vme_xy, wme_xy = np.zeros((ny2, Nx)), np.zeros((ny2, Nx)), np.zeros((ny2, Nx))
    thme_xy = [np.zeros((ny2, Nx)) for _ in crth]
    if Nz > 1 and not homogeneous_x:
        for j in range(1, Nyp + 1):
            ume_xy[j] = np.sum(u1[j], axis=0) / float(Nz)
            wme_xy[j] = np.sum(u3[j], axis=0) / float(Nz)
            for n in range(o.Nth):
                thme_xy[n][j] = np.sum(th[n][j], axis=0) / float(Nz)
        for j in range(1, Nyp + 2):
            vme_xy[j] = np.sum(u2[j], axis=0) / float(Nz)
    else:
        ume_xy[1:Nyp + 1] = ume[1:Nyp + 1, None]
        wme_xy[1:Nyp + 1] = wme[1:Nyp + 1, None]
        vme_xy[1:Nyp + 2] = vme[1:Nyp + 2, None]
        for n in range(o.Nth):
            thme_xy[n][1:Nyp + 1] = thme[n][1:Nyp + 1, None]

    def zero_cs():
        return np.zeros_like(cr1)

    # compute_TKE_diss (:859-1062); the x derivatives skip the kz = 0 row
    # outside the homogeneous branch (k_start, :862-866)
    k0 = 0 if homogeneous_x else 1
    eps = np.zeros(ny2)

    # pointwise fields the y* binning averages (Bin_Ystar_and_Write, :1877-1972)
    ptw = {}
    eps_f1 = np.zeros_like(u1)

    def interp_sq(s, j):   # (dyf(j-1) s(j)^2 + dyf(j) s(j-1)^2) / (2 dy(j)), summed
        f = (dyf[j - 1] * s[j] ** 2 + dyf[j] * s[j - 1] ** 2) / (2.0 * dy[j])
        eps_f1[j] += f
        return np.sum(f)

    for cr, kfac, kk in ((cr1, cikx, k0), (cr3, cikx, k0), (cr1, cikz, 0), (cr3, cikz, 0)):
        cs = zero_cs()                                     # du/dx dw/dx du/dz dw/dz
        cs[1:Nyp + 1, kk:tk + 1, I] = _krows(kfac, kk) * cr[1:Nyp + 1, kk:tk + 1, I]
        s = _phys(o, cs)
        for j in range(2, Nyp + 1):
            eps[j] += interp_sq(s, j)
    for kfac, kk in ((cikx, k0), (cikz, 0)):               # dv/dx dv/dz
        cs = zero_cs()
        cs[2:Nyp + 1, kk:tk + 1, I] = _krows(kfac, kk) * cr2[2:Nyp + 1, kk:tk + 1, I]
        s = _phys(o, cs)
        for j in range(2, Nyp + 1):
            eps[j] += np.sum(s[j] ** 2)
            eps_f1[j] += s[j] ** 2
    for j in range(2, Nyp + 1):
        su = ((u1[j] - ume_xy[j]) - (u1[j - 1] - ume_xy[j - 1])) / dy[j]      # du/dy
        sv = ((u2[j + 1] - vme_xy[j + 1]) - (u2[j - 1] - vme_xy[j - 1])) / (gy[j + 1] - gy[j - 1])
        sw = ((u3[j] - wme_xy[j]) - (u3[j - 1] - wme_xy[j - 1])) / dy[j]      # dw/dy
        eps[j] += np.sum(su ** 2) + np.sum(sv ** 2) + np.sum(sw ** 2)
        eps_f1[j] += su ** 2 + sv ** 2 + sw ** 2
    out["epsilon"][:] = o.nu * eps / NN
    ptw["epsilon"] = o.nu * eps_f1

    # compute_MKE_diss (:1130-1284): returns at once in the homogeneous branch,
    # leaving epsilon_m and the mean x gradients 0
    dudx_m, dvdx_m, dwdx_m = np.zeros((ny2, Nx)), np.zeros((ny2, Nx)), np.zeros((ny2, Nx))
    if not homogeneous_x:
        epm = np.zeros(ny2)

        def row_phys(cr, jlo):            # x derivative of the kz = 0 row, rows jlo..Nyp
            cs = zero_cs()
            cs[jlo:Nyp + 1, 0, I] = o.cikx[:Nxp] * cr[jlo:Nyp + 1, 0, I]
            return _phys(o, cs)[:, 0, :]
        s = row_phys(cr1, 1)
        for j in range(1, Nyp + 1):
            epm[j] += np.sum((dyf[j - 1] * s[j] ** 2 + dyf[j] * s[j - 1] ** 2) / (2.0 * dy[j]))
        dudx_m[1:Nyp + 1] = s[1:Nyp + 1]
        s = row_phys(cr2, 1)
        for j in range(1, Nyp + 1):
            epm[j] += np.sum(s[j] ** 2)
        dvdx_m[1:Nyp + 1] = s[1:Nyp + 1]
        for j in range(2, Nyp + 1):
            epm[j] += np.sum(((ume_xy[j] - ume_xy[j - 1]) / dy[j]) ** 2)
        s = row_phys(cr3, 1)
        for j in range(1, Nyp + 1):
            epm[j] += np.sum((dyf[j - 1] * s[j] ** 2 + dyf[j] * s[j - 1] ** 2) / (2.0 * dy[j]))
        dwdx_m[1:Nyp + 1] = s[1:Nyp + 1]
        for j in range(2, Nyp + 1):
            epm[j] += np.sum(((vme_xy[j + 1] - vme_xy[j - 1]) / (gy[j + 1] - gy[j - 1])) ** 2)
            epm[j] += np.sum(((wme_xy[j] - wme_xy[j - 1]) / dy[j] + tws) ** 2)
        out["epsilon_m"][:] = o.nu * epm / float(Nx)

    # compute_TKE_diss_les (:2054-2120)
    if nu_t is not None:
        nt = nu_t[:, :Nz, :Nx]
        s1 = np.zeros_like(u1)
        for j in range(1, Nyp + 1):
            s1[j] = (u1[j] * ((nt[j + 1] * (u1[j + 1] - u1[j]) / dy[j + 1]
                               - nt[j] * (u1[j] - u1[j - 1]) / dy[j]) / dyf[j])
                     + u3[j] * ((nt[j + 1] * (u3[j + 1] - u3[j]) / dy[j + 1]
                                 - nt[j] * (u3[j] - u3[j - 1]) / dy[j]) / dyf[j]))
        for j in range(2, Nyp + 1):
            temp = (0.5 * (s1[j] + s1[j - 1])
                    + u2[j] * ((0.5 * (nt[j] + nt[j + 1]) * (u2[j + 1] - u2[j]) / dyf[j]
                                - 0.5 * (nt[j] + nt[j - 1]) * (u2[j] - u2[j - 1]) / dyf[j - 1]) / dy[j]))
            out["eps_sgs2"][j] = np.sum(temp) / NN
        # nu_sgs: the plane mean of nu_t (nu_t_mean, for/les.f90:927-937)
        for j in range(1, Nyp + 1):
            out["nu_sgs"][j] = np.sum(nt[j]) / NN

    # compute_TKE (:1290-1331), with the z means uu_xy, vv_xy at each x
    uu_xy, vv_xy = np.zeros((ny2, Nx)), np.zeros((ny2, Nx))
    tke_f1 = np.zeros_like(u1)
    for name, u, me, xy in (("urms", u1, ume_xy, uu_xy), ("vrms", u2, vme_xy, vv_xy),
                            ("wrms", u3, wme_xy, None)):
        for j in range(1, Nyp + 1):
            d2 = (u[j] - me[j]) ** 2
            tke_f1[j] += 0.5 * d2
            out[name][j] = np.sum(d2) / NN
            if xy is not None:
                xy[j] = np.sum(d2, axis=0) / float(Nz)
    ptw["TKE"] = tke_f1
    ptw["KE"] = 0.5 * (u1 ** 2 + u2 ** 2 + u3 ** 2)
    urms_b = np.sqrt(integrate_y_var(o, out["urms"]))
    vrms_b = np.sqrt(integrate_y_var(o, out["vrms"]))
    wrms_b = np.sqrt(integrate_y_var(o, out["wrms"]))
    for name in ("urms", "vrms", "wrms"):
        out[name][1:Nyp + 1] = np.sqrt(out[name][1:Nyp + 1])

    # compute_TKE_Production (:1408-1545): uw on GYF, uv and wv on GY, each
    # also as z means at each x (vvar_xy, uvar_xy, wvar_xy)
    uw_xy, uv_xy, wv_xy = np.zeros((ny2, Nx)), np.zeros((ny2, Nx)), np.zeros((ny2, Nx))
    for j in range(1, Nyp + 1):
        prod = (u1[j] - ume_xy[j]) * (u3[j] - wme_xy[j])
        out["uw"][j] = np.sum(prod) / NN
        uw_xy[j] = np.sum(prod, axis=0) / float(Nz)
    for j in range(2, Nyp + 1):
        fu = (dyf[j - 1] * (u1[j] - ume_xy[j]) + dyf[j] * (u1[j - 1] - ume_xy[j - 1])) / (2.0 * dy[j])
        fw = (dyf[j - 1] * (u3[j] - wme_xy[j]) + dyf[j] * (u3[j - 1] - wme_xy[j - 1])) / (2.0 * dy[j])
        pu, pw = fu * (u2[j] - vme_xy[j]), fw * (u2[j] - vme_xy[j])
        out["uv"][j] = np.sum(pu) / NN
        out["wv"][j] = np.sum(pw) / NN
        uv_xy[j] = np.sum(pu, axis=0) / float(Nz)
        wv_xy[j] = np.sum(pw, axis=0) / float(Nz)
    if Nz > 1:
        for j in range(1, Nyp + 1):
            out["uu_dudx"][j] = np.sum(uu_xy[j] * dudx_m[j]) / float(Nx)
            out["wu_dwdx"][j] = np.sum(uw_xy[j] * dwdx_m[j]) / float(Nx)
        for j in range(2, Nyp + 1):
            out["vu_dvdx"][j] = np.sum(uv_xy[j] * dvdx_m[j]) / float(Nx)
            out["vv_dvdy"][j] = np.sum((vme_xy[j + 1] - vme_xy[j - 1]) / (gy[j + 1] - gy[j - 1])
                                       * vv_xy[j]) / float(Nx)
            out["uv_dudy"][j] = np.sum((ume_xy[j] - ume_xy[j - 1]) / dy[j] * uv_xy[j]) / float(Nx)
            out["wv_dwdy"][j] = np.sum(((wme_xy[j] - wme_xy[j - 1]) / dy[j] + tws)
                                       * wv_xy[j]) / float(Nx)

    # MKE on GY (:133-150)
    for j in range(2, Nyp + 1):
        out["mke"][j] = 0.5 * np.sum(
            (dyf[j - 1] * ume_xy[j] ** 2 + dyf[j] * ume_xy[j - 1] ** 2) / (2.0 * dy[j])
            + (dyf[j - 1] * (wme_xy[j] + tws * (gyf[j] - 0.5 * p.ly)) ** 2
               + dyf[j] * (wme_xy[j - 1] + tws * (gyf[j - 1] - 0.5 * p.ly)) ** 2) / (2.0 * dy[j])
            + vme_xy[j] ** 2) / float(Nx)
    # gradients of the mean (:153-156) and mean-square shear (:159-171)
    for j in range(1, Nyp + 1):
        out["dudy"][j] = (ume[j] - ume[j - 1]) / (gyf[j] - gyf[j - 1])
        out["dwdy"][j] = (wme[j] - wme[j - 1]) / (gyf[j] - gyf[j - 1])
        ptw.setdefault("shear2", np.zeros_like(u1))[j] = (((u1[j + 1] - u1[j - 1]) / (2.0 * dyf[j])) ** 2
                                                          + ((u3[j + 1] - u3[j - 1]) / (2.0 * dyf[j])) ** 2)
        out["shear"][j] = np.sum(((u1[j + 1] - u1[j - 1]) / (2.0 * dyf[j])) ** 2
                                 + ((u3[j + 1] - u3[j - 1]) / (2.0 * dyf[j])) ** 2) / NN
    out["cp"][:] = o.p_.c[:, 0, 0].real

    # compute_Vorticity (:1555-1752)
    J = slice(1, Nyp + 1)
    Jp, Jm = slice(2, Nyp + 2), slice(0, Nyp)
    cs = zero_cs()
    cs[J, K, I] = (cikz * 0.5 * (cr2[Jp, K, I] + cr2[J, K, I])
                   - (cr3[Jp, K, I] - cr3[Jm, K, I]) / (2.0 * dyf[J, None, None]))
    s = _phys(o, cs) - tws
    for j in range(1, Nyp + 1):
        out["omega_x"][j] = np.sqrt(np.sum(s[j] ** 2) / NN)
    cs = zero_cs()
    cs[J, K, I] = cikx * cr3[J, K, I] - cikz * cr1[J, K, I]
    s = _phys(o, cs)
    for j in range(1, Nyp + 1):
        out["omega_y"][j] = np.sqrt(np.sum(s[j] ** 2) / NN)
    cs = zero_cs()
    cs[J, K, I] = ((cr1[Jp, K, I] - cr1[Jm, K, I]) / (2.0 * dyf[J, None, None])
                   - cikx * 0.5 * (cr2[Jp, K, I] + cr2[J, K, I]))
    s = _phys(o, cs)
    for j in range(1, Nyp + 1):
        out["omega_z"][j] = np.sqrt(np.sum(s[j] ** 2) / NN)

    # scalars (:248-468)
    gx = np.array([(i * p.lx) / Nx for i in range(Nx)])
    ths = []
    u1y_left_b = 0.0
    for n in range(o.Nth):
        prof = {k: np.zeros(ny2) for k in TH_PROFILES}
        c1 = zero_cs()
        c1[J, K, I] = cikx * crth[n][J, K, I]
        c2 = zero_cs()
        c2[J, K, I] = ((crth[0][Jp, K, I] - crth[0][Jm, K, I])
                       / (gyf[2:Nyp + 2] - gyf[0:Nyp])[:, None, None])
        c3 = zero_cs()
        c3[J, K, I] = cikz * crth[n][J, K, I]
        r1, r2, r3 = _phys(o, c1), _phys(o, c2), _phys(o, c3)
        t, tm, txy = th[n], thme[n], thme_xy[n]
        for j in range(1, Nyp + 1):
            prof["thrms"][j] = np.sqrt(np.sum((t[j] - txy[j]) ** 2) / NN)
            # thw_zstar bins (th_1 - thme_xy(n)) times the GY-averaged u2 fluctuation (:346-349)
            ptw.setdefault("thw", np.zeros_like(u1))[j] = (th[0][j] - txy[j]) * 0.5 * (
                (u2[j] - vme_xy[j]) + (u2[j + 1] - vme_xy[j + 1]))
            prof["thv"][j] = np.sum((t[j] - txy[j]) * (0.5 * (u2[j] + u2[j + 1])
                                                       - 0.5 * (vme_xy[j] + vme_xy[j + 1]))) / NN
            prof["thv_m"][j] = np.sum((txy[j] + p.dthdx[n] * (gx - 0.5 * p.lx))
                                      * (0.5 * (vme_xy[j] + vme_xy[j + 1]))) / float(Nx)
            prof["dthdy"][j] = (tm[j] - tm[j - 1]) / (gyf[j] - gyf[j - 1])
            ptw.setdefault("chi", np.zeros_like(u1))[j] = ((r1[j] + p.dthdx[n]) ** 2 + r2[j] ** 2
                                                       + (r3[j] + p.dthdz[n]) ** 2)
            prof["pe_diss"][j] = np.sum((r1[j] + p.dthdx[n]) ** 2 + r2[j] ** 2
                                        + (r3[j] + p.dthdz[n]) ** 2) / NN
        prof["thme"][:] = tm
        if kappa_t is not None:
            kt = kappa_t[n][:, :Nz, :Nx]
            for j in range(1, Nyp + 1):
                prof["kappa_sgs"][j] = np.sum(kt[j]) / NN
        if n == 0:
            u1y_left = np.zeros(ny2)
            for j in range(1, Nyp + 1):
                u1y_left[j] = np.sum(gyf[j] * u1[j, :, 0]) / float(Nz)
            u1y_left_b = integrate_y_var(o, u1y_left)
        ths.append(prof)

    # y-averaged spectrum of u1 on the kz = 0 row, after the physical round
    # trip the reference makes (:650-675)
    f = Field(o.Ny, Nz, Nx)
    f.r[:, :Nz, :Nx] = u1
    o.fft_xz_to_fourier(f)
    cuu = np.abs(f.c[:, 0, :Nxp]) ** 2
    spec = np.zeros(Nxp)
    for j in range(2, Nyp + 1):
        spec += 0.5 * (cuu[j] + cuu[j - 1]) * dy[j]
    spec /= p.ly

    scal = dict(time=o.time, dt=o.delta_t, ubulk=ubulk, urms_b=urms_b, vrms_b=vrms_b,
                wrms_b=wrms_b, u1y_left_b=u1y_left_b)
    res = {"profiles": {k: v[1:Nyp + 1].copy() for k, v in out.items()},
           "th": [{k: v[1:Nyp + 1].copy() for k, v in d.items()} for d in ths],
           "spectrum": spec, "scalars": scal}
    if o.Nth > 0:
        bpe, pdf, bins = compute_bpe(o, th[0], homogeneous_x)
        scal["bpe"] = bpe
        res["th1_pdf"], res["th1_bin"] = pdf, bins
        res["zstar"] = {k: bin_ystar(o, th[0], ptw[k], homogeneous_x) for k in ZSTAR}
    return res


# the fields Bin_Ystar_and_Write averages, in the order diablo_stats returns them
ZSTAR = ("shear2", "thw", "chi", "epsilon", "TKE", "KE")


def _th_bins(o: OracleChannel, th1, homogeneous_x: bool):
    """Bin index of every point of rows jstart_th(1)..jend_th(1) and the bin
    edges th_bin(0:Nbin), as compute_BPE and Bin_Ystar_and_Write form them."""
    from .channel import PI_REF
    p = o.p
    Nx = o.Nx
    nbin = Nx
    d0 = float(p.dthdx[0])
    gx = np.array([(i * p.lx) / Nx for i in range(Nx)])
    s1 = th1 + d0 * (gx - 0.5 * p.lx)[None, None, :]
    j0, j1 = o.jstart_th[0], o.jend_th[0]
    bins = {}
    if not homogeneous_x:
        thmin = -d0 * 0.5 * p.lx * float(np.float32(1.1))
        thmax = d0 * 0.5 * p.lx * float(np.float32(1.1))
        dth = (thmax - thmin) / nbin + 1e-14
        th_bin = np.array([thmin + i * dth for i in range(nbin + 1)])
        for j in range(j0, j1 + 1):
            bins[j] = np.clip(np.trunc((s1[j] - thmin) / dth).astype(np.int64), 0, nbin - 1)
    else:
        ro = o.Ro_inv
        th_bin = np.array([-(ro + 1e-14) * math.cos(i * PI_REF / nbin) for i in range(nbin + 1)])
        for j in range(j0, j1 + 1):
            arg = -np.minimum(np.maximum(s1[j], -ro), ro) / (ro + 1e-14)
            bins[j] = np.clip(np.trunc(np.arccos(arg) * nbin / PI_REF).astype(np.int64), 0, nbin - 1)
    return bins, th_bin


def bin_ystar(o: OracleChannel, th1, field, homogeneous_x: bool):
    """Bin_Ystar_and_Write (for/statistics.f90:1877-1972): the dyf-weighted
    mean of `field` over the points of each th_1 bin (the bins of compute_BPE);
    an empty bin gives 0/0 = NaN, as in the reference."""
    bins, _ = _th_bins(o, th1, homogeneous_x)
    nbin = o.Nx
    pdf, fb = np.zeros(nbin), np.zeros(nbin)
    for j, b in bins.items():
        np.add.at(pdf, b.ravel(), o.dyf[j])
        np.add.at(fb, b.ravel(), (field[j, :o.Nz, :o.Nx] * o.dyf[j]).ravel())
    with np.errstate(invalid="ignore", divide="ignore"):
        return fb / pdf


def compute_bpe(o: OracleChannel, th1, homogeneous_x: bool):
    """compute_BPE (for/statistics.f90:1755-1876): the background potential
    energy of Tseng & Ferziger from the y-weighted PDF of th_1 plus its
    background gradient, on Nbin = Nx bins -- evenly spaced in the
    x-inhomogeneous branch, acos-spaced in [-Ro_inv, Ro_inv] in the homogeneous
    one (the reference's comments swap the two labels; the code is what is
    restated).  ``pi`` is the reference's float32 value and the literal 1.1 is
    single precision.  A negative bin index (th below the evenly spaced range,
    out of bounds in the reference) is taken as bin 0.  Returns (BPE, PDF, the
    lower bin edges th_bin(0:Nbin-1))."""
    p = o.p
    nbin = o.Nx
    bins, th_bin = _th_bins(o, th1, homogeneous_x)
    pdf = np.zeros(nbin)
    for j, b in bins.items():
        np.add.at(pdf, b.ravel(), o.dyf[j])
    pdf = pdf / np.sum(pdf)
    y_r = np.zeros(nbin + 1)
    for i in range(1, nbin + 1):
        y_r[i] = y_r[i - 1] + pdf[i - 1]
    y_r = y_r * p.ly
    bpe = 0.0
    for i in range(nbin):
        bpe = bpe - (0.5 * (th_bin[i + 1] + th_bin[i]) * 0.5 * (y_r[i + 1] + y_r[i])) * \
            (y_r[i + 1] - y_r[i]) / p.ly
    return bpe, pdf, th_bin[:nbin].copy()
