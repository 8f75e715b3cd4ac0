"""numpy restatement of the reference's LES closures (test infrastructure only).

* Type 1, constant Smagorinsky: ``les_chan`` (for/les.f90:20-270, 850-925)
  and its ``eps_sgs1`` statistic (:924-1068),
  and ``les_chan_th`` (for/les.f90:1091-1200), with ``compute_strain_chan``
  (:1463-1510), ``apply_BC_les``/``apply_BC_th_les`` (:2001-2105),
  ``ghost_les_mpi`` and ``ghost_CS2_mpi`` at one y-rank (:2107-2270, :2444-2530).
* Type 2, dynamic Smagorinsky: the reference stops on it
  (for/les.f90:272-277, :1214-1218), so this is a restatement of the published
  model (Germano et al. 1991 with Lilly's 1992 least-squares contraction):
  sharp spectral test filter of width 2 Delta in x and z, coefficient averaged
  over x-z planes, negative eddy viscosity clipped to zero.  It reuses the
  type-1 stress layout (the S2 and dU1/dy, dU3/dy parts stay implicit) and
  replaces the constant -2 c_s^2 Delta^2 by -2 C(y) Delta^2.  Parity for it is
  unpinned against the reference, which has no such model.
* Types 4 and 5, anisotropic minimum dissipation (Rozema; Verstappen):
  ``les_chan`` (:279-850) with ``compute_rotation_chan(_invariant)``
  (:1584-1675), ``compute_strain_chan_invariant`` (:1514-1577) and
  ``compute_all_gradients_chan`` (:1681-1767); the type-5 scalar model of
  ``les_chan_th`` (:1219-1400).  Planes the reference leaves stale (and never
  reads afterwards) are zero here.

Arrays follow oracle/channel.py (numpy index [j, k, i]).
"""
from __future__ import annotations

import numpy as np

from oracle.channel import Field

C_SMAG = 0.17          # for/les.f90:38
C_AMD = 0.2887         # for/les.f90:42
BETA_SGS = 3.0         # for/les.f90:58
TEST_RATIO = 2.0       # test / grid filter width of the dynamic model


_NAMES = ("S1", "S2", "S3", "S4", "S5", "S6", "temp", "fthx", "fthz", "O4", "O5", "O6",
          "SI1", "SI2", "SI3", "SI4", "SI5", "SI6",
          "du1dx", "du2dy", "du3dz", "du2dx", "du3dx", "du1dz", "du2dz", "du1dy", "du3dy")


def _fields(o):
    if not hasattr(o, "_les"):
        mk = lambda: Field(o.Ny, o.Nz, o.Nx)
        o._les = {name: mk() for name in _NAMES}
        for n in range(o.Nth):
            for nm in ("dthdx", "dthdy", "dthdz"):
                o._les[f"{nm}{n}"] = mk()
    return o._les


def apply_bc_les(o):
    """Neumann walls: copy the first interior plane into the ghosts (:2001-2058)."""
    p, Nyp, K, I = o.p, o.Nyp, slice(0, o.twoNkz + 1), slice(0, o.Nxp)
    for cu, bmax, bmin in ((o.u1.c, p.u_bc_ymax, p.u_bc_ymin), (o.u3.c, p.w_bc_ymax, p.w_bc_ymin)):
        if bmax == 1:
            cu[Nyp, K, I] = cu[Nyp - 1, K, I]
            cu[Nyp + 1, K, I] = cu[Nyp, K, I]
        if bmin == 1:
            cu[1, K, I] = cu[2, K, I]
            cu[0, K, I] = cu[1, K, I]


def apply_bc_th_les(o):
    """:2062-2105"""
    p, Nyp, K, I = o.p, o.Nyp, slice(0, o.twoNkz + 1), slice(0, o.Nxp)
    for n in range(o.Nth):
        cth = o.th[n].c
        if p.th_bc_ymax[n] == 1:
            cth[Nyp, K, I] = cth[Nyp - 1, K, I]
            cth[Nyp + 1, K, I] = cth[Nyp, K, I]
        if p.th_bc_ymin[n] == 1:
            cth[1, K, I] = cth[2, K, I]
            cth[0, K, I] = cth[1, K, I]


def compute_strain(o, F):
    """compute_strain_chan (:1463-1510) + ghost_CS2_mpi at one rank."""
    Nyp, K, I = o.Nyp, slice(0, o.twoNkz + 1), slice(0, o.Nxp)
    cikx, cikz = o.cikx[None, None, :o.Nxp], o.cikz[None, :, None]
    cu1, cu2, cu3 = o.u1.c, o.u2.c, o.u3.c
    dy, dyf = o.dy[:, None, None], o.dyf[:, None, None]
    A = slice(0, Nyp + 2)
    F["S1"].c[A, K, I] = cikx * cu1[A, K, I]
    F["S3"].c[A, K, I] = cikz * cu3[A, K, I]
    F["S5"].c[A, K, I] = 0.5 * (cikz * cu1[A, K, I] + cikx * cu3[A, K, I])
    B = slice(0, Nyp + 1)
    F["S2"].c[B, K, I] = (cu2[1:Nyp + 2, K, I] - cu2[B, K, I]) / dyf[B]
    G = slice(1, Nyp + 2)
    F["S4"].c[G, K, I] = 0.5 * ((cu1[G, K, I] - cu1[0:Nyp + 1, K, I]) / dy[G] + cikx * cu2[G, K, I])
    F["S6"].c[G, K, I] = 0.5 * (cikz * cu2[G, K, I] + (cu3[G, K, I] - cu3[0:Nyp + 1, K, I]) / dy[G])
    F["S2"].c[Nyp + 1, K, I] = -10000.0          # ghost_CS2_mpi sentinel (:2521-2527)
    for nm in ("S1", "S2", "S3", "S4", "S5", "S6"):
        o.fft_xz_to_physical(F[nm])


def _dxz(o):
    """dx(1), dz(1): the uniform x and z spacings (for/domain.f90)."""
    return o.p.lx / o.Nx, o.p.lz / o.Nz


def compute_rotation(o, F, invariant):
    """compute_rotation_chan (:1584-1620) / _invariant (:1624-1675)."""
    Nyp, K, I = o.Nyp, slice(0, o.twoNkz + 1), slice(0, o.Nxp)
    cikx, cikz = o.cikx[None, None, :o.Nxp], o.cikz[None, :, None]
    cu1, cu2, cu3 = o.u1.c, o.u2.c, o.u3.c
    A = slice(0, Nyp + 2)
    G = slice(1, Nyp + 2)
    Gm = slice(0, Nyp + 1)
    dyG = o.dy[G, None, None]
    for nm in ("O4", "O5", "O6"):
        F[nm].c[:] = 0
    if not invariant:
        F["O5"].c[A, K, I] = 0.5 * (cikz * cu1[A, K, I] - cikx * cu3[A, K, I])
        F["O4"].c[G, K, I] = 0.5 * ((cu1[G, K, I] - cu1[Gm, K, I]) / dyG - cikx * cu2[G, K, I])
        F["O6"].c[G, K, I] = 0.5 * (cikz * cu2[G, K, I] - (cu3[G, K, I] - cu3[Gm, K, I]) / dyG)
    else:
        dx, dz = _dxz(o)
        deltax, deltaz = dx * BETA_SGS, dz * BETA_SGS
        deltay = (o.dy[G] * 2.0)[:, None, None]
        F["O5"].c[A, K, I] = 0.5 * (cikz * cu1[A, K, I] * (deltaz / deltax)
                                    - cikx * cu3[A, K, I] * (deltax / deltaz))
        F["O4"].c[G, K, I] = 0.5 * ((cu1[G, K, I] - cu1[Gm, K, I]) / dyG * (deltay / deltax)
                                    - cikx * cu2[G, K, I] * (deltax / deltay))
        F["O6"].c[G, K, I] = 0.5 * (cikz * cu2[G, K, I] * (deltaz / deltay)
                                    - (cu3[G, K, I] - cu3[Gm, K, I]) / dyG * (deltay / deltaz))
    for nm in ("O4", "O5", "O6"):
        o.fft_xz_to_physical(F[nm])


def compute_strain_invariant(o, F):
    """compute_strain_chan_invariant (:1514-1577)."""
    Nyp, K, I = o.Nyp, slice(0, o.twoNkz + 1), slice(0, o.Nxp)
    cikx, cikz = o.cikx[None, None, :o.Nxp], o.cikz[None, :, None]
    cu1, cu2, cu3 = o.u1.c, o.u2.c, o.u3.c
    dx, dz = _dxz(o)
    deltax, deltaz = dx * BETA_SGS, dz * BETA_SGS
    A = slice(0, Nyp + 2)
    B = slice(0, Nyp + 1)
    G = slice(1, Nyp + 2)
    Gm = slice(0, Nyp + 1)
    dyG = o.dy[G, None, None]
    deltay = (o.dy[G] * 2.0)[:, None, None]
    for nm in ("SI1", "SI2", "SI3", "SI4", "SI5", "SI6"):
        F[nm].c[:] = 0
    F["SI1"].c[A, K, I] = cikx * cu1[A, K, I]
    F["SI3"].c[A, K, I] = cikz * cu3[A, K, I]
    F["SI5"].c[A, K, I] = 0.5 * (cikz * cu1[A, K, I] * (deltaz / deltax)
                                 + cikx * cu3[A, K, I] * (deltax / deltaz))
    F["SI2"].c[B, K, I] = (cu2[1:Nyp + 2, K, I] - cu2[B, K, I]) / o.dyf[B, None, None]
    F["SI4"].c[G, K, I] = 0.5 * ((cu1[G, K, I] - cu1[Gm, K, I]) / dyG * (deltay / deltax)
                                 + cikx * cu2[G, K, I] * (deltax / deltay))
    F["SI6"].c[G, K, I] = 0.5 * (cikz * cu2[G, K, I] * (deltaz / deltay)
                                 + (cu3[G, K, I] - cu3[Gm, K, I]) / dyG * (deltay / deltaz))
    F["SI2"].c[Nyp + 1, K, I] = -10000.0          # ghost_CS2_mpi sentinel
    for nm in ("SI1", "SI2", "SI3", "SI4", "SI5", "SI6"):
        o.fft_xz_to_physical(F[nm])


def compute_all_gradients(o, F):
    """compute_all_gradients_chan (:1681-1767)."""
    Nyp, K, I = o.Nyp, slice(0, o.twoNkz + 1), slice(0, o.Nxp)
    cikx, cikz = o.cikx[None, None, :o.Nxp], o.cikz[None, :, None]
    cu1, cu2, cu3 = o.u1.c, o.u2.c, o.u3.c
    A = slice(0, Nyp + 2)
    G = slice(1, Nyp + 2)
    Gm = slice(0, Nyp + 1)
    dyG = o.dy[G, None, None]
    names = ["du1dx", "du2dy", "du3dz", "du2dx", "du3dx", "du1dz", "du2dz", "du1dy", "du3dy"]
    for n in range(o.Nth):
        names += [f"dthdx{n}", f"dthdy{n}", f"dthdz{n}"]
    for nm in names:
        F[nm].c[:] = 0
    F["du1dx"].c[A, K, I] = cikx * cu1[A, K, I]
    F["du1dz"].c[A, K, I] = cikz * cu1[A, K, I]
    F["du2dx"].c[A, K, I] = cikx * cu2[A, K, I]
    F["du2dz"].c[A, K, I] = cikz * cu2[A, K, I]
    F["du3dx"].c[A, K, I] = cikx * cu3[A, K, I]
    F["du3dz"].c[A, K, I] = cikz * cu3[A, K, I]
    F["du1dy"].c[G, K, I] = (cu1[G, K, I] - cu1[Gm, K, I]) / dyG
    # d u2/dy at j uses dyf(j-1), as the reference does (:1710)
    F["du2dy"].c[G, K, I] = (cu2[G, K, I] - cu2[Gm, K, I]) / o.dyf[Gm, None, None]
    F["du3dy"].c[G, K, I] = (cu3[G, K, I] - cu3[Gm, K, I]) / dyG
    for n in range(o.Nth):
        cth = o.th[n].c
        F[f"dthdx{n}"].c[G, K, I] = cikx * cth[G, K, I]
        F[f"dthdz{n}"].c[G, K, I] = cikz * cth[G, K, I]
        F[f"dthdy{n}"].c[G, K, I] = (cth[G, K, I] - cth[Gm, K, I]) / dyG
    for nm in names:
        o.fft_xz_to_physical(F[nm])


def _amd_terms(S, O, j, dlt, gyf_point, o, invariant):
    """-(I3 - I4) and the denominator of the AMD coefficient at one plane.
    S, O: strain (or scaled-invariant strain) and rotation dicts (physical);
    dlt = (deltax, deltay, deltaz) weights; gyf_point selects the GYF form
    (GY quantities averaged) or the GY form (GYF quantities interpolated)
    of for/les.f90:298-350 / :357-460 (Rozema) and :591-650 / :655-735
    (Verstappen, all weights 1)."""
    dx, dy, dz = dlt
    if gyf_point:
        av = lambda f: 0.5 * (f[j + 1] + f[j])
        a1, a2, a3, a5 = S["1"][j], S["2"][j], S["3"][j], S["5"][j]
        a4, a6 = av(S["4"]), av(S["6"])
        o4, o5, o6 = av(O["4"]), O["5"][j], av(O["6"])
    else:
        ip = lambda f: (f[j] * o.dyf[j - 1] + f[j - 1] * o.dyf[j]) / (2.0 * o.dy[j])
        a1, a2, a3, a5 = ip(S["1"]), ip(S["2"]), ip(S["3"]), ip(S["5"])
        a4, a6 = S["4"][j], S["6"][j]
        o4, o5, o6 = O["4"][j], ip(O["5"]), O["6"][j]
    i3 = (dx * a1 ** 3.0 + dy * a2 ** 3.0 + dz * a3 ** 3.0
          + (2.0 * dx + dy) * a1 * a4 ** 2.0
          + (2.0 * dx + dz) * a1 * a5 ** 2.0
          + (2.0 * dy + dx) * a2 * a4 ** 2.0
          + (2.0 * dy + dz) * a2 * a6 ** 2.0
          + (2.0 * dz + dx) * a3 * a5 ** 2.0
          + (2.0 * dz + dy) * a3 * a6 ** 2.0
          + 2.0 * (dx + dy + dz) * a4 * a5 * a6)
    num = (-i3
           - dy * a1 * o4 ** 2.0 - dz * a1 * o5 ** 2.0
           - dx * a2 * o4 ** 2.0 - dz * a2 * o6 ** 2.0
           - dx * a3 * o5 ** 2.0 - dy * a3 * o6 ** 2.0
           - 2.0 * dz * a4 * o5 * o6
           + 2.0 * dy * a5 * o4 * o6
           - 2.0 * dx * a6 * o4 * o5)
    den = (a1 ** 2.0 + a2 ** 2.0 + a3 ** 2.0 + 2.0 * a4 ** 2.0 + 2.0 * o4 ** 2.0
           + 2.0 * a5 ** 2.0 + 2.0 * o5 ** 2.0 + 2.0 * a6 ** 2.0 + 2.0 * o6 ** 2.0)
    pos = num > 0.0
    return np.where(pos, num / np.where(pos, den, 1.0), 0.0)


def _amd_coefficients(o, F, model):
    """max(0, -(I3 - I4)) / (I1 - I2) at GYF (s1) and GY (temp) points.
    Rozema (4): weights delta_i^2, GYF rows 1..Nyp, GY rows 2..Nyp+1, with
    deltay^2 = (2 dy(j))^2 at both kinds of point (:290-298, :356).
    Verstappen (5): scaled-invariant strain and rotation, unit weights, GYF
    rows jstart..jend, GY rows 2..Nyp (:589-700)."""
    Nyp = o.Nyp
    O = {"4": F["O4"].r, "5": F["O5"].r, "6": F["O6"].r}
    s1 = np.zeros_like(F["S1"].r)
    temp = np.zeros_like(F["S1"].r)
    if model == 4:
        S = {str(q): F[f"S{q}"].r for q in range(1, 7)}
        dx, dz = _dxz(o)
        deltax, deltaz = (dx * BETA_SGS) ** 2.0, (dz * BETA_SGS) ** 2.0
        for j in range(1, Nyp + 1):
            s1[j] = _amd_terms(S, O, j, (deltax, (o.dy[j] * 2.0) ** 2.0, deltaz), True, o, False)
        for j in range(2, Nyp + 2):
            temp[j] = _amd_terms(S, O, j, (deltax, (o.dy[j] * 2.0) ** 2.0, deltaz), False, o, False)
    else:
        S = {str(q): F[f"SI{q}"].r for q in range(1, 7)}
        for j in range(o.jstart, o.jend + 1):
            s1[j] = _amd_terms(S, O, j, (1.0, 1.0, 1.0), True, o, True)
        for j in range(2, Nyp + 1):
            temp[j] = _amd_terms(S, O, j, (1.0, 1.0, 1.0), False, o, True)
    return s1, temp


def _amd_deltas(o, model):
    """delta_yf, delta_y of the AMD models (:500-516, :776-797)."""
    n = o.Ny + 2
    delta_yf = np.zeros(n)
    delta_y = np.zeros(n)
    dx, dz = _dxz(o)
    for j in range(1, o.Nyp + 2):
        if model == 4:
            delta_yf[j] = -2.0 * C_AMD ** 2.0
            delta_y[j] = -2.0 * C_AMD ** 2.0
        else:
            delta_yf[j] = -2.0 * C_AMD ** 2.0 * 3.0 / (1.0 / (dx * BETA_SGS) ** 2.0
                                                       + 1.0 / (o.dyf[j] * 2.0) ** 2.0
                                                       + 1.0 / (dz * BETA_SGS) ** 2.0)
            delta_y[j] = -2.0 * C_AMD ** 2.0 * 3.0 / (1.0 / (dx * BETA_SGS) ** 2.0
                                                      + 1.0 / (o.dy[j] * 2.0) ** 2.0
                                                      + 1.0 / (dz * BETA_SGS) ** 2.0)
    return delta_yf, delta_y


def _interp_gy(o, a, j):
    """(a(j) dyf(j-1) + a(j-1) dyf(j)) / (2 dy(j)): a GYF field at GY point j."""
    return (a[j] * o.dyf[j - 1] + a[j - 1] * o.dyf[j]) / (2.0 * o.dy[j])


def _strain_norms(o, S):
    """|S| at GYF points (j = 1..Nyp) and at GY points (j = 1..Nyp+1) (:123-166)."""
    Nyp = o.Nyp
    s_f = np.zeros_like(S["S1"])
    s_g = np.zeros_like(S["S1"])
    for j in range(1, Nyp + 1):
        s_f[j] = np.sqrt(2.0 * S["S1"][j] ** 2.0
                         + 4.0 * (0.5 * (S["S4"][j + 1] + S["S4"][j])) ** 2.0
                         + 4.0 * S["S5"][j] ** 2.0
                         + 2.0 * S["S2"][j] ** 2.0
                         + 4.0 * (0.5 * (S["S6"][j + 1] + S["S6"][j])) ** 2.0
                         + 2.0 * S["S3"][j] ** 2.0)
    for j in range(1, Nyp + 2):
        s_g[j] = np.sqrt(2.0 * _interp_gy(o, S["S1"], j) ** 2.0
                         + 4.0 * S["S4"][j] ** 2.0
                         + 4.0 * _interp_gy(o, S["S5"], j) ** 2.0
                         + 2.0 * _interp_gy(o, S["S2"], j) ** 2.0
                         + 4.0 * S["S6"][j] ** 2.0
                         + 2.0 * _interp_gy(o, S["S3"], j) ** 2.0)
    return s_f, s_g


def _filter_widths(o):
    """delta_yf (GYF) and delta_y (GY): -2 c^2 Delta^2 without the constant (:224-245)."""
    dx1 = o.p.lx / o.Nx
    dz1 = o.p.lz / o.Nz
    d2f = np.zeros(o.Ny + 2)
    d2g = np.zeros(o.Ny + 2)
    for j in range(1, o.Nyp + 1):
        d2f[j] = (dx1 * BETA_SGS * o.dyf[j] * 1.0 * dz1 * BETA_SGS) ** (2.0 / 3.0)
    for j in range(1, o.Nyp + 2):
        d2g[j] = (dx1 * BETA_SGS * o.dy[j] * 2.0 * dz1 * BETA_SGS) ** (2.0 / 3.0)
    return d2f, d2g


def _test_filter(o, phys):
    """Sharp spectral test filter of width 2 Delta on physical planes [j, k, i]:
    keep |kx| <= Nkx/2 and |kz| <= Nkz/2 of the resolved band."""
    Nx, Nz = o.Nx, o.Nz
    f = np.fft.rfft2(phys[:, :Nz, :Nx], axes=(1, 2))
    kxi = np.arange(f.shape[2])
    kzi = np.abs(np.fft.fftfreq(Nz, 1.0 / Nz))
    mask = (kxi[None, :] <= o.Nkx // 2) & (kzi[:, None] <= o.Nkz // 2)
    f *= mask[None]
    out = np.zeros_like(phys)
    out[:, :Nz, :Nx] = np.fft.irfft2(f, s=(Nz, Nx), axes=(1, 2))
    return out


def _dynamic_coefficient(o, S, s_f, d2f):
    """C(y) at GYF points from the Germano identity with Lilly's contraction.
    Velocities, strain and |S| are taken at GYF points (u2, S4, S6 averaged
    from the neighbouring GY points); <.> is the x-z plane mean."""
    Nyp, Nx, Nz = o.Nyp, o.Nx, o.Nz
    R = slice(1, Nyp + 1)
    u1, u2, u3 = o.u1.r, o.u2.r, o.u3.r
    U = [np.zeros_like(u1) for _ in range(3)]
    U[0][R] = u1[R]
    U[1][R] = 0.5 * (u2[R] + u2[2:Nyp + 2])
    U[2][R] = u3[R]
    Sf = {"11": S["S1"], "22": S["S2"], "33": S["S3"], "13": S["S5"]}
    S12 = np.zeros_like(u1)
    S23 = np.zeros_like(u1)
    S12[R] = 0.5 * (S["S4"][R] + S["S4"][2:Nyp + 2])
    S23[R] = 0.5 * (S["S6"][R] + S["S6"][2:Nyp + 2])
    Sf["12"] = S12
    Sf["23"] = S23
    pairs = (("11", 0, 0), ("22", 1, 1), ("33", 2, 2), ("12", 0, 1), ("13", 0, 2), ("23", 1, 2))
    weight = {"11": 1.0, "22": 1.0, "33": 1.0, "12": 2.0, "13": 2.0, "23": 2.0}
    Uh = [_test_filter(o, u) for u in U]
    Sh = {nm: _test_filter(o, Sf[nm]) for nm, _, _ in pairs}
    sh = np.zeros_like(u1)
    sh[R] = np.sqrt(sum(weight[nm] * 2.0 * Sh[nm][R] ** 2 for nm, _, _ in pairs))
    num = np.zeros(o.Ny + 2)
    den = np.zeros(o.Ny + 2)
    d2 = d2f[:, None, None]
    for nm, a, b in pairs:
        L = _test_filter(o, U[a] * U[b]) - Uh[a] * Uh[b]
        M = 2.0 * d2 * (_test_filter(o, s_f * Sf[nm]) - TEST_RATIO ** 2 * sh * Sh[nm])
        num[R] += weight[nm] * np.mean((L * M)[R, :Nz, :Nx], axis=(1, 2))
        den[R] += weight[nm] * np.mean((M * M)[R, :Nz, :Nx], axis=(1, 2))
    C = np.zeros(o.Ny + 2)
    ok = den[R] > 0
    C[R] = np.where(ok, num[R] / np.where(ok, den[R], 1.0), 0.0)
    return C


def les_chan(o):
    """Eddy viscosity and SGS stress divergence for the momentum equations."""
    p = o.p
    Nyp, Nx, Nz, K, I = o.Nyp, o.Nx, o.Nz, slice(0, o.twoNkz + 1), slice(0, o.Nxp)
    j1, j2 = o.jstart, Nyp - 1                       # rankY == NprocY-1 branch (:62-66)
    o.apply_bc_vel_post()                             # :80
    o.apply_bc_th_post()                              # :81
    apply_bc_les(o)                                   # :89
    apply_bc_th_les(o)                                # :90
    F = _fields(o)
    model = p.les_model_type
    if model not in (1, 2, 4, 5):
        raise NotImplementedError(f"LES model {model}")
    compute_strain(o, F)
    if model == 4:
        compute_rotation(o, F, invariant=False)                   # :283
    elif model == 5:
        compute_strain_invariant(o, F)                            # :576
        compute_rotation(o, F, invariant=True)                    # :579
        compute_all_gradients(o, F)                               # :582
    for f in (o.u1, o.u2, o.u3):                      # :118-120
        o.fft_xz_to_physical(f)
    S = {nm: F[nm].r for nm in ("S1", "S2", "S3", "S4", "S5", "S6")}
    R = slice(1, Nyp + 1)
    G = slice(1, Nyp + 2)
    u1, u3 = o.u1.r, o.u3.r
    dyg = o.dy[G, None, None]
    nt = o.nu_t
    nt[:] = 0.0
    if model in (4, 5):
        s1, temp = _amd_coefficients(o, F, model)
        rows = range(1, Nyp + 1) if model == 4 else range(o.jstart, o.jend + 1)
        for j in rows:                                            # :467-478, :742-751
            S["S1"][j] = s1[j] * S["S1"][j]
            S["S5"][j] = s1[j] * S["S5"][j]
            S["S2"][j] = 0.0
            S["S3"][j] = s1[j] * S["S3"][j]
        for j in range(2, Nyp + 2):                               # :483-494, :756-768
            S["S4"][j] = temp[j] * (S["S4"][j] - 0.5 * (u1[j] - u1[j - 1]) / o.dy[j])
            S["S6"][j] = temp[j] * (S["S6"][j] - 0.5 * (u3[j] - u3[j - 1]) / o.dy[j])
        delta_yf, delta_y = _amd_deltas(o, model)
        for j in range(2, (Nyp if model == 4 else Nyp + 1) + 1):  # :521-527, :802-808
            nt[j, :Nz, :Nx] = -0.5 * delta_y[j] * temp[j, :Nz, :Nx]
    else:
        s_f, s_g = _strain_norms(o, S)
        d2f, d2g = _filter_widths(o)
        if model == 1:
            cf_ = np.full(o.Ny + 2, C_SMAG ** 2.0)
            cg_ = cf_
        else:
            Cf = _dynamic_coefficient(o, S, s_f, d2f)
            cf_ = Cf
            cg_ = np.zeros(o.Ny + 2)
            for j in range(2, Nyp + 1):                   # C at GY points
                cg_[j] = (Cf[j] * o.dyf[j - 1] + Cf[j - 1] * o.dyf[j]) / (2.0 * o.dy[j])
        delta_yf = -2.0 * cf_ * d2f
        delta_y = -2.0 * cg_ * d2g
        if model == 1:
            S["S1"][R] = s_f[R] * S["S1"][R]              # :169-178
            S["S5"][R] = s_f[R] * S["S5"][R]
            S["S2"][R] = 0.0
            S["S3"][R] = s_f[R] * S["S3"][R]
            S["S4"][G] = s_g[G] * (S["S4"][G] - 0.5 * (u1[G] - u1[0:Nyp + 1]) / dyg)   # :181-193
            S["S6"][G] = s_g[G] * (S["S6"][G] - 0.5 * (u3[G] - u3[0:Nyp + 1]) / dyg)
            for j in range(2, Nyp + 1):                   # :235-241
                nt[j, :Nz, :Nx] = -0.5 * delta_y[j] * s_g[j, :Nz, :Nx]
        else:
            # clipped viscosities at GY (nu_t) and GYF (nuf); the stresses carry
            # -2 nu S themselves, so the delta scalings below become ones
            for j in range(2, Nyp + 1):
                nt[j, :Nz, :Nx] = np.maximum(-0.5 * delta_y[j] * s_g[j, :Nz, :Nx], 0.0)
            nuf = np.zeros_like(nt)
            for j in range(1, Nyp + 1):
                nuf[j] = np.maximum(-0.5 * delta_yf[j] * s_f[j], 0.0)
            for nm in ("S1", "S3", "S5"):
                S[nm][R] = -2.0 * nuf[R] * S[nm][R]
            S["S2"][R] = 0.0
            S["S4"][G] = -2.0 * nt[G] * (S["S4"][G] - 0.5 * (u1[G] - u1[0:Nyp + 1]) / dyg)
            S["S6"][G] = -2.0 * nt[G] * (S["S6"][G] - 0.5 * (u3[G] - u3[0:Nyp + 1]) / dyg)
            delta_yf = np.ones(o.Ny + 2)
            delta_y = np.ones(o.Ny + 2)
    nt[1] = 0.0; nt[2] = 0.0; nt[Nyp] = 0.0; nt[Nyp + 1] = 0.0   # ghost_les_mpi (:2241-2262)
    for nm in ("S1", "S3", "S4", "S5", "S6"):          # :245-253
        o.fft_xz_to_fourier(F[nm])
    C1, C3, C4, C5, C6 = (F[nm].c for nm in ("S1", "S3", "S4", "S5", "S6"))
    C1[R, K, I] *= delta_yf[R, None, None]            # :256-274
    C5[R, K, I] *= delta_yf[R, None, None]
    C3[R, K, I] *= delta_yf[R, None, None]
    C4[G, K, I] *= delta_y[G, None, None]
    C6[G, K, I] *= delta_y[G, None, None]
    cikx, cikz = o.cikx[None, None, :o.Nxp], o.cikz[None, :, None]
    cf1, cf2, cf3 = o.f1.c, o.f2.c, o.f3.c
    J = slice(j1, j2 + 1)
    JP = slice(j1 + 1, j2 + 2)
    dyf = o.dyf[J, None, None]
    cf1[J, K, I] = cf1[J, K, I] - cikx * C1[J, K, I] - (C4[JP, K, I] - C4[J, K, I]) / dyf - cikz * C5[J, K, I]
    cf3[J, K, I] = cf3[J, K, I] - cikx * C5[J, K, I] - (C6[JP, K, I] - C6[J, K, I]) / dyf - cikz * C3[J, K, I]
    J2 = slice(2, Nyp + 1)
    cf2[J2, K, I] = cf2[J2, K, I] - cikx * C4[J2, K, I] - cikz * C6[J2, K, I]
    temp = F["temp"]
    for u, ck in ((u1, cikx), (u3, cikz)):           # :862-880
        temp.r[J2, :Nz, :Nx] = nt[J2, :Nz, :Nx] * (u[J2, :Nz, :Nx] - u[1:Nyp, :Nz, :Nx]) / o.dy[J2, None, None]
        o.fft_xz_to_fourier(temp)
        cf2[J2, K, I] = cf2[J2, K, I] + ck * temp.c[J2, K, I]
    if getattr(o, "flag_save_les", False) and o.rk_step == 1:     # :924
        o.eps_sgs1 = eps_sgs1(o, C1, C3, C4, C5, C6, nt)
        o.flag_save_les = False


def eps_sgs1(o, C1, C3, C4, C5, C6, nt):
    """eps_sgs1_mean of les_chan (for/les.f90:940-1068): the plane mean of
    u_i times the SGS force of cf_i, evaluated as the reference does, each force
    transformed to physical space and multiplied point by point; the u1 and u3
    parts are averaged from GYF onto GY.  Velocities are the physical fields of
    les_chan (after the LES wall values).  Returns (Ny,) for j = 1..Nyp."""
    Nyp, Nx, Nz, K, I = o.Nyp, o.Nx, o.Nz, slice(0, o.twoNkz + 1), slice(0, o.Nxp)
    cikx, cikz = o.cikx[None, None, :o.Nxp], o.cikz[None, :, None]
    u1, u2, u3 = (f.r[:, :Nz, :Nx] for f in (o.u1, o.u2, o.u3))
    eps = np.zeros(o.Ny + 2)
    tmp = Field(o.Ny, o.Nz, o.Nx)
    R, RP, J2 = slice(1, Nyp + 1), slice(2, Nyp + 2), slice(2, Nyp + 1)
    dyf = o.dyf[R, None, None]
    # parts of CF1 and CF3 on GYF, interpolated onto GY (:944-984)
    for u, first, pair, last in ((u1, C1, C4, C5), (u3, C5, C6, C3)):
        tmp.buf[:] = 0.0
        tmp.c[R, K, I] = -cikx * first[R, K, I] - (pair[RP, K, I] - pair[R, K, I]) / dyf - cikz * last[R, K, I]
        o.fft_xz_to_physical(tmp)
        t = tmp.r[:, :Nz, :Nx]
        for j in range(2, Nyp + 1):
            eps[j] += np.sum(0.5 * (u[j] * t[j] + u[j - 1] * t[j - 1]))
    # part of CF2 on GY (:986-1003)
    tmp.buf[:] = 0.0
    tmp.c[J2, K, I] = -cikx * C4[J2, K, I] - cikz * C6[J2, K, I]
    o.fft_xz_to_physical(tmp)
    for j in range(2, Nyp + 1):
        eps[j] += np.sum(tmp.r[j, :Nz, :Nx] * u2[j])
    # the explicit cross terms of CF2 (:1004-1052)
    for u, ck in ((u1, cikx), (u3, cikz)):
        tmp.buf[:] = 0.0
        tmp.r[J2, :Nz, :Nx] = nt[J2, :Nz, :Nx] * (u[J2] - u[1:Nyp]) / o.dy[J2, None, None]
        o.fft_xz_to_fourier(tmp)
        tmp.c[J2, K, I] = ck * tmp.c[J2, K, I]
        o.fft_xz_to_physical(tmp)
        for j in range(2, Nyp + 1):
            eps[j] += np.sum(tmp.r[j, :Nz, :Nx] * u2[j])
    eps /= float(Nx * Nz)                                          # :1064-1068
    return eps[1:Nyp + 1].copy()


def _amd_scalar(o, F, n):
    """Type-5 scalar coefficients for scalar n (for/les.f90:1239-1330, numerators
    :1245 and :1285):
    s1_th at GYF rows jstart_th..jend_th, temp_th at GY rows 2..Nyp+1."""
    dx, dz = _dxz(o)
    deltax, deltaz = dx * BETA_SGS, dz * BETA_SGS
    g = {nm: F[nm].r for nm in ("du1dx", "du2dy", "du3dz", "du2dx", "du3dx", "du1dz", "du2dz",
                                "du1dy", "du3dy")}
    tx, ty, tz = F[f"dthdx{n}"].r, F[f"dthdy{n}"].r, F[f"dthdz{n}"].r
    s1 = np.zeros_like(tx)
    temp = np.zeros_like(tx)
    for j in range(o.jstart_th[n], o.jend_th[n] + 1):
        deltay = o.dyf[j] * 2.0
        tyf = 0.5 * (ty[j + 1] + ty[j])
        num = -(deltax ** 2 * g["du1dx"][j] * tx[j] ** 2
                + deltay ** 2 * g["du2dy"][j] * tyf ** 2
                + deltaz ** 2 * g["du3dz"][j] * tz[j] ** 2
                + (deltay ** 2 * 0.5 * (g["du1dy"][j + 1] + g["du1dy"][j])
                   + deltax ** 2 * 0.5 * (g["du2dx"][j + 1] + g["du2dx"][j])) * tx[j] * tyf
                + (deltaz ** 2 * g["du1dz"][j] + deltax ** 2 * g["du3dx"][j]) * tx[j] * tz[j]
                + (deltaz ** 2 * 0.5 * (g["du2dz"][j + 1] + g["du2dz"][j])
                   + deltay ** 2 * 0.5 * (g["du3dy"][j + 1] + g["du3dy"][j])) * tyf * tz[j])
        den = (deltax * tx[j]) ** 2 + (deltay * tyf) ** 2 + (deltaz * tz[j]) ** 2
        pos = num > 0.0
        s1[j] = np.where(pos, num / np.where(pos, den, 1.0), 0.0)
    for j in range(2, o.Nyp + 2):
        deltay = o.dy[j] * 2.0
        ip = lambda f: (f[j] * o.dyf[j - 1] + f[j - 1] * o.dyf[j]) / (2.0 * o.dy[j])
        txg, tzg, tyg = ip(tx), ip(tz), ty[j]
        num = -(deltax ** 2 * ip(g["du1dx"]) * txg ** 2
                + deltay ** 2 * ip(g["du2dy"]) * tyg ** 2
                + deltaz ** 2 * ip(g["du3dz"]) * tzg ** 2
                + (deltay ** 2 * g["du1dy"][j] + deltax ** 2 * g["du2dx"][j]) * txg * tyg
                + (deltaz ** 2 * ip(g["du1dz"]) + deltax ** 2 * ip(g["du3dx"])) * txg * tzg
                + (deltaz ** 2 * g["du2dz"][j] + deltay ** 2 * g["du3dy"][j]) * tyg * tzg)
        den = (deltax * txg) ** 2 + (deltay * tyg) ** 2 + (deltaz * tzg) ** 2
        pos = num > 0.0
        temp[j] = np.where(pos, num / np.where(pos, den, 1.0), 0.0)
    return s1, temp


def les_chan_th(o):
    """SGS scalar flux: kappa_t = nu_t with the horizontal flux through FFTs
    (types 1, 2, 4; :1130-1200), or the AMD scalar model (type 5; :1219-1412)."""
    p = o.p
    Nyp, Nx, Nz, K, I = o.Nyp, o.Nx, o.Nz, slice(0, o.twoNkz + 1), slice(0, o.Nxp)
    if p.les_model_type not in (1, 2, 4, 5):
        raise NotImplementedError(f"LES model {p.les_model_type}")
    if p.les_model_type == 5:
        F = _fields(o)
        delta_yf, delta_y = _amd_deltas(o, 5)
        cikx, cikz = o.cikx[None, None, :o.Nxp], o.cikz[None, :, None]
        for n in range(o.Nth):
            s1, temp = _amd_scalar(o, F, n)
            Jt = slice(o.jstart_th[n], o.jend_th[n] + 1)
            fx, fz = F["fthx"], F["fthz"]
            fx.r[:] = 0.0
            fz.r[:] = 0.0
            fx.r[Jt] = s1[Jt] * F[f"dthdx{n}"].r[Jt]                 # :1334-1340
            fz.r[Jt] = s1[Jt] * F[f"dthdz{n}"].r[Jt]
            kt = o.kappa_t[n]
            kt[:] = 0.0
            for j in range(2, Nyp + 1):                                # :1372-1378
                kt[j, :Nz, :Nx] = -0.5 * delta_y[j] * temp[j, :Nz, :Nx]
            kt[1] = 0.0; kt[2] = 0.0; kt[Nyp] = 0.0; kt[Nyp + 1] = 0.0   # ghost_les_th_mpi
            o.fft_xz_to_fourier(fx)
            o.fft_xz_to_fourier(fz)
            G = slice(1, Nyp + 2)
            fx.c[G, K, I] = 0.5 * delta_yf[G, None, None] * fx.c[G, K, I]    # :1391-1399
            fz.c[G, K, I] = 0.5 * delta_yf[G, None, None] * fz.c[G, K, I]
            cfth = o.fth[n].c
            cfth[Jt, K, I] = cfth[Jt, K, I] - cikx * fx.c[Jt, K, I] - cikz * fz.c[Jt, K, I]
        for n in range(o.Nth):
            o.fft_xz_to_physical(o.th[n])
        return
    G = slice(1, Nyp + 2)
    for n in range(o.Nth):
        o.kappa_t[n][G] = 1.0 * o.nu_t[G]
    cs1 = o.s1
    for n in range(o.Nth):
        cth, cfth = o.th[n].c, o.fth[n].c
        Jt = slice(o.jstart_th[n], o.jend_th[n] + 1)
        for ck in (o.cikx[None, None, :o.Nxp], o.cikz[None, :, None]):
            cs1.c[G, K, I] = ck * cth[G, K, I]
            o.fft_xz_to_physical(cs1)
            cs1.r[G, :Nz, :Nx] = o.kappa_t[n][G, :Nz, :Nx] * cs1.r[G, :Nz, :Nx]
            o.fft_xz_to_fourier(cs1)
            cfth[Jt, K, I] = cfth[Jt, K, I] + ck * cs1.c[Jt, K, I]
    for n in range(o.Nth):
        o.fft_xz_to_physical(o.th[n])
