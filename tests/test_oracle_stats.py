"""Known-answer tests of the plane-statistics oracle (oracle/stats.py, the
restatement of save_stats_chan, for/statistics.f90:44-712) and a cross-check
of its physical-space sums against a Parseval evaluation from the Fourier
coefficients -- the formulation the CUDA library uses.

The known answers use fields built from single Fourier modes in physical
space, whose plane averages are known in closed form: <cos^2> = 1/2, products
of different modes average to 0, and derivatives of the modes use the
reference's wavenumbers (float32 pi).
"""
import math

import numpy as np
import pytest

from tests.helpers import small_params, grid_for, initial_fields


def _oracle(p, gy):
    from oracle.channel import OracleChannel
    return OracleChannel(p, gy)


def _set_phys(o, fld, arr):
    fld.r[:] = 0.0
    fld.r[:, :o.Nz, :o.Nx] = arr
    o.fft_xz_to_fourier(fld)


def _modal_case():
    p = small_params(nx=32, ny=33, nz=24, n_th=1, ro=2.0, delta=0.5, dthdx=[0.3], dthdz=[-0.2],
                     re=250.0)
    gy = grid_for(p)
    o = _oracle(p, gy)
    y = o.gyf
    x = np.arange(o.Nx) * (2 * np.pi / o.Nx)
    z = np.arange(o.Nz) * (2 * np.pi / o.Nz)
    cx = np.cos(x)[None, None, :]
    cz = np.cos(z)[None, :, None]
    one = np.ones((1, o.Nz, o.Nx))
    U, A = 1.0 - y ** 2, 0.1 * np.sin(2.0 * y)
    V0, V = 0.05 * (1.0 - y ** 2) * y, 0.07 * np.cos(y)
    W = 0.2 * y * (1.0 - y ** 2)
    T, B, C = 0.5 * y + 0.1 * y ** 2, 0.03 * np.cos(3 * y), 0.02 * y
    _set_phys(o, o.u1, U[:, None, None] * one + A[:, None, None] * cz)
    _set_phys(o, o.u2, V0[:, None, None] * one + V[:, None, None] * cx)
    _set_phys(o, o.u3, W[:, None, None] * cx)
    _set_phys(o, o.th[0], T[:, None, None] * one + B[:, None, None] * cx + C[:, None, None] * cz)
    return p, o


def test_stats_modal_known_answers():
    from oracle.stats import save_stats_chan
    p, o = _modal_case()
    s = save_stats_chan(o)
    # the profiles after the wall values were applied, read from the modes
    c1, c2, c3, ct = o.u1.c, o.u2.c, o.u3.c, o.th[0].c
    U, A = c1[:, 0, 0].real, 2 * c1[:, 1, 0].real
    V0, V = c2[:, 0, 0].real, 2 * c2[:, 0, 1].real
    W = 2 * c3[:, 0, 1].real
    T, B, C = ct[:, 0, 0].real, 2 * ct[:, 0, 1].real, 2 * ct[:, 1, 0].real
    gy, gyf, dy, dyf = o.gy, o.gyf, o.dy, o.dyf
    kx, kz = o.kx[1], o.kz[1]
    assert kx == pytest.approx(2 * float(np.float32(np.pi)) / p.lx, rel=1e-15)
    tws = 0.3 * 0.5 / 0.5   # (1/(Ro_inv/delta)) dTHdX(1), Ro_inv = 0.5
    ny = p.ny
    J = np.arange(1, ny + 1)
    pr, th = s["profiles"], s["th"][0]

    def close(name, got, want, rel=1e-11):
        scale = max(np.abs(want).max(), 1e-30)
        err = np.abs(np.asarray(got) - np.asarray(want)).max() / scale
        assert err < rel, (name, err)

    close("ume", pr["ume"], U[J])
    close("vme", pr["vme"], V0[J])
    close("urms", pr["urms"], np.abs(A[J]) / math.sqrt(2))
    close("vrms", pr["vrms"], np.abs(V[J]) / math.sqrt(2))
    close("wrms", pr["wrms"], np.abs(W[J]) / math.sqrt(2))
    assert np.abs(pr["uw"]).max() < 1e-15 and np.abs(pr["uv"]).max() < 1e-15
    G = np.arange(2, ny + 1)
    IW = (dyf[G - 1] * W[G] + dyf[G] * W[G - 1]) / (2 * dy[G])
    close("wv", pr["wv"][1:], IW * V[G] / 2)
    assert pr["wv"][0] == 0.0 and pr["epsilon"][0] == 0.0 and pr["mke"][0] == 0.0
    d = lambda f: (f[J + 1] - f[J - 1]) / (2 * dyf[J])
    close("shear", pr["shear"], d(U) ** 2 + d(A) ** 2 / 2 + d(W) ** 2 / 2)
    close("omega_x", pr["omega_x"], np.sqrt(d(W) ** 2 / 2 + tws ** 2))
    close("omega_y", pr["omega_y"], np.sqrt((kx ** 2 * W[J] ** 2 + kz ** 2 * A[J] ** 2) / 2))
    close("omega_z", pr["omega_z"],
          np.sqrt(d(U) ** 2 + d(A) ** 2 / 2 + kx ** 2 * (0.5 * (V[J + 1] + V[J])) ** 2 / 2))
    eps = (kx ** 2 * V[G] ** 2 / 2
           + ((A[G] - A[G - 1]) / dy[G]) ** 2 / 2
           + kx ** 2 * (dyf[G - 1] * W[G] ** 2 + dyf[G] * W[G - 1] ** 2) / (2 * dy[G]) / 2
           + kz ** 2 * (dyf[G - 1] * A[G] ** 2 + dyf[G] * A[G - 1] ** 2) / (2 * dy[G]) / 2
           + ((V[G + 1] - V[G - 1]) / (gy[G + 1] - gy[G - 1])) ** 2 / 2
           + ((W[G] - W[G - 1]) / dy[G]) ** 2 / 2)
    close("epsilon", pr["epsilon"][1:], eps / p.re)
    wm = lambda g: tws * (gyf[g] - 0.5 * p.ly)
    mke = 0.5 * ((dyf[G - 1] * U[G] ** 2 + dyf[G] * U[G - 1] ** 2) / (2 * dy[G])
                 + (dyf[G - 1] * wm(G) ** 2 + dyf[G] * wm(G - 1) ** 2) / (2 * dy[G]) + V0[G] ** 2)
    close("mke", pr["mke"][1:], mke)
    close("dudy", pr["dudy"], (U[J] - U[J - 1]) / (gyf[J] - gyf[J - 1]))
    close("vv_dvdy", pr["vv_dvdy"][1:], (V0[G + 1] - V0[G - 1]) / (gy[G + 1] - gy[G - 1]) * V[G] ** 2 / 2)
    close("wv_dwdy", pr["wv_dwdy"][1:], tws * IW * V[G] / 2)
    for k in ("uu_dudx", "wu_dwdx", "vu_dvdx", "epsilon_m", "nu_sgs", "eps_sgs2"):
        assert not pr[k].any(), k
    # scalar
    close("thme", th["thme"], T[J])
    close("dthdy", th["dthdy"], (T[J] - T[J - 1]) / (gyf[J] - gyf[J - 1]))
    close("thrms", th["thrms"], np.sqrt((B[J] ** 2 + C[J] ** 2) / 2))
    close("thv", th["thv"], B[J] * 0.5 * (V[J] + V[J + 1]) / 2)
    close("thv_m", th["thv_m"], (T[J] + 0.3 * (-p.lx / (2 * p.nx))) * 0.5 * (V0[J] + V0[J + 1]))
    D = gyf[J + 1] - gyf[J - 1]
    pe = (kx ** 2 * B[J] ** 2 / 2 + 0.3 ** 2
          + ((T[J + 1] - T[J - 1]) / D) ** 2 + ((B[J + 1] - B[J - 1]) / D) ** 2 / 2
          + ((C[J + 1] - C[J - 1]) / D) ** 2 / 2
          + kz ** 2 * C[J] ** 2 / 2 + 0.2 ** 2)
    close("pe_diss", th["pe_diss"], pe)
    # scalars and the kz = 0 spectrum of u1 (its only kz = 0 mode is the mean)
    trap = lambda f: sum(0.5 * (f[j] + f[j - 1]) * dy[j] for j in range(2, ny + 1)) / p.ly
    sc = s["scalars"]
    assert sc["ubulk"] == pytest.approx(trap(U), rel=1e-13)
    assert sc["urms_b"] == pytest.approx(math.sqrt(trap(A ** 2 / 2)), rel=1e-12)
    assert sc["u1y_left_b"] == pytest.approx(trap(gyf * U), rel=1e-12)
    assert s["spectrum"][0] == pytest.approx(trap(U ** 2), rel=1e-12)
    assert np.abs(s["spectrum"][1:]).max() < 1e-20
    assert s["spectrum"].size == p.nx // 2


def test_stats_les_terms_known_answers():
    from oracle.stats import save_stats_chan
    p = small_params(nx=16, ny=25, nz=12, n_th=0, grav_y=0.0)
    gy = grid_for(p)
    o = _oracle(p, gy)
    U = 1.0 - o.gyf ** 2
    _set_phys(o, o.u1, U[:, None, None] * np.ones((1, o.Nz, o.Nx)))
    nu0 = 0.0125
    nu_t = np.zeros((p.ny + 2, p.nz + 2, p.nx + 2))
    nu_t[:, :p.nz, :p.nx] = nu0
    s = save_stats_chan(o, nu_t=nu_t)
    U = o.u1.c[:, 0, 0].real
    dy, dyf = o.dy, o.dyf
    J = np.arange(1, p.ny + 1)
    s1 = np.zeros(p.ny + 2)
    s1[J] = U[J] * nu0 * ((U[J + 1] - U[J]) / dy[J + 1] - (U[J] - U[J - 1]) / dy[J]) / dyf[J]
    G = np.arange(2, p.ny + 1)
    want = 0.5 * (s1[G] + s1[G - 1])
    got = s["profiles"]["eps_sgs2"]
    assert got[0] == 0.0
    assert np.abs(got[1:] - want).max() < 1e-11 * np.abs(want).max()
    assert np.abs(s["profiles"]["nu_sgs"] - nu0).max() < 1e-16


def _parseval(o, tws, nu_t=None):
    """The statistics from the Fourier coefficients, as the CUDA kernel forms
    them: sum over packed modes with weight 1 (kx = 0) or 2, the kx = 0
    column read as its Hermitian part, fluctuations = (0,0) removed."""
    p = o.p
    Nyp, tk, nkx1 = o.Nyp, o.twoNkz, o.Nkx + 1
    nk2 = tk + 1
    gy, gyf, dy, dyf = o.gy, o.gyf, o.dy, o.dyf

    def sym(c):
        a = c[:, :nk2, :nkx1].copy()
        mirror = [0] + [nk2 - q for q in range(1, nk2)]
        a[:, :, 0] = 0.5 * (a[:, :, 0] + np.conj(a[:, mirror, 0]))
        return a
    c1, c2, c3 = sym(o.u1.c), sym(o.u2.c), sym(o.u3.c)
    ct = [sym(t.c) for t in o.th]
    w = np.full(nkx1, 2.0)
    w[0] = 1.0
    W = w[None, :]
    kx = o.kx[:nkx1][None, :]
    kz = o.kz[:nk2][:, None]
    ik = lambda k, a: 1j * k * a

    def hat(a):
        b = a.copy()
        b[0, 0] = 0.0
        return b
    S = lambda a: float(np.sum(W * np.abs(a) ** 2))
    R = lambda a, b: float(np.sum(W * np.real(a * np.conj(b))))
    out = {k: np.zeros(Nyp + 2) for k in ("uu", "vv", "ww", "uw", "uv", "wv", "shear", "ox", "oy",
                                          "oz", "eps")}
    tho = [{k: np.zeros(Nyp + 2) for k in ("tt", "tv", "pe")} for _ in ct]
    for j in range(1, Nyp + 1):
        out["uu"][j], out["vv"][j], out["ww"][j] = S(hat(c1[j])), S(hat(c2[j])), S(hat(c3[j]))
        out["uw"][j] = R(hat(c1[j]), hat(c3[j]))
        d1 = (c1[j + 1] - c1[j - 1]) / (2 * dyf[j])
        d3 = (c3[j + 1] - c3[j - 1]) / (2 * dyf[j])
        out["shear"][j] = S(d1) + S(d3)
        ox = ik(kz, 0.5 * (c2[j + 1] + c2[j])) - d3
        ox[0, 0] -= tws
        out["ox"][j] = S(ox)
        out["oy"][j] = S(ik(kx, c3[j]) - ik(kz, c1[j]))
        out["oz"][j] = S(d1 - ik(kx, 0.5 * (c2[j + 1] + c2[j])))
        if j >= 2:
            i1 = (dyf[j - 1] * hat(c1[j]) + dyf[j] * hat(c1[j - 1])) / (2 * dy[j])
            i3 = (dyf[j - 1] * hat(c3[j]) + dyf[j] * hat(c3[j - 1])) / (2 * dy[j])
            out["uv"][j], out["wv"][j] = R(i1, hat(c2[j])), R(i3, hat(c2[j]))
            k2 = kx ** 2 + kz ** 2
            e = np.sum(W * k2 * (dyf[j - 1] * (np.abs(c1[j]) ** 2 + np.abs(c3[j]) ** 2)
                                 + dyf[j] * (np.abs(c1[j - 1]) ** 2 + np.abs(c3[j - 1]) ** 2))) / (2 * dy[j])
            e += np.sum(W * k2 * np.abs(c2[j]) ** 2)
            e += (S(hat(c1[j]) - hat(c1[j - 1])) + S(hat(c3[j]) - hat(c3[j - 1]))) / dy[j] ** 2
            e += S(hat(c2[j + 1]) - hat(c2[j - 1])) / (gy[j + 1] - gy[j - 1]) ** 2
            out["eps"][j] = e
        for n, c in enumerate(ct):
            tho[n]["tt"][j] = S(hat(c[j]))
            tho[n]["tv"][j] = R(hat(c[j]), hat(0.5 * (c2[j] + c2[j + 1])))
            r1, r3 = ik(kx, c[j]), ik(kz, c[j])
            r1[0, 0] += p.dthdx[n]
            r3[0, 0] += p.dthdz[n]
            r2 = (ct[0][j + 1] - ct[0][j - 1]) / (gyf[j + 1] - gyf[j - 1])
            tho[n]["pe"][j] = S(r1) + S(r2) + S(r3)
    return out, tho


@pytest.mark.parametrize("seed", [3, 11])
def test_stats_physical_sums_match_parseval(seed):
    """The oracle's physical-space plane sums and the Parseval evaluation of
    the CUDA kernel agree to round-off on a random turbulent state with two
    scalars and a thermal-wind shift."""
    from oracle.stats import save_stats_chan, thermal_wind_shear
    p = small_params(nx=24, ny=33, nz=18, n_th=2, ro=4.0, delta=0.8, dthdx=[0.25, -0.1],
                     dthdz=[0.05, 0.0], th_bc_ymin=[0, 1], th_bc_ymin_c1=[0.3, 0.0])
    gy = grid_for(p)
    o = _oracle(p, gy)
    f = initial_fields(p, gy, kind="turbulent", seed=seed)
    for fld, name in ((o.u1, "u1"), (o.u2, "u2"), (o.u3, "u3")):
        _set_phys(o, fld, f[name][:, :p.nz, :p.nx])
    for n in range(p.n_th):
        _set_phys(o, o.th[n], f[f"th{n}"][:, :p.nz, :p.nx])
    s = save_stats_chan(o)
    tws = thermal_wind_shear(p)
    q, qt = _parseval(o, tws)
    J = slice(1, p.ny + 1)
    pr = s["profiles"]

    def close(name, got, want, rel=1e-11):
        scale = max(np.abs(want).max(), 1e-30)
        err = np.abs(np.asarray(got) - np.asarray(want)).max() / scale
        assert err < rel, (name, err)
    close("urms", pr["urms"], np.sqrt(q["uu"][J]))
    close("vrms", pr["vrms"], np.sqrt(q["vv"][J]))
    close("wrms", pr["wrms"], np.sqrt(q["ww"][J]))
    close("uw", pr["uw"], q["uw"][J])
    close("uv", pr["uv"], q["uv"][J])
    close("wv", pr["wv"], q["wv"][J])
    close("shear", pr["shear"], q["shear"][J])
    close("omega_x", pr["omega_x"], np.sqrt(q["ox"][J]))
    close("omega_y", pr["omega_y"], np.sqrt(q["oy"][J]))
    close("omega_z", pr["omega_z"], np.sqrt(q["oz"][J]))
    close("epsilon", pr["epsilon"], q["eps"][J] / p.re)
    for n in range(p.n_th):
        close("thrms", s["th"][n]["thrms"], np.sqrt(qt[n]["tt"][J]))
        close("thv", s["th"][n]["thv"], qt[n]["tv"][J])
        close("pe_diss", s["th"][n]["pe_diss"], qt[n]["pe"][J])


def test_stats_nonhomogeneous_known_answers():
    """Branch of IC types 5-8: the means are z-line averages at each x, so a
    kz = 0 mode is mean flow (no fluctuation), epsilon's x derivatives skip
    the kz = 0 row, and epsilon_m and the production terms use the mean
    gradients of those x-dependent means."""
    from oracle.stats import save_stats_chan
    p = small_params(nx=32, ny=33, nz=24, n_th=0, grav_y=0.0, re=250.0)
    gy = grid_for(p)
    o = _oracle(p, gy)
    y = o.gyf
    x = np.arange(o.Nx) * (2 * np.pi / o.Nx)
    z = np.arange(o.Nz) * (2 * np.pi / o.Nz)
    cx, sx = np.cos(x)[None, None, :], np.sin(x)[None, None, :]
    cz = np.cos(z)[None, :, None]
    one = np.ones((1, o.Nz, o.Nx))
    U, B, A = 1.0 - y ** 2, 0.2 * np.cos(y), 0.1 * np.sin(2.0 * y)
    V, D, E = 0.07 * np.cos(y), 0.05 * y, 0.03 * (1 - y ** 2)
    W = 0.2 * y * (1.0 - y ** 2)
    c = lambda f: f[:, None, None]
    _set_phys(o, o.u1, c(U) * one + c(B) * cx + c(A) * cz)
    _set_phys(o, o.u2, c(V) * cx + cz * (c(D) + c(E) * cx))
    _set_phys(o, o.u3, c(W) * cx)
    s = save_stats_chan(o, homogeneous_x=False)
    c1, c2, c3 = o.u1.c, o.u2.c, o.u3.c
    U, B, A = c1[:, 0, 0].real, 2 * c1[:, 0, 1].real, 2 * c1[:, 1, 0].real
    V, D, E = 2 * c2[:, 0, 1].real, 2 * c2[:, 1, 0].real, 4 * c2[:, 1, 1].real
    W = 2 * c3[:, 0, 1].real
    gy, gyf, dy, dyf = o.gy, o.gyf, o.dy, o.dyf
    kx, kz, nu = o.kx[1], o.kz[1], 1.0 / p.re
    ny = p.ny
    J = np.arange(1, ny + 1)
    G = np.arange(2, ny + 1)
    pr = s["profiles"]

    def close(name, got, want, rel=1e-11):
        scale = max(np.abs(want).max(), 1e-30)
        err = np.abs(np.asarray(got) - np.asarray(want)).max() / scale
        assert err < rel, (name, err)
    close("urms", pr["urms"], np.abs(A[J]) / math.sqrt(2))
    close("vrms", pr["vrms"], np.sqrt((D[J] ** 2 + E[J] ** 2 / 2) / 2))
    assert np.abs(pr["wrms"]).max() < 1e-14
    IA = (dyf[G - 1] * A[G] + dyf[G] * A[G - 1]) / (2 * dy[G])
    close("uv", pr["uv"][1:], IA * D[G] / 2)
    dgy = gy[G + 1] - gy[G - 1]
    eps = (kx ** 2 * E[G] ** 2 / 4                                                   # dv/dx
           + kz ** 2 * (dyf[G - 1] * A[G] ** 2 + dyf[G] * A[G - 1] ** 2) / (2 * dy[G]) / 2   # du/dz
           + kz ** 2 * (D[G] ** 2 + E[G] ** 2 / 2) / 2                              # dv/dz
           + ((A[G] - A[G - 1]) / dy[G]) ** 2 / 2                                    # du/dy
           + (((D[G + 1] - D[G - 1]) / dgy) ** 2 + ((E[G + 1] - E[G - 1]) / dgy) ** 2 / 2) / 2)
    close("epsilon", pr["epsilon"][1:], nu * eps)
    Bm = np.where(J >= 2, B[J - 1], 0.0)
    Wm = np.where(J >= 2, W[J - 1], 0.0)
    epm = (kx ** 2 * (dyf[J - 1] * B[J] ** 2 + dyf[J] * Bm ** 2) / (2 * dy[J]) / 2
           + kx ** 2 * V[J] ** 2 / 2
           + kx ** 2 * (dyf[J - 1] * W[J] ** 2 + dyf[J] * Wm ** 2) / (2 * dy[J]) / 2)
    epm[1:] += (((U[G] - U[G - 1]) / dy[G]) ** 2 + ((B[G] - B[G - 1]) / dy[G]) ** 2 / 2
                + ((V[G + 1] - V[G - 1]) / dgy) ** 2 / 2 + ((W[G] - W[G - 1]) / dy[G]) ** 2 / 2)
    close("epsilon_m", pr["epsilon_m"], nu * epm)
    mke = 0.5 * ((dyf[G - 1] * (U[G] ** 2 + B[G] ** 2 / 2) + dyf[G] * (U[G - 1] ** 2 + B[G - 1] ** 2 / 2))
                 / (2 * dy[G])
                 + (dyf[G - 1] * W[G] ** 2 / 2 + dyf[G] * W[G - 1] ** 2 / 2) / (2 * dy[G])
                 + V[G] ** 2 / 2)
    close("mke", pr["mke"][1:], mke)
    close("vv_dvdy", pr["vv_dvdy"][1:], (V[G + 1] - V[G - 1]) / dgy * D[G] * E[G] / 2)
    for k in ("uu_dudx", "wu_dwdx", "vu_dvdx"):
        assert np.abs(pr[k]).max() < 1e-13 * max(np.abs(pr["vv_dvdy"]).max(), 1e-30), k


def test_bpe_single_bin_known_answer():
    """compute_BPE with th = 0 and no background gradient: every point falls in
    the acos bin of 0, which the reference's float32 pi puts at Nbin/2 - 1
    (acos(0) * Nbin / pi = 0.49999998 Nbin), so Y_r jumps from 0 to Ly there and
    BPE = -Ly/2 times the bin's mid value."""
    from oracle.channel import PI_REF
    from oracle.stats import compute_bpe
    p = small_params(nx=32, ny=25, nz=12, n_th=1, ro=2.0, grav_y=0.0)
    gy = grid_for(p)
    o = _oracle(p, gy)
    th1 = np.zeros((p.ny + 2, p.nz, p.nx))
    bpe, pdf, bins = compute_bpe(o, th1, True)
    b = p.nx // 2 - 1
    assert pdf[b] == pytest.approx(1.0, rel=1e-15) and np.count_nonzero(pdf) == 1
    edge = lambda i: -(0.5 + 1e-14) * math.cos(i * PI_REF / p.nx)
    assert bins[b] == edge(b)
    assert bpe == pytest.approx(-0.5 * p.ly * 0.5 * (edge(b) + edge(b + 1)), rel=1e-14)


def test_bpe_evenly_spaced_bins_sorted_profile():
    """x-inhomogeneous branch: th_1 = 0 and a background gradient dTHdX only, so
    s = dTHdX (x - Lx/2) is spread evenly over x; the PDF is y-weighted and
    uniform across the occupied bins, and BPE follows from the bins directly."""
    from oracle.stats import compute_bpe
    p = small_params(nx=32, ny=25, nz=12, n_th=1, dthdx=[0.4], grav_y=0.0)
    gy = grid_for(p)
    o = _oracle(p, gy)
    th1 = np.zeros((p.ny + 2, p.nz, p.nx))
    bpe, pdf, bins = compute_bpe(o, th1, False)
    assert pdf.sum() == pytest.approx(1.0, rel=1e-14)
    # the Nx positions x_i fall in bins 1.1 Lx/Nx wide: every bin holds a whole
    # number of the (equally y-weighted) x columns, and they appear in x order
    counts = pdf * p.nx
    assert np.allclose(counts, np.round(counts), atol=1e-9)
    d0, x = 0.4, np.arange(p.nx) * p.lx / p.nx
    s = d0 * (x - 0.5 * p.lx)
    thmin = -d0 * 0.5 * p.lx * float(np.float32(1.1))
    dth = (-2 * thmin) / p.nx + 1e-14
    want = np.bincount(np.trunc((s - thmin) / dth).astype(int), minlength=p.nx) / p.nx
    assert np.allclose(pdf, want, atol=1e-12)
    y_r = np.concatenate([[0.0], np.cumsum(want)]) * p.ly
    mids = 0.5 * (np.arange(p.nx + 1)[1:] + np.arange(p.nx)) * dth + thmin
    ref = -np.sum(mids * 0.5 * (y_r[1:] + y_r[:-1]) * np.diff(y_r)) / p.ly
    assert bpe == pytest.approx(ref, rel=1e-12)
    assert bins[0] == thmin


def test_ystar_binning_single_bin_known_answer():
    """Bin_Ystar_and_Write with th_1 = 0 and no background gradient: every
    point lands in one th bin, whose value is the dyf-weighted mean of the field
    over rows jstart_th..jend_th; the other bins are empty (0/0 = NaN, as the
    reference writes them)."""
    from oracle.stats import bin_ystar
    p = small_params(nx=16, ny=25, nz=12, n_th=1, ro=2.0, grav_y=0.0)
    gy = grid_for(p)
    o = _oracle(p, gy)
    th1 = np.zeros((p.ny + 2, p.nz, p.nx))
    U = 1.0 - o.gyf ** 2
    field = np.broadcast_to(0.5 * U[:, None, None] ** 2, (p.ny + 2, p.nz, p.nx))
    fb = bin_ystar(o, th1, field, True)
    b = p.nx // 2 - 1
    J = range(o.jstart_th[0], o.jend_th[0] + 1)
    want = sum(o.dyf[j] * 0.5 * U[j] ** 2 for j in J) / sum(o.dyf[j] for j in J)
    assert fb[b] == pytest.approx(want, rel=1e-13)
    assert np.isnan(np.delete(fb, b)).all()
