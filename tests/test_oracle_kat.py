"""Analytic known-answer tests that pin the CPU oracle (the reference ships
no tests or fixtures to pin it against).

Each test checks one property the reference's algorithm has by construction:
FFT normalisation/packing (for/fft.f90:247-382), dealiasing, the projection
(for/channel.f90:946-1023), the Thomas recurrence (:1335-1540), a laminar
steady state, and the amplification of a Stokes mode under RK3/CN
(for/flow.f90:78-86 with for/channel.f90:29-877)."""
import math

import numpy as np
import pytest

from tests.helpers import small_params, grid_for
from oracle.channel import OracleChannel, PI_REF, BETA_BAR, ZETA_BAR, H_FRAC


def _oracle(**kw):
    p = small_params(**kw)
    return p, OracleChannel(p, grid_for(p))


def test_pi_is_the_single_precision_value():
    assert PI_REF == float(np.float32(math.pi))
    assert abs(PI_REF - math.pi) / math.pi == pytest.approx(2.78e-8, rel=1e-2)


def test_single_mode_and_packing():
    p, o = _oracle(nx=32, ny=9, nz=24, n_th=0)
    x = np.arange(p.nx) * p.lx / p.nx
    z = np.arange(p.nz) * p.lz / p.nz
    X, Z = np.meshgrid(x, z)             # [k, i]
    ax, az = 3, 5                        # kx index 3, kz index +5 and -5
    f = o.u1
    f.r[:, :p.nz, :p.nx] = np.cos(2 * np.pi * (ax * X / p.lx + az * Z / p.lz))[None]
    o.fft_xz_to_fourier(f)
    c = f.c[:, :2 * o.Nkz + 1, :o.Nxp]
    expect = np.zeros_like(c)
    expect[:, az, ax] = 0.5              # e^{+i(ax x + az z)} lands at (kx=3, kz=+5)
    np.testing.assert_allclose(c, expect, atol=1e-14)
    # the reference's z packing: kz = -k is stored at index 2Nkz+1-k
    assert o.kz[2 * o.Nkz + 1 - az] == pytest.approx(-o.kz[az])


def test_round_trip_and_dealiasing():
    p, o = _oracle(nx=48, ny=9, nz=32, n_th=0)
    rng = np.random.default_rng(0)
    f = o.u1
    f.r[:, :p.nz, :p.nx] = rng.standard_normal((p.ny + 2, p.nz, p.nx))
    o.fft_xz_to_fourier(f)
    c0 = f.c[:, :2 * o.Nkz + 1, :o.Nxp].copy()
    # modes above Nkx are zeroed (for/fft.f90:264-266)
    assert np.all(c0[:, :, o.Nkx + 1:] == 0)
    o.fft_xz_to_physical(f)
    # the physical field is now band-limited: transforming back is the identity
    o.fft_xz_to_fourier(f)
    c1 = f.c[:, :2 * o.Nkz + 1, :o.Nxp]
    np.testing.assert_allclose(c1, c0, rtol=0, atol=1e-14 * np.abs(c0).max())
    # and its spectrum has nothing in the dealiased band
    f2 = o.u2
    f2.c[:] = 0
    f2.c[:, :2 * o.Nkz + 1, :o.Nxp] = c0
    o.fft_xz_to_physical(f2)
    full = np.fft.rfft2(f2.r[:, :p.nz, :p.nx], axes=(1, 2))
    kz_idx = np.abs(np.fft.fftfreq(p.nz, 1.0 / p.nz))
    band = kz_idx > o.Nkz
    assert np.abs(full[:, band, :]).max() < 1e-12 * np.abs(full).max()
    assert np.abs(full[:, :, o.Nkx + 1:]).max() < 1e-12 * np.abs(full).max()


def test_spectral_derivative_uses_reference_wavenumbers():
    p, o = _oracle(nx=32, ny=9, nz=16, n_th=0)
    x = np.arange(p.nx) * p.lx / p.nx
    f = o.u1
    f.r[:, :p.nz, :p.nx] = np.sin(2 * np.pi * 2 * x / p.lx)[None, None, :]
    o.fft_xz_to_fourier(f)
    f.c[:, :2 * o.Nkz + 1, :o.Nxp] *= o.cikx[None, None, :o.Nxp]
    o.fft_xz_to_physical(f)
    k = 2 * (2.0 * PI_REF) / p.lx
    expect = np.broadcast_to(k * np.cos(2 * np.pi * 2 * x / p.lx), f.r[:, :p.nz, :p.nx].shape)
    np.testing.assert_allclose(f.r[:, :p.nz, :p.nx], expect, rtol=0, atol=1e-13)


def test_projection_removes_the_divergence():
    p, o = _oracle(nx=32, ny=33, nz=24, n_th=0)
    rng = np.random.default_rng(1)
    for f in (o.u1, o.u2, o.u3):
        f.r[:, :p.nz, :p.nx] = rng.standard_normal((p.ny + 2, p.nz, p.nx))
        o.fft_xz_to_fourier(f)
    o.rem_div_chan()
    K, I = slice(0, o.twoNkz + 1), slice(0, o.Nxp)
    cu1, cu2, cu3 = o.u1.c, o.u2.c, o.u3.c
    worst = 0.0
    # rows 2..Nyp-1 are the interior rows of the pressure equation; rows 1
    # and Nyp carry its wall conditions (for/channel.f90:1974-2015)
    for j in range(2, o.Nyp):
        d = (o.cikx[None, :o.Nxp] * cu1[j, K, I] + (cu2[j + 1, K, I] - cu2[j, K, I]) / o.dyf[j]
             + o.cikz[:, None] * cu3[j, K, I])
        worst = max(worst, np.abs(d).max())
    assert worst < 1e-12


def test_thomas_residual():
    rng = np.random.default_rng(2)
    n, cols = 40, 7
    a = rng.uniform(-1, 0, (n, cols)); c = rng.uniform(-1, 0, (n, cols))
    b = 2.5 + rng.uniform(0, 1, (n, cols))
    a[0] = 0; c[-1] = 0
    g = rng.standard_normal((n, cols))
    A, B, C, G = a.copy(), b.copy(), c.copy(), g.copy()
    OracleChannel.thomas_real(A, B, C, G, n - 2)
    res = b * G + np.vstack([np.zeros((1, cols)), a[1:] * G[:-1]]) + np.vstack([c[:-1] * G[1:], np.zeros((1, cols))]) - g
    assert np.abs(res).max() < 1e-13


def _laplacian_rows(o, lo, hi):
    """Dense form of the reference's y stencil for u1/u3 on rows lo..hi."""
    dy, dyf = o.dy, o.dyf
    n = hi - lo + 1
    L = np.zeros((n, n))
    for r, j in enumerate(range(lo, hi + 1)):
        wp = 1.0 / (dy[j + 1] * dyf[j])
        wm = 1.0 / (dy[j] * dyf[j])
        L[r, r] = -(wp + wm)
        if r > 0:
            L[r, r - 1] = wm
        if r < n - 1:
            L[r, r + 1] = wp
    return L


def test_laminar_poiseuille_is_steady():
    # discrete steady state of nu*L(U) = px0 with U = 0 on the wall rows
    p, o = _oracle(nx=16, ny=33, nz=12, n_th=0, f_type=1, px0=-0.3, re=50.0, delta_t=5e-3, grav_y=0.0)
    lo, hi = 2, o.Nyp - 1
    L = _laplacian_rows(o, lo, hi)
    U = np.linalg.solve(o.nu * p.nu_v_scale * L, np.full(hi - lo + 1, p.px0))
    for f in (o.u1, o.u2, o.u3):
        f.c[:] = 0
    o.u1.c[lo:hi + 1, 0, 0] = U
    o.step(5)
    got = o.u1.c[lo:hi + 1, 0, 0].real
    assert np.abs(got - U).max() < 1e-11 * np.abs(U).max()
    rest = o.u1.c[:, :o.twoNkz + 1, :o.Nxp].copy()
    rest[:, 0, 0] = 0
    assert np.abs(rest).max() < 1e-14


def test_stokes_mode_amplification():
    # u3 = v(y) exp(i kx x): divergence-free, no pressure, no nonlinear term;
    # v an eigenvector of the discrete y operator, so every RK substep scales it
    p, o = _oracle(nx=16, ny=33, nz=12, n_th=0, re=20.0, delta_t=4e-3, grav_y=0.0)
    lo, hi = 2, o.Nyp - 1
    L = _laplacian_rows(o, lo, hi)
    lam, vec = np.linalg.eig(L)
    i0 = np.argmax(lam.real)                   # the smoothest decaying mode
    lam0, v = lam[i0].real, vec[:, i0].real
    kxi = 1
    for f in (o.u1, o.u2, o.u3):
        f.c[:] = 0
    o.u3.c[lo:hi + 1, 0, kxi] = 1e-3 * v
    nsteps = 4
    o.step(nsteps)
    # scalar recursion of the scheme for this mode
    a = -o.nu * o.kx2[kxi] ** p.beta
    lv = p.nu_v_scale * lam0
    u, cf_prev = 1.0, 0.0
    for _ in range(nsteps):
        for rk in range(3):
            h = H_FRAC[rk] * p.delta_t
            cf = a * u
            rhs = u + ZETA_BAR[rk] * h * cf_prev + BETA_BAR[rk] * h * cf + 0.5 * o.nu * h * lv * u
            u = rhs / (1.0 - 0.5 * o.nu * h * lv)
            cf_prev = cf
    got = o.u3.c[lo:hi + 1, 0, kxi]
    np.testing.assert_allclose(got.real, u * 1e-3 * v, rtol=0, atol=1e-13)
    assert np.abs(got.imag).max() < 1e-16
    assert 0 < u < 1  # it decays


def test_scalar_filter_transfer_function():
    # filter_chan (for/channel.f90:1241-1329): sigma = 1 on the mean mode, a
    # smooth roll-off in |k| down to near zero at the largest stored modes
    p, o = _oracle(nx=32, ny=9, nz=24, n_th=1)
    c = o.th[0].c
    c[:] = 1.0 + 1.0j
    o.filter_chan(0)
    J = slice(o.jstart_th[0], o.jend_th[0] + 1)
    f = c[J, :o.twoNkz + 1, :o.Nxp]
    assert np.all(f[:, 0, 0] == 1.0 + 1.0j)
    assert np.all(np.abs(f) <= np.sqrt(2.0) + 1e-15)
    assert np.abs(f[:, o.Nkz, o.Nkx]).max() < 0.5
    # rows outside jstart_th..jend_th are untouched
    assert np.all(c[:o.jstart_th[0]] == 1.0 + 1.0j)
