"""Known-answer tests that pin the LES part of the CPU oracle (oracle/les.py).

The reference has no LES tests or fixtures; these check properties the
restated formulas have by construction:
* constant Smagorinsky (for/les.f90:94-270): for a plane shear flow
  u1 = U(y), nu_t(j) = C_s^2 Delta_g(j)^2 |dU/dy| at the GY points, zero on
  the planes ghost_les_mpi clears (:2241-2262), and the whole stress sits in
  the implicit Crank-Nicolson rows, so les_chan leaves cf unchanged;
* dynamic Smagorinsky (Germano/Lilly): the plane-averaged coefficient is
  invariant under scaling of the velocity, and vanishes for a flow without
  x-z variation (the resolved Leonard stress is then zero);
* anisotropic minimum dissipation (for/les.f90:279-850, 1219-1412): no eddy
  viscosity in a plane shear flow (-(I3 - I4) vanishes identically there),
  and nu_t and the type-5 kappa_t are homogeneous of degree one in the
  velocity.
"""
import numpy as np
import pytest

from diablo3_test_b200.config import (LES_SMAGORINSKY, LES_DYNAMIC_SMAGORINSKY, LES_AMD_ROZEMA,
                                      LES_AMD_VERSTAPPEN)
from tests.helpers import small_params, grid_for, initial_fields, setup_oracle


def _oracle(model, **kw):
    from oracle.channel import OracleChannel
    base = dict(nx=32, ny=33, nz=24, use_les=True, create_new_flow=False, les_model_type=model)
    base.update(kw)
    p = small_params(n_th=0, **base)
    return OracleChannel(p, grid_for(p))


def _shear(o, amp=1.0):
    for f in (o.u1, o.u2, o.u3):
        f.c[:] = 0
    y = o.gyf
    o.u1.c[:, 0, 0] = amp * (1.0 - y ** 2) + 0.3 * y ** 3


def test_smagorinsky_plane_shear():
    from oracle import les
    o = _oracle(LES_SMAGORINSKY)
    _shear(o)
    cf0 = [f.c.copy() for f in (o.f1, o.f2, o.f3)]
    u1c = o.u1.c[:, 0, 0].real.copy()
    les.les_chan(o)
    # the wall rows change only through apply_BC_vel_mpi_post; use interior planes
    _, d2g = les._filter_widths(o)
    Nyp = o.Nyp
    for j in range(3, Nyp):
        dudy = abs(u1c[j] - u1c[j - 1]) / o.dy[j]
        expect = les.C_SMAG ** 2 * d2g[j] * dudy
        got = o.nu_t[j, :o.Nz, :o.Nx]
        np.testing.assert_allclose(got, expect, rtol=1e-12, atol=0)
    for j in (0, 1, 2, Nyp, Nyp + 1):
        assert np.all(o.nu_t[j] == 0)
    K, I = slice(0, o.twoNkz + 1), slice(0, o.Nxp)
    for f, c0 in zip((o.f1, o.f2, o.f3), cf0):
        assert np.abs(f.c[:, K, I] - c0[:, K, I]).max() < 1e-12


def test_smagorinsky_viscosity_is_linear_in_velocity():
    from oracle import les
    nts = []
    for amp in (1.0, 3.0):
        p = small_params(nx=32, ny=33, nz=24, n_th=0, use_les=True, create_new_flow=False,
                         les_model_type=LES_SMAGORINSKY)
        gy = grid_for(p)
        f = initial_fields(p, gy, kind="turbulent", seed=11)
        o = setup_oracle(p, gy, {k: amp * v for k, v in f.items()})
        les.les_chan(o)
        nts.append(o.nu_t.copy())
    np.testing.assert_allclose(nts[1], 3.0 * nts[0], rtol=1e-10, atol=1e-14)


def _dynamic_C(amp, seed=12):
    from oracle import les
    p = small_params(nx=32, ny=33, nz=24, n_th=0, use_les=True, create_new_flow=False,
                     les_model_type=LES_DYNAMIC_SMAGORINSKY)
    gy = grid_for(p)
    f = initial_fields(p, gy, kind="turbulent", seed=seed)
    o = setup_oracle(p, gy, {k: amp * v for k, v in f.items()})
    les.apply_bc_les(o)
    F = les._fields(o)
    les.compute_strain(o, F)
    for fl in (o.u1, o.u2, o.u3):
        o.fft_xz_to_physical(fl)
    S = {nm: F[nm].r for nm in ("S1", "S2", "S3", "S4", "S5", "S6")}
    s_f, _ = les._strain_norms(o, S)
    d2f, _ = les._filter_widths(o)
    return les._dynamic_coefficient(o, S, s_f, d2f)


def test_dynamic_coefficient_is_scale_invariant():
    c1 = _dynamic_C(1.0)
    c2 = _dynamic_C(2.5)
    assert np.abs(c1).max() > 0
    np.testing.assert_allclose(c2, c1, rtol=1e-9, atol=1e-14)


def test_dynamic_coefficient_vanishes_without_xz_variation():
    from oracle import les
    o = _oracle(LES_DYNAMIC_SMAGORINSKY)
    _shear(o)
    les.les_chan(o)
    assert np.abs(o.nu_t).max() < 1e-20


@pytest.mark.parametrize("model", [LES_AMD_ROZEMA, LES_AMD_VERSTAPPEN])
def test_amd_no_viscosity_in_plane_shear(model):
    from oracle import les
    o = _oracle(model)
    _shear(o)
    les.les_chan(o)
    assert np.all(o.nu_t == 0)


@pytest.mark.parametrize("model", [LES_AMD_ROZEMA, LES_AMD_VERSTAPPEN])
def test_amd_viscosity_is_linear_in_velocity(model):
    from oracle import les
    out = []
    for amp in (1.0, 2.0):
        p = small_params(nx=32, ny=33, nz=24, n_th=1, use_les=True, create_new_flow=False,
                         les_model_type=model)
        gy = grid_for(p)
        f = initial_fields(p, gy, kind="turbulent", seed=13)
        o = setup_oracle(p, gy, {k: amp * v for k, v in f.items()})
        les.les_chan(o)
        les.les_chan_th(o)
        out.append((o.nu_t.copy(), o.kappa_t[0].copy()))
    assert np.abs(out[0][0]).max() > 0 and np.abs(out[0][1]).max() > 0
    np.testing.assert_allclose(out[1][0], 2.0 * out[0][0], rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(out[1][1], 2.0 * out[0][1], rtol=1e-9, atol=1e-14)


def _parseval_mean(o, a, b):
    """Plane means of the product of two band-limited fields from their packed
    Fourier coefficients: weight 1 on the kx = 0 column, 2 elsewhere."""
    K, I = slice(0, o.twoNkz + 1), slice(0, o.Nxp)
    w = np.full(o.Nxp, 2.0)
    w[0] = 1.0
    return np.sum(w * np.real(a[:, K, I] * np.conj(b[:, K, I])), axis=(1, 2))


def test_eps_sgs1_physical_loops_equal_parseval_sums():
    """eps_sgs1 (for/les.f90:940-1068) as the reference forms it (forces to
    physical space, point products, plane sums) against the Parseval sums over
    the retained modes that the CUDA kernel evaluates: one and the same number
    for band-limited fields.  Random Hermitian-consistent stresses from real
    fields, random velocities and nu_t."""
    from oracle.channel import Field
    from oracle.les import eps_sgs1
    o = _oracle(LES_SMAGORINSKY)
    rng = np.random.default_rng(3)
    Nx, Nz, Ny = o.Nx, o.Nz, o.Ny

    def real_field():
        f = Field(Ny, Nz, Nx)
        f.r[:, :Nz, :Nx] = rng.standard_normal((Ny + 2, Nz, Nx))
        o.fft_xz_to_fourier(f)          # band-limited from here on
        return f

    C = [real_field() for _ in range(5)]
    U = [real_field() for _ in range(3)]
    uc = [u.c.copy() for u in U]
    for u in U:
        o.fft_xz_to_physical(u)
    o.u1, o.u2, o.u3 = U
    nt = np.zeros((Ny + 2, Nz + 2, Nx + 2))
    nt[2:Ny, :Nz, :Nx] = rng.random((Ny - 2, Nz, Nx))
    C1, C3, C4, C5, C6 = (c.c for c in C)
    got = eps_sgs1(o, C1, C3, C4, C5, C6, nt)

    K, I = slice(0, o.twoNkz + 1), slice(0, o.Nxp)
    ikx, ikz = 1j * o.kx[None, None, :o.Nxp], 1j * o.kz[None, :o.twoNkz + 1, None]
    R, RP = slice(1, Ny + 1), slice(2, Ny + 2)
    F1 = np.zeros_like(C1); F3 = np.zeros_like(C1); F2 = np.zeros_like(C1)
    dyf = o.dyf[R, None, None]
    F1[R, K, I] = -ikx * C1[R, K, I] - (C4[RP, K, I] - C4[R, K, I]) / dyf - ikz * C5[R, K, I]
    F3[R, K, I] = -ikx * C5[R, K, I] - (C6[RP, K, I] - C6[R, K, I]) / dyf - ikz * C3[R, K, I]
    t1, t3 = Field(Ny, Nz, Nx), Field(Ny, Nz, Nx)
    u1p, u3p = U[0].r[:, :Nz, :Nx], U[2].r[:, :Nz, :Nx]
    t1.r[2:Ny + 1, :Nz, :Nx] = nt[2:Ny + 1, :Nz, :Nx] * (u1p[2:Ny + 1] - u1p[1:Ny]) / o.dy[2:Ny + 1, None, None]
    t3.r[2:Ny + 1, :Nz, :Nx] = nt[2:Ny + 1, :Nz, :Nx] * (u3p[2:Ny + 1] - u3p[1:Ny]) / o.dy[2:Ny + 1, None, None]
    o.fft_xz_to_fourier(t1)
    o.fft_xz_to_fourier(t3)
    J2 = slice(2, Ny + 1)
    F2[J2, K, I] = (-ikx * C4[J2, K, I] - ikz * C6[J2, K, I] + ikx * t1.c[J2, K, I] + ikz * t3.c[J2, K, I])
    p1, p3, p2 = _parseval_mean(o, uc[0], F1), _parseval_mean(o, uc[2], F3), _parseval_mean(o, uc[1], F2)
    ref = np.zeros(Ny + 2)
    for j in range(2, Ny + 1):
        ref[j] = 0.5 * (p1[j] + p1[j - 1]) + 0.5 * (p3[j] + p3[j - 1]) + p2[j]
    assert got[0] == 0.0
    assert np.abs(got - ref[1:Ny + 1]).max() <= 1e-12 * np.abs(ref).max()
