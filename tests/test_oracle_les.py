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
