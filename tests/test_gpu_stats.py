"""Parity of the CUDA plane statistics (diablo_stats, the x-homogeneous
save_stats_chan of for/statistics.f90:44-712) with the oracle
(oracle/stats.py), through the C ABI.

The device evaluates the plane averages from the Fourier coefficients
(Parseval) and the z-line averages of the x-inhomogeneous branch from physical
fields; the oracle sums physical grid values as the reference does, so the two
agree to round-off.  Each case steps the GPU channel, loads its state into
the oracle and compares every profile on the same state: max abs error <=
1e-10 x the profile's largest magnitude (1e-12 x for the means and scalars).
At the full 256 x 257 x 256 size the checks are size-independent: the rms
profiles against plane variances of the GPU's own physical download,
determinism, and signs.
"""
import numpy as np
import pytest

from diablo3_test_b200 import _lib, ics
from diablo3_test_b200.config import LES_DYNAMIC_SMAGORINSKY, LES_SMAGORINSKY, MIXED
from tests.helpers import small_params, grid_for, initial_fields, setup_gpu, field_ids

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _oracle_from_gpu(ch, p, gy):
    """An oracle channel holding the GPU context's current Fourier state."""
    from oracle.channel import OracleChannel
    o = OracleChannel(p, gy)
    for name, fid in field_ids(p) + [("p", _lib.P)]:
        buf = ch.download(fid)
        dst = {"u1": o.u1, "u2": o.u2, "u3": o.u3, "p": o.p_}.get(name)
        if dst is None:
            dst = o.th[int(name[2:])]
        dst.buf[:] = buf
    t, _, dt = ch.time
    o.time, o.delta_t = t, dt
    return o


def _compare(sg, so, p):
    for k, a in so["profiles"].items():
        b = sg["profiles"][k]
        scale = max(np.abs(a).max(), 1e-300)
        err = np.abs(b - a).max() / scale
        assert err <= TOL, (k, err)
    for n in range(p.n_th):
        for k, a in so["th"][n].items():
            b = sg["th"][n][k]
            scale = max(np.abs(a).max(), 1e-300)
            err = np.abs(b - a).max() / scale
            assert err <= TOL, (f"th{n}", k, err)
    a, b = so["spectrum"], sg["spectrum"]
    assert np.abs(b - a).max() <= TOL * np.abs(a).max()
    if p.n_th > 0:   # compute_BPE: the same bins, the same y-weighted PDF
        assert np.array_equal(sg["th1_bin"], so["th1_bin"])
        assert np.abs(sg["th1_pdf"] - so["th1_pdf"]).max() <= 1e-12
        for k, a in so["zstar"].items():   # y* bin means; empty bins NaN on both sides
            b = sg["zstar"][k]
            assert np.array_equal(np.isnan(a), np.isnan(b)), k
            ok = ~np.isnan(a)
            if ok.any():
                scale = max(np.abs(a[ok]).max(), 1e-300)
                assert np.abs(b[ok] - a[ok]).max() <= TOL * scale, (k, np.abs(b[ok] - a[ok]).max() / scale)
    for k, a in so["scalars"].items():
        b = sg["scalars"][k]
        assert abs(b - a) <= 1e-12 * max(abs(a), 1e-300) or a == b, (k, a, b)


DNS_CASES = {
    "two_scalars_thermal_wind": dict(n_th=2, ro=4.0, delta=0.8, dthdx=[0.25, -0.1], dthdz=[0.05, 0.0],
                                     th_bc_ymin=[0, 1], th_bc_ymin_c1=[0.3, 0.0], pr=[1.0, 0.71]),
    "neumann_walls_forcing": dict(n_th=1, u_bc_ymax=1, w_bc_ymax=1, u_bc_ymax_c1=0.1, f_type=1,
                                  px0=-0.5),
    "no_scalars": dict(n_th=0, grav_y=0.0),
}


@pytest.mark.parametrize("case", sorted(DNS_CASES))
@pytest.mark.parametrize("precision", [0, MIXED])
def test_stats_match_oracle(cuda_device, case, precision):
    from oracle.stats import save_stats_chan
    p = small_params(nx=32, ny=33, nz=24, precision=precision, **DNS_CASES[case])
    gy = grid_for(p)
    ch = setup_gpu(p, gy, initial_fields(p, gy, kind="turbulent", seed=7))
    try:
        ch.step(3)
        o = _oracle_from_gpu(ch, p, gy)
        sg = ch.stats()
        so = save_stats_chan(o)
        _compare(sg, so, p)
        # the wall values applied by stats are those the oracle applied
        for name, fid in field_ids(p):
            g = ch.download(fid)
            ref = {"u1": o.u1, "u2": o.u2, "u3": o.u3}.get(name) or o.th[int(name[2:])]
            assert np.abs(g - ref.buf).max() <= 1e-15 * max(np.abs(ref.buf).max(), 1.0)
        assert np.abs(sg["profiles"]["urms"]).max() > 0
    finally:
        ch.close()


@pytest.mark.parametrize("model,precision", [(LES_SMAGORINSKY, 0), (LES_DYNAMIC_SMAGORINSKY, 0),
                                             (LES_DYNAMIC_SMAGORINSKY, MIXED)])
def test_stats_les_match_oracle(cuda_device, model, precision):
    from oracle.stats import save_stats_chan
    p = small_params(nx=32, ny=33, nz=24, n_th=1, use_les=True, create_new_flow=False, re=400.0,
                     les_model_type=model, precision=precision)
    gy = grid_for(p)
    ch = setup_gpu(p, gy, initial_fields(p, gy, kind="turbulent", seed=5))
    try:
        ch.step(2)
        nu_t = ch.download_nu_t()
        o = _oracle_from_gpu(ch, p, gy)
        sg = ch.stats()
        # kappa_t = nu_t for the Smagorinsky models (for/les.f90:1130-1146)
        so = save_stats_chan(o, nu_t=nu_t, kappa_t=[nu_t] * p.n_th)
        _compare(sg, so, p)
        assert np.abs(sg["th"][0]["kappa_sgs"]).max() > 0
        assert np.abs(sg["profiles"]["nu_sgs"]).max() > 0
        assert np.abs(sg["profiles"]["eps_sgs2"]).max() > 0
    finally:
        ch.close()


NONHOM_CASES = {
    "front_two_scalars": dict(n_th=2, ro=4.0, delta=0.8, dthdx=[0.25, -0.1], dthdz=[0.05, 0.0],
                              th_bc_ymin=[0, 1], th_bc_ymin_c1=[0.3, 0.0], pr=[1.0, 0.71]),
    "no_scalars": dict(n_th=0, grav_y=0.0),
}


@pytest.mark.parametrize("case", sorted(NONHOM_CASES))
@pytest.mark.parametrize("precision", [0, MIXED])
def test_stats_nonhomogeneous_match_oracle(cuda_device, case, precision):
    """The branch of IC types 5-8 (homogeneousX false): z-line means,
    epsilon_m and the production terms of the mean x gradients."""
    from oracle.stats import save_stats_chan
    p = small_params(nx=32, ny=33, nz=24, precision=precision, **NONHOM_CASES[case])
    gy = grid_for(p)
    ch = setup_gpu(p, gy, initial_fields(p, gy, kind="turbulent", seed=8))
    try:
        ch.step(2)
        o = _oracle_from_gpu(ch, p, gy)
        sg = ch.stats(homogeneous_x=False)
        so = save_stats_chan(o, homogeneous_x=False)
        _compare(sg, so, p)
        for k in ("epsilon_m", "uu_dudx", "wu_dwdx", "vu_dvdx"):
            assert np.abs(sg["profiles"][k]).max() > 0, k
    finally:
        ch.close()


def test_stats_nonhomogeneous_les_matches_oracle(cuda_device):
    from oracle.stats import save_stats_chan
    p = small_params(nx=32, ny=33, nz=24, n_th=1, use_les=True, create_new_flow=False, re=400.0,
                     les_model_type=LES_SMAGORINSKY)
    gy = grid_for(p)
    ch = setup_gpu(p, gy, initial_fields(p, gy, kind="turbulent", seed=6))
    try:
        ch.step(2)
        nu_t = ch.download_nu_t()
        o = _oracle_from_gpu(ch, p, gy)
        sg = ch.stats(homogeneous_x=False)
        so = save_stats_chan(o, nu_t=nu_t, homogeneous_x=False, kappa_t=[nu_t] * p.n_th)
        _compare(sg, so, p)
    finally:
        ch.close()


def test_stats_rejects_short_buffers(cuda_device):
    import ctypes
    p = small_params()
    gy = grid_for(p)
    ch = setup_gpu(p, gy, initial_fields(p, gy))
    try:
        n = ch.lib.diablo_stats_size(ch.ctx)
        assert n == p.ny * (len(_lib.STAT_PROFILES) + p.n_th * len(_lib.STAT_TH_PROFILES)) \
            + p.nx // 2 + ((2 + len(_lib.STAT_ZSTAR)) * p.nx if p.n_th > 0 else 0) \
            + len(_lib.STAT_SCALARS)
        out = np.zeros(n)
        ptr = out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        assert ch.lib.diablo_stats(ch.ctx, 1, ptr, n - 1) == _lib.ERR_ARG
        assert ch.lib.diablo_stats(ch.ctx, 1, None, n) == _lib.ERR_ARG
    finally:
        ch.close()


def test_stats_full_size_properties(cuda_device):
    """256 x 257 x 256, two scalars, mixed precision, after 2 steps: urms,
    vrms and thrms equal the plane standard deviations of the GPU's own
    physical download (a transform path independent of the Parseval sums);
    the means equal the (0,0) coefficients; two calls agree bit for bit;
    squares are non-negative."""
    p, gy = ics.config_c2(precision=MIXED)
    fields = ics.log_law_turbulent(p, gy, seed=2)
    ch = setup_gpu(p, gy, fields)
    try:
        ch.step(2)
        s1 = ch.stats()
        s2 = ch.stats()
        for k in s1["profiles"]:
            assert np.array_equal(s1["profiles"][k], s2["profiles"][k]), k
        pr = s1["profiles"]
        for name, fid, key in (("u1", _lib.U1, "urms"), ("u2", _lib.U2, "vrms")):
            phys = ch.download(fid, _lib.LAYOUT_PHYSICAL)[:, :p.nz, :p.nx]
            four = ch.download(fid).view(np.complex128)
            for j in (1, 2, 40, 128, 200, 256, 257):
                v = phys[j]
                assert abs(v.std() - pr[key][j - 1]) <= 1e-10 * max(pr[key].max(), 1e-30), (name, j)
                mean_key = {"u1": "ume", "u2": "vme"}[name]
                assert pr[mean_key][j - 1] == four[j, 0, 0].real
        th = ch.download(_lib.TH + 1, _lib.LAYOUT_PHYSICAL)[:, :p.nz, :p.nx]
        for j in (3, 100, 255):
            assert abs(th[j].std() - s1["th"][1]["thrms"][j - 1]) <= 1e-10 * s1["th"][1]["thrms"].max()
        for k in ("urms", "vrms", "wrms", "shear", "omega_x", "omega_y", "omega_z", "epsilon"):
            assert np.all(pr[k] >= 0), k
        assert np.all(np.isfinite(np.concatenate(list(pr.values()))))
        assert s1["scalars"]["ubulk"] > 0
    finally:
        ch.close()
