"""Parity of the CUDA channel step with the CPU oracle, through the C ABI.

Tolerance (FP64 path): relative L2 error <= 1e-10 per field over the
significant Fourier entries after a few steps; the xz transforms <= 1e-13.
"""
import numpy as np
import pytest

from diablo3_test_b200 import _lib
from tests.helpers import (small_params, grid_for, initial_fields, setup_oracle, setup_gpu,
                           oracle_state, gpu_state, rel_err, sig)

pytestmark = pytest.mark.gpu

TOL_STEP = 1e-10
TOL_FFT = 1e-13


def _oracle_fft(p, gy):
    from oracle.channel import OracleChannel
    return OracleChannel(p, gy)


@pytest.mark.parametrize("nx,ny,nz", [(32, 33, 24), (64, 65, 64), (48, 17, 16), (256, 9, 256)])
def test_fft_xz_pair_matches_oracle(cuda_device, nx, ny, nz):
    from diablo3_test_b200.channel import Channel
    p = small_params(nx=nx, ny=ny, nz=nz, n_th=0)
    gy = grid_for(p)
    rng = np.random.default_rng(7)
    v = rng.standard_normal((ny + 2, nz + 2, nx + 2))
    o = _oracle_fft(p, gy)
    o.u1.buf[:] = v
    o.fft_xz_to_fourier(o.u1)
    with Channel(p, gy) as ch:
        vv = np.zeros_like(v)
        ch.fft_xz_to_fourier(v.copy(), vv)
        assert rel_err(sig(p, vv), sig(p, o.u1.buf)) < TOL_FFT
        # in place (v == vv), as the reference calls it
        w = v.copy()
        ch.fft_xz_to_fourier(w, w)
        assert rel_err(sig(p, w), sig(p, o.u1.buf)) < TOL_FFT
        # back to physical space: the dealiased projection of v
        back = np.zeros_like(v)
        ch.fft_xz_to_physical(w.copy(), back)
        o.fft_xz_to_physical(o.u1)
        ref = o.u1.buf[:, :nz, :nx]
        assert rel_err(back[:, :nz, :nx], ref) < TOL_FFT
        # modes above Nkx are written as zero; entries outside the significant
        # box are left as they were
        c = w.view(np.complex128)
        c0 = v.view(np.complex128)
        nk2 = 2 * (nz // 3) + 1
        assert np.all(c[:, :nk2, nx // 3 + 1:nx // 2] == 0)
        assert np.array_equal(c[:, nk2:, :], c0[:, nk2:, :]) and np.array_equal(c[:, :, nx // 2], c0[:, :, nx // 2])
        assert np.all(back[:, :, nx:] == 0) and np.all(back[:, nz:, :] == 0)


def test_upload_rejects_modes_above_nkx(cuda_device):
    from diablo3_test_b200.channel import Channel
    p = small_params(n_th=0)
    gy = grid_for(p)
    with Channel(p, gy) as ch:
        buf = ch.new_field()
        c = buf.view(np.complex128)
        c[3, 1, p.nx // 3 + 1] = 1.0
        with pytest.raises(_lib.DiabloError) as e:
            ch.upload(_lib.U1, buf)
        assert e.value.status == _lib.ERR_STATE


def test_upload_download_roundtrip_bit_exact(cuda_device):
    from diablo3_test_b200.channel import Channel
    p = small_params(n_th=1)
    gy = grid_for(p)
    rng = np.random.default_rng(3)
    buf = np.zeros((p.ny + 2, p.nz + 2, p.nx + 2))
    c = buf.view(np.complex128)
    s = (slice(None), slice(0, 2 * (p.nz // 3) + 1), slice(0, p.nx // 3 + 1))
    c[s] = rng.standard_normal(c[s].shape) + 1j * rng.standard_normal(c[s].shape)
    with Channel(p, gy) as ch:
        for fid in (_lib.U1, _lib.U2, _lib.U3, _lib.P, _lib.TH):
            ch.upload(fid, buf)
            out = ch.download(fid)
            assert np.array_equal(out, buf)


CASES = {
    "dirichlet_scalar_neumann": dict(),
    "neumann_top_u_w": dict(u_bc_ymax=1, w_bc_ymax=1, u_bc_ymax_c1=0.1),
    "pressure_gradient_rotation": dict(f_type=1, px0=-0.5, ro=5.0, grav_x=0.1, grav_z=-0.2),
    "two_scalars_dirichlet": dict(n_th=2, pr=[0.71, 1.0], th_bc_ymin=[0, 1], th_bc_ymax=[0, 1],
                                  th_bc_ymin_c1=[-1.0, 0.0], th_bc_ymax_c1=[1.0, 0.0]),
    "hyperviscosity_background_gradient": dict(beta=2.0, dthdx=[0.3], dthdz=[-0.1], nu_v_scale=0.5),
    "moving_walls": dict(u_bc_ymin_c1=-0.3, u_bc_ymax_c1=0.4, w_bc_ymin_c1=0.2),
    "front_thermal_wind": dict(flavor="Front", ro=2.0, delta=1.5, dthdx=[0.2], dthdz=[0.05], grav_y=1.0),
    "oscillating_pressure_gradient": dict(f_type=2, px0=-0.2, amp_omega0=0.3, omega0=40.0),
    "filtered_scalars": dict(n_th=2, pr=[0.71, 1.0], filter_th=[True, False], filter_int=[2, 1],
                             th_bc_ymin=[0, 1], th_bc_ymax=[0, 1], th_bc_ymin_c1=[-1.0, 0.0],
                             th_bc_ymax_c1=[1.0, 0.0]),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_step_matches_oracle(cuda_device, case):
    kw = dict(CASES[case])
    n_th = kw.pop("n_th", 1)
    p = small_params(n_th=n_th, **kw)
    gy = grid_for(p)
    fields = initial_fields(p, gy)
    o = setup_oracle(p, gy, fields)
    ch = setup_gpu(p, gy, fields)
    try:
        # after pre_first_step
        so, sg = oracle_state(o), gpu_state(ch)
        for k in so:
            assert rel_err(sg[k], so[k]) < TOL_STEP, (case, "pre", k)
        # one substep, then complete steps
        o.time_step += 1
        o.rk_step = 1
        o.rk_chan_1()
        ch.rk_chan_1(1)
        so, sg = oracle_state(o), gpu_state(ch)
        for k in so:
            assert rel_err(sg[k], so[k]) < TOL_STEP, (case, "rk1", k, rel_err(sg[k], so[k]))
        for rk in (2, 3):
            o.rk_step = rk
            o.rk_chan_1()
            ch.rk_chan_1(rk)
        o.time += o.delta_t
        ch.set_time(o.time, o.time_step, p.delta_t)
        o.step(3)
        ch.step(3)
        so, sg = oracle_state(o), gpu_state(ch)
        for k in so:
            assert rel_err(sg[k], so[k]) < TOL_STEP, (case, "4 steps", k, rel_err(sg[k], so[k]))
        assert ch.check_finite()
    finally:
        ch.close()


def test_mixed_precision_close_to_fp64(cuda_device):
    from diablo3_test_b200.channel import Channel
    from diablo3_test_b200.config import MIXED
    p = small_params(nx=64, ny=65, nz=64, n_th=1, re=500.0, delta_t=1e-3)
    gy = grid_for(p)
    fields = initial_fields(p, gy, kind="turbulent", seed=4)
    a = setup_gpu(p, gy, fields)
    b = setup_gpu(p, gy, fields)
    try:
        b.set_precision(MIXED)
        a.step(10)
        b.step(10)
        sa, sb = gpu_state(a), gpu_state(b)
        for k in ("u1", "u2", "u3"):
            assert rel_err(sb[k], sa[k]) < 1e-6, (k, rel_err(sb[k], sa[k]))
    finally:
        a.close()
        b.close()


def test_mixed_precision_100_steps_within_1e6(cuda_device):
    # the workload's accuracy bar: <= 1e-6 relative velocity error over 100
    # steps (turbulent log-law state, 96 x 97 x 64, pressure-gradient forcing)
    from diablo3_test_b200.config import MIXED
    p = small_params(nx=96, ny=97, nz=64, n_th=2, re=180.0, delta_t=5e-4, f_type=1, px0=-1.0,
                     grav_y=0.0, pr=[0.71, 1.0])
    gy = grid_for(p, cs=2.0)
    fields = initial_fields(p, gy, kind="turbulent", seed=8)
    a = setup_gpu(p, gy, fields)
    b = setup_gpu(p, gy, fields)
    try:
        b.set_precision(MIXED)
        a.step(100)
        b.step(100)
        sa, sb = gpu_state(a), gpu_state(b)
        for k in ("u1", "u2", "u3", "th0", "th1"):
            assert rel_err(sb[k], sa[k]) < 1e-6, (k, rel_err(sb[k], sa[k]))
    finally:
        a.close()
        b.close()
