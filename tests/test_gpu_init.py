"""poisson_p_chan (initial pressure, for/channel.f90:1026-1234) and courant
(variable time step, for/advance.f90:47-158) on the device against the
oracle, through the C ABI: every field <= 1e-10 relative, delta_t and time to
1e-12."""
import numpy as np
import pytest

from diablo3_test_b200.config import LES_SMAGORINSKY, MIXED
from tests.helpers import (small_params, grid_for, initial_fields, oracle_state, gpu_state, rel_err,
                           field_ids)
from diablo3_test_b200 import _lib

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _pair(p, gy, fields, compute_pressure):
    from oracle.channel import OracleChannel
    from diablo3_test_b200.channel import Channel
    o = OracleChannel(p, gy)
    o.u1.r[:] = fields["u1"]
    o.u2.r[:] = fields["u2"]
    o.u3.r[:] = fields["u3"]
    for n in range(p.n_th):
        o.th[n].r[:] = fields[f"th{n}"]
    for f in [o.u1, o.u2, o.u3] + o.th:
        o.fft_xz_to_fourier(f)
    o.pre_first_step(compute_pressure=compute_pressure)
    ch = Channel(p, gy)
    for name, fid in field_ids(p):
        ch.upload(fid, np.ascontiguousarray(fields[name]), _lib.LAYOUT_PHYSICAL)
    ch.pre_first_step(compute_pressure=compute_pressure)
    return o, ch


def _check(o, ch, what):
    so, sg = oracle_state(o), gpu_state(ch)
    for k in so:
        e = rel_err(sg[k], so[k])
        assert e < TOL, (what, k, e)


@pytest.mark.parametrize("kw", [dict(), dict(n_th=1, ri=[0.7], th_bc_ymin=[0], th_bc_ymax=[0],
                                             th_bc_ymin_c1=[-1.0], th_bc_ymax_c1=[1.0]),
                                dict(u_bc_ymax=1, w_bc_ymax=1)])
def test_initial_pressure_matches_oracle(cuda_device, kw):
    kw = dict(kw)
    n_th = kw.pop("n_th", 0)
    p = small_params(n_th=n_th, **kw)
    gy = grid_for(p)
    fields = initial_fields(p, gy, kind="turbulent", seed=21)
    o, ch = _pair(p, gy, fields, True)
    try:
        so, sg = oracle_state(o), gpu_state(ch)
        assert np.abs(so["p"]).max() > 0
        _check(o, ch, "pre_first_step with pressure")
        o.step(2)
        ch.step(2)
        _check(o, ch, "2 steps")
    finally:
        ch.close()


@pytest.mark.parametrize("case", ["dns", "dns_every_2", "les", "rotation_scalar", "front"])
def test_variable_dt_matches_oracle(cuda_device, case):
    kw = dict(variable_dt=True, update_dt=1, cfl=0.5, max_dt=0.02, delta_t=1e-3, re=300.0)
    n_th = 1
    if case == "dns_every_2":
        kw["update_dt"] = 2
    elif case == "les":
        kw.update(use_les=True, create_new_flow=False, les_model_type=LES_SMAGORINSKY)
    elif case == "rotation_scalar":
        kw.update(ro=2.0, th_bc_ymin=[0], th_bc_ymin_c1=[-0.5], th_bc_ymax=[0], th_bc_ymax_c1=[0.5])
    elif case == "front":
        # the 'Front' branch of courant: thermal-wind shifts of u1 and u3
        kw.update(flavor="Front", ro=2.0, delta=1.5, dthdx=[0.2], dthdz=[0.05], grav_y=1.0)
    p = small_params(n_th=n_th, **kw)
    gy = grid_for(p)
    fields = initial_fields(p, gy, kind="turbulent", seed=22)
    o, ch = _pair(p, gy, fields, False)
    try:
        t, n, dt = ch.time
        assert abs(dt - o.delta_t) <= 1e-12 * o.delta_t and dt != 1e-3
        for _ in range(3):
            o.step(1)
            ch.step(1)
            t, n, dt = ch.time
            assert abs(dt - o.delta_t) <= 1e-12 * o.delta_t, (dt, o.delta_t)
            assert abs(t - o.time) <= 1e-12 * abs(o.time)
        _check(o, ch, "3 variable steps")
    finally:
        ch.close()


def test_variable_dt_mixed_runs(cuda_device):
    from diablo3_test_b200.channel import Channel
    p = small_params(n_th=1, variable_dt=True, update_dt=1, cfl=0.5, max_dt=0.02)
    gy = grid_for(p)
    fields = initial_fields(p, gy, kind="turbulent", seed=23)
    ch = Channel(p, gy)
    try:
        ch.set_precision(MIXED)
        for name, fid in field_ids(p):
            ch.upload(fid, np.ascontiguousarray(fields[name]), _lib.LAYOUT_PHYSICAL)
        ch.pre_first_step()
        dt0 = ch.time[2]
        ch.step(3)
        assert ch.check_finite()
        assert ch.time[2] != 0 and dt0 > 0
    finally:
        ch.close()
