"""Parity of the CUDA channel step with the CPU oracle at the wall-normal
sizes and transform lengths the benchmark workloads run, through the C ABI.

The column kernels are instantiated per R = ceil((Ny + 2) / 32), the rows a
lane owns in the warp partition solver; the transforms per length.  Every
instantiation a workload reaches is checked here against the oracle's
restatement of the implicit solves (for/channel.f90:657-877), Thomas
(:1335-1540) and rem_div_chan (:946-1023):

- R = 4 .. 9 on a small xz grid (Ny = 97, 129, 161, 193, 225, 257), with one
  and two scalars;
- the 64 x 193 x 32 plain-DNS workload itself (Re 1000, Pr 1, dt 1e-3) for
  20 steps;
- a 256 x 33 x 256 slice of the Re_tau = 180 workload (two scalars), so the
  256-point transforms run inside a full substep;
- a 96-point x transform (radix 3) inside a step;
- the LES physical-space solve at Ny = 129 (constant and dynamic
  Smagorinsky).

Tolerance: relative L2 error <= 1e-10 per field over the significant
Fourier entries, after pre_first_step, after one substep and after the
further steps; nu_t too for LES.  The pressure is the one field measured
against a running scale: each substep sets p <- p + phi/h
(for/channel.f90:905-911), and in a nearly laminar state the increments can
be several hundred times the result (64 x 193 x 32: |p| = 8.3 after the
first substep, 0.02 after the second), so the round-off of the increments,
not of the result, sets p's error.  p is therefore compared relative to the
largest norm it has had in the run.
"""
import numpy as np
import pytest

from diablo3_test_b200 import _lib, ics
from diablo3_test_b200.config import LES_SMAGORINSKY, LES_DYNAMIC_SMAGORINSKY
from tests.helpers import (small_params, grid_for, initial_fields, setup_oracle, setup_gpu,
                           oracle_state, gpu_state, rel_err)

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _check(o, ch, what, les=False, pscale=None):
    so, sg = oracle_state(o), gpu_state(ch)
    for k in so:
        if k == "p" and pscale is not None:
            pscale[0] = max(pscale[0], float(np.linalg.norm(so[k])))
            e = float(np.linalg.norm(sg[k] - so[k])) / max(pscale[0], 1e-300)
        else:
            e = rel_err(sg[k], so[k])
        assert e < TOL, (what, k, e)
    if les:
        p = o.p
        e = rel_err(ch.download_nu_t()[:, :p.nz, :p.nx], o.nu_t[:, :p.nz, :p.nx])
        assert e < TOL, (what, "nu_t", e)


def _run(p, gy, fields, steps, les=False):
    """pre_first_step, one RK substep, the rest of that step, then `steps`
    more steps, comparing every field after each stage."""
    o = setup_oracle(p, gy, fields)
    ch = setup_gpu(p, gy, fields)
    ps = [0.0]
    try:
        if not les:
            _check(o, ch, "pre_first_step", pscale=ps)
        o.time_step += 1
        o.rk_step = 1
        o.rk_chan_1()
        ch.set_time(o.time, o.time_step, p.delta_t)
        ch.rk_chan_1(1)
        _check(o, ch, "rk1", les, ps)
        for rk in (2, 3):
            o.rk_step = rk
            o.rk_chan_1()
            ch.rk_chan_1(rk)
        o.time += o.delta_t
        ch.set_time(o.time, o.time_step, p.delta_t)
        _check(o, ch, "1 step", les, ps)
        if steps:
            o.step(steps)
            ch.step(steps)
            _check(o, ch, f"{steps + 1} steps", les, ps)
        assert ch.check_finite()
    finally:
        ch.close()


@pytest.mark.parametrize("ny", [97, 129, 161, 193, 225, 257])
@pytest.mark.parametrize("n_th", [1, 2])
def test_column_kernel_rows_per_lane(cuda_device, ny, n_th):
    kw = {}
    if n_th == 2:
        kw = dict(pr=[0.71, 1.0], th_bc_ymin=[0, 1], th_bc_ymax=[0, 1], th_bc_ymin_c1=[-1.0, 0.0],
                  th_bc_ymax_c1=[1.0, 0.0])
    p = small_params(nx=32, ny=ny, nz=24, n_th=n_th, re=400.0, delta_t=1e-3, f_type=1, px0=-0.5, **kw)
    gy = grid_for(p, cs=2.0)
    _run(p, gy, initial_fields(p, gy, kind="turbulent", seed=ny + n_th), steps=2)


def test_plain_dns_workload_20_steps(cuda_device):
    # the 64 x 193 x 32 DNS workload (R = 7 column kernel, 64- and 32-point
    # transforms): laminar parabola plus seeded noise, one buoyant scalar
    p, gy = ics.config_c1()
    fields = ics.laminar_dns(p, gy, seed=1, amp=0.01)
    _run(p, gy, fields, steps=19)


def test_re_tau_180_slice_256_transforms(cuda_device):
    # 256 x 33 x 256 with the Re_tau = 180 workload's parameters: the
    # 256-point x and z transforms inside a full substep
    import dataclasses
    p, _ = ics.config_c2()
    p = dataclasses.replace(p, ny=33)
    from diablo3_test_b200.grid import create_grid, TANH_ENDS_SYMMETRIC
    gy, _ = create_grid(p.ny, 2.0, TANH_ENDS_SYMMETRIC, 2.0)
    fields = ics.log_law_turbulent(p, gy, seed=2)
    _run(p, gy, fields, steps=0)


def test_radix3_transform_inside_a_step(cuda_device):
    p = small_params(nx=96, ny=33, nz=48, n_th=1)
    gy = grid_for(p)
    _run(p, gy, initial_fields(p, gy, kind="turbulent", seed=11), steps=2)


@pytest.mark.parametrize("model", [LES_SMAGORINSKY, LES_DYNAMIC_SMAGORINSKY])
def test_les_physical_solve_ny129(cuda_device, model):
    p = small_params(nx=32, ny=129, nz=24, n_th=1, use_les=True, create_new_flow=False, re=400.0,
                     les_model_type=model)
    gy = grid_for(p, cs=2.2)
    _run(p, gy, initial_fields(p, gy, kind="turbulent", seed=5), steps=1, les=True)


def test_nonfinite_state_is_reported(cuda_device):
    # a NaN seeded into one physical velocity point on the host spreads
    # through the step; diablo_check_finite reports DIABLO_ERR_NONFINITE
    # (the reference's only guard of this kind stops on dt <= 0,
    # for/advance.f90:113-117)
    from diablo3_test_b200.channel import Channel
    p = small_params(n_th=1)
    gy = grid_for(p)
    fields = initial_fields(p, gy)
    with Channel(p, gy) as ch:
        for name, fid in [("u1", _lib.U1), ("u2", _lib.U2), ("u3", _lib.U3), ("th0", _lib.TH)]:
            ch.upload(fid, np.ascontiguousarray(fields[name]), _lib.LAYOUT_PHYSICAL)
        ch.pre_first_step()
        ch.step(1)
        assert ch.lib.diablo_check_finite(ch.ctx) == 0
        bad = np.ascontiguousarray(fields["u2"]).copy()
        bad[p.ny // 2, 3, 5] = np.nan
        ch.upload(_lib.U2, bad, _lib.LAYOUT_PHYSICAL)
        ch.step(1)
        assert ch.lib.diablo_check_finite(ch.ctx) == _lib.ERR_NONFINITE
        assert not ch.check_finite()
