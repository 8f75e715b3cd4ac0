"""Parity of the CUDA LES substep with the CPU oracle (oracle/les.py), through
the C ABI.

Constant Smagorinsky (model 1) and the anisotropic minimum dissipation
models of Rozema (4) and Verstappen (5) follow les_chan / les_chan_th of the
reference (for/les.f90:20-925, 1091-1412) with the eddy-viscosity terms of
the Crank-Nicolson rows (for/channel.f90:519-547, 657-877).  The
dynamic model (2) has no reference implementation (the reference stops on
it, for/les.f90:272-277); both sides restate Germano/Lilly with a sharp
spectral test filter.  Tolerance: relative L2 error <= 1e-10 per field and
for nu_t.
"""
import numpy as np
import pytest

from diablo3_test_b200 import _lib
from diablo3_test_b200.config import (LES_SMAGORINSKY, LES_DYNAMIC_SMAGORINSKY, LES_AMD_ROZEMA,
                                      LES_AMD_VERSTAPPEN, MIXED)
from tests.helpers import (small_params, grid_for, initial_fields, setup_oracle, setup_gpu,
                           oracle_state, gpu_state, rel_err)

pytestmark = pytest.mark.gpu

TOL = 1e-10

LES_CASES = {
    "smagorinsky": dict(les_model_type=LES_SMAGORINSKY),
    "smagorinsky_neumann_top": dict(les_model_type=LES_SMAGORINSKY, u_bc_ymax=1, w_bc_ymax=1,
                                    u_bc_ymax_c1=0.1),
    "smagorinsky_two_scalars": dict(les_model_type=LES_SMAGORINSKY, n_th=2, pr=[0.71, 1.0],
                                    th_bc_ymin=[0, 1], th_bc_ymax=[0, 1],
                                    th_bc_ymin_c1=[-1.0, 0.0], th_bc_ymax_c1=[1.0, 0.0]),
    "smagorinsky_rotation_forcing": dict(les_model_type=LES_SMAGORINSKY, f_type=1, px0=-0.5, ro=5.0,
                                         grav_x=0.1, dthdx=[0.3]),
    "amd_rozema": dict(les_model_type=LES_AMD_ROZEMA),
    "amd_rozema_neumann_walls": dict(les_model_type=LES_AMD_ROZEMA, u_bc_ymin=1, w_bc_ymin=1,
                                     u_bc_ymax=1, w_bc_ymax=1),
    "amd_verstappen": dict(les_model_type=LES_AMD_VERSTAPPEN),
    "amd_verstappen_two_scalars": dict(les_model_type=LES_AMD_VERSTAPPEN, n_th=2, pr=[0.71, 1.0],
                                       th_bc_ymin=[0, 1], th_bc_ymax=[0, 1],
                                       th_bc_ymin_c1=[-1.0, 0.0], th_bc_ymax_c1=[1.0, 0.0],
                                       u_bc_ymin=1, w_bc_ymin=1),
    "dynamic": dict(les_model_type=LES_DYNAMIC_SMAGORINSKY),
    "dynamic_neumann_top": dict(les_model_type=LES_DYNAMIC_SMAGORINSKY, u_bc_ymax=1, w_bc_ymax=1),
}


def _les_params(kw, **extra):
    kw = dict(kw)
    n_th = kw.pop("n_th", 1)
    base = dict(nx=32, ny=33, nz=24, use_les=True, create_new_flow=False, re=400.0)
    base.update(kw)
    base.update(extra)
    return small_params(n_th=n_th, **base)


def _compare(o, ch, what):
    so, sg = oracle_state(o), gpu_state(ch)
    for k in so:
        e = rel_err(sg[k], so[k])
        assert e < TOL, (what, k, e)
    p = o.p
    nt_o = o.nu_t[:, :p.nz, :p.nx]
    nt_g = ch.download_nu_t()[:, :p.nz, :p.nx]
    e = rel_err(nt_g, nt_o)
    assert e < TOL, (what, "nu_t", e)


@pytest.mark.parametrize("case", sorted(LES_CASES))
def test_les_step_matches_oracle(cuda_device, case):
    p = _les_params(LES_CASES[case])
    gy = grid_for(p)
    fields = initial_fields(p, gy, kind="turbulent", seed=5)
    o = setup_oracle(p, gy, fields)
    ch = setup_gpu(p, gy, fields)
    try:
        o.time_step += 1
        o.rk_step = 1
        o.rk_chan_1()
        ch.set_time(o.time, o.time_step, p.delta_t)
        ch.rk_chan_1(1)
        _compare(o, ch, "rk1")
        assert np.abs(o.nu_t).max() > 0
        for rk in (2, 3):
            o.rk_step = rk
            o.rk_chan_1()
            ch.rk_chan_1(rk)
        o.time += o.delta_t
        ch.set_time(o.time, o.time_step, p.delta_t)
        o.step(2)
        ch.step(2)
        _compare(o, ch, "3 steps")
        assert ch.check_finite()
    finally:
        ch.close()


def test_les_gate_closed_for_new_flow(cuda_device):
    # create_new_flow with time_step <= 100: the LES term is skipped
    # (for/channel.f90:259) and nu_t stays zero
    p = _les_params(dict(les_model_type=LES_SMAGORINSKY), create_new_flow=True)
    gy = grid_for(p)
    fields = initial_fields(p, gy, kind="turbulent", seed=6)
    o = setup_oracle(p, gy, fields)
    ch = setup_gpu(p, gy, fields)
    try:
        o.step(2)
        ch.step(2)
        _compare(o, ch, "gate closed")
        assert np.all(o.nu_t == 0)
    finally:
        ch.close()


@pytest.mark.parametrize("model", [LES_SMAGORINSKY, LES_DYNAMIC_SMAGORINSKY, LES_AMD_VERSTAPPEN])
def test_les_mixed_precision_close_to_fp64(cuda_device, model):
    # the LES model and its transforms in FP32, solves and state in FP64
    from diablo3_test_b200.config import FP64
    p = _les_params(dict(les_model_type=model))
    gy = grid_for(p)
    fields = initial_fields(p, gy, kind="turbulent", seed=7)
    a = setup_gpu(p, gy, fields)
    b = setup_gpu(p, gy, fields)
    try:
        b.set_precision(MIXED)
        a.step(3)
        b.step(3)
        sa, sb = gpu_state(a), gpu_state(b)
        errs = {k: rel_err(sb[k], sa[k]) for k in sa}
        nt = rel_err(b.download_nu_t()[:, :p.nz, :p.nx], a.download_nu_t()[:, :p.nz, :p.nx])
        assert max(v for k, v in errs.items() if k != "p") < 1e-6, errs
        assert errs["p"] < 1e-4, errs
        assert nt < 1e-4, nt
        assert b.check_finite()
    finally:
        a.close()
        b.close()


EPS_CASES = {
    "smagorinsky": dict(les_model_type=LES_SMAGORINSKY),
    "smagorinsky_neumann_top": dict(les_model_type=LES_SMAGORINSKY, u_bc_ymax=1, w_bc_ymax=1,
                                    u_bc_ymax_c1=0.1),
    "dynamic": dict(les_model_type=LES_DYNAMIC_SMAGORINSKY),
    "amd_rozema": dict(les_model_type=LES_AMD_ROZEMA),
    "amd_verstappen": dict(les_model_type=LES_AMD_VERSTAPPEN, n_th=2, pr=[0.71, 1.0]),
}


@pytest.mark.parametrize("case", sorted(EPS_CASES))
def test_les_eps_sgs1_matches_oracle(cuda_device, case):
    """eps_sgs1 (for/les.f90:924-1068): a statistics save requests it, the
    next step's first substep forms it.  The GPU's Parseval sums against the
    oracle's physical-space loops, relative to the profile's largest value."""
    p = _les_params(EPS_CASES[case])
    gy = grid_for(p)
    fields = initial_fields(p, gy, kind="turbulent", seed=9)
    o = setup_oracle(p, gy, fields)
    ch = setup_gpu(p, gy, fields)
    try:
        o.step(1)
        ch.step(1)
        with pytest.raises(_lib.DiabloError) as e:       # nothing requested yet
            ch.les_eps_sgs1()
        assert e.value.status == _lib.ERR_STATE
        ch.stats()                                       # flag_save_LES
        o.apply_bc_vel_post()                            # what save_stats_chan applies
        o.apply_bc_th_post()
        o.flag_save_les = True
        with pytest.raises(_lib.DiabloError):            # requested, not yet formed
            ch.les_eps_sgs1()
        o.step(1)
        ch.step(1)
        eg, eo = ch.les_eps_sgs1(), o.eps_sgs1
        scale = np.abs(eo).max()
        assert scale > 0
        assert np.abs(eg - eo).max() <= TOL * scale, np.abs(eg - eo).max() / scale
        assert eg[0] == 0.0
        _compare(o, ch, "after the eps_sgs1 step")
        # formed once per request: a further step leaves the value in place
        ch.step(1)
        assert np.array_equal(ch.les_eps_sgs1(), eg)
    finally:
        ch.close()


def test_les_eps_sgs1_mixed_close_to_fp64(cuda_device):
    p = _les_params(dict(les_model_type=LES_DYNAMIC_SMAGORINSKY))
    gy = grid_for(p)
    fields = initial_fields(p, gy, kind="turbulent", seed=10)
    a = setup_gpu(p, gy, fields)
    b = setup_gpu(p, gy, fields)
    try:
        b.set_precision(MIXED)
        for ch in (a, b):
            ch.step(1)
            ch.stats()
            ch.step(1)
        ea, eb = a.les_eps_sgs1(), b.les_eps_sgs1()
        assert np.abs(eb - ea).max() <= 1e-4 * np.abs(ea).max()
    finally:
        a.close()
        b.close()


def test_les_eps_sgs1_blank_while_gate_closed(cuda_device):
    # a new flow's first 100 steps skip the LES term; the request is answered
    # with blanks (for/channel.f90:271-274)
    p = _les_params(dict(les_model_type=LES_SMAGORINSKY), create_new_flow=True)
    gy = grid_for(p)
    ch = setup_gpu(p, gy, initial_fields(p, gy, kind="turbulent", seed=6))
    try:
        ch.step(1)
        ch.stats()
        ch.step(1)
        assert np.all(ch.les_eps_sgs1() == 0.0)
    finally:
        ch.close()
