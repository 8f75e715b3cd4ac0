"""The column step's bounded device wait (diablo_set_wait_bound).  In the
single-launch column step (opt-in, DIABLO_GENERAL_SOLVER=3) each column
group's projection waits on a device counter for the group's three velocity
solves.  Here the host
withholds one arrival, so every such wait runs out after a short bound:
the kernel must return on its own, diablo_step must report
DIABLO_ERR_TIMEOUT, and the context must be usable again once the bound is
restored (the failure is injected from the host; nothing faults on the GPU).
"""
import numpy as np
import pytest

from diablo3_test_b200 import _lib
from tests.helpers import small_params, grid_for, initial_fields, setup_gpu, setup_oracle, gpu_state, \
    oracle_state, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture
def one_launch(monkeypatch):
    # the single-launch column step (read when a context is created)
    monkeypatch.setenv("DIABLO_GENERAL_SOLVER", "3")


def test_withheld_arrival_times_out_and_the_context_recovers(cuda_device, one_launch):
    p = small_params(nx=32, ny=33, nz=24, n_th=1)
    gy = grid_for(p)
    fields = initial_fields(p, gy)
    ch = setup_gpu(p, gy, fields)
    try:
        lib = ch.lib
        assert lib.diablo_set_wait_bound(ch.ctx, 2000, 1) == _lib.OK
        assert lib.diablo_step(ch.ctx, 1) == _lib.ERR_TIMEOUT
        # the record was read and cleared; a synchronize finds nothing new
        assert lib.diablo_synchronize(ch.ctx) == _lib.OK
        # restored bound: a fresh state steps normally and matches the oracle
        assert lib.diablo_set_wait_bound(ch.ctx, 1 << 24, 0) == _lib.OK
        for name, fid in [("u1", _lib.U1), ("u2", _lib.U2), ("u3", _lib.U3), ("th0", _lib.TH)]:
            ch.upload(fid, np.ascontiguousarray(fields[name]), _lib.LAYOUT_PHYSICAL)
        ch.set_time(0.0, 0, p.delta_t)
        ch.pre_first_step()
        o = setup_oracle(p, gy, fields)
        o.step(2)
        ch.step(2)
        so, sg = oracle_state(o), gpu_state(ch)
        for k in ("u1", "u2", "u3", "th0"):
            assert rel_err(sg[k], so[k]) < 1e-10, k
    finally:
        ch.close()


def test_one_launch_step_matches_the_oracle(cuda_device, one_launch):
    p = small_params(nx=32, ny=97, nz=24, n_th=2, pr=[0.71, 1.0], re=400.0, delta_t=1e-3, f_type=1, px0=-0.5)
    gy = grid_for(p, cs=2.0)
    fields = initial_fields(p, gy, kind="turbulent", seed=3)
    o = setup_oracle(p, gy, fields)
    ch = setup_gpu(p, gy, fields)
    try:
        o.step(3)
        ch.step(3)
        so, sg = oracle_state(o), gpu_state(ch)
        for k in so:
            assert rel_err(sg[k], so[k]) < 1e-10, k
    finally:
        ch.close()


def test_wait_bound_rejects_bad_arguments(cuda_device):
    p = small_params(n_th=0)
    gy = grid_for(p)
    ch = setup_gpu(p, gy, initial_fields(p, gy))
    try:
        assert ch.lib.diablo_set_wait_bound(ch.ctx, 0, 0) == _lib.ERR_ARG
        assert ch.lib.diablo_set_wait_bound(ch.ctx, 10, -1) == _lib.ERR_ARG
    finally:
        ch.close()
