"""diablo_step_host, the host-authoritative round trip (upload the state from
host arrays, step, download into the same arrays) with each field's download
overlapping the next step's upload: after several steps the host arrays must
be bit-identical to the same round trip made of separate upload, step and
download calls, in FP64 and mixed precision; the layout contract and the
host-pointer requirement are enforced."""
import numpy as np
import pytest
import torch

from diablo3_test_b200 import _lib
from diablo3_test_b200.config import MIXED
from tests.helpers import small_params, grid_for, initial_fields, setup_gpu

pytestmark = pytest.mark.gpu


def _ids(p):
    return [_lib.U1, _lib.U2, _lib.U3, _lib.P] + [_lib.TH + n for n in range(p.n_th)]


def _pinned(p):
    shape = (p.ny + 2, p.nz + 2, p.nx + 2)
    return [torch.zeros(shape, dtype=torch.float64, pin_memory=True).numpy() for _ in _ids(p)]


@pytest.mark.parametrize("mixed", [False, True])
def test_step_host_matches_separate_calls(cuda_device, mixed):
    p = small_params(nx=48, ny=65, nz=32, n_th=2, re=600.0)
    gy = grid_for(p)
    fields = initial_fields(p, gy, kind="turbulent", seed=5)
    a, b = setup_gpu(p, gy, fields), setup_gpu(p, gy, fields)
    try:
        if mixed:
            a.set_precision(MIXED)
            b.set_precision(MIXED)
        ba, bb = _pinned(p), _pinned(p)
        for x, y, fid in zip(ba, bb, _ids(p)):
            a.download(fid, out=x)
            b.download(fid, out=y)
        a.step_host(ba, 4)
        for _ in range(4):
            for y, fid in zip(bb, _ids(p)):
                b.upload(fid, y)
            b.step(1)
            for y, fid in zip(bb, _ids(p)):
                b.download(fid, out=y)
        for q, (x, y) in enumerate(zip(ba, bb)):
            assert np.array_equal(x, y), q
        assert a.time[1] == b.time[1] == 4
        # a device array, and a broken layout contract, are rejected
        dev = [torch.zeros(x.shape, dtype=torch.float64, device="cuda") for x in ba]
        arr = (_lib.ctypes.c_void_p * len(dev))(*[t.data_ptr() for t in dev])
        assert a.lib.diablo_step_host(a.ctx, arr, 1) == _lib.ERR_ARG
        bad = [x.copy() for x in ba]
        c = bad[0].view(np.complex128)
        c[3, 1, p.nx // 3 + 2] = 1.0 + 1.0j      # a mode Nkx < i < Nxp
        badp = _pinned(p)
        for x, y in zip(badp, bad):
            x[...] = y
        with pytest.raises(_lib.DiabloError) as e:
            a.step_host(badp, 1)
        assert e.value.status == _lib.ERR_STATE
    finally:
        a.close()
        b.close()
