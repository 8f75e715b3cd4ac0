"""The allocation-free forward transform, for callers that cannot allocate
device memory (drivers that own every byte through their own pool, code that
cannot afford cudaMalloc's device-wide synchronisation, callers without a
context).  It must give what the context-based diablo_fft_xz_to_fourier
gives, call after call, although all calls share one static scratch array.

This file is named so that pytest collects it last."""
import ctypes

import numpy as np
import pytest

from diablo3_test_b200 import _lib
from tests.helpers import small_params, grid_for, sig, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-13  # same kernels on both paths; relative L2 over significant entries


def _noalloc(lib, p, v_dev, vv_dev):
    return lib.diablo_fft_xz_to_fourier_noalloc(p.nx, p.ny, p.nz, ctypes.c_void_p(v_dev.data_ptr()),
                                                ctypes.c_void_p(vv_dev.data_ptr()), None)


@pytest.mark.parametrize("nx,ny,nz", [(32, 33, 24), (64, 65, 64)])
def test_noalloc_matches_context_transform_on_consecutive_calls(cuda_device, nx, ny, nz):
    import torch
    from diablo3_test_b200.channel import Channel
    lib = _lib.load()
    p = small_params(nx=nx, ny=ny, nz=nz, n_th=0)
    gy = grid_for(p)
    rng = np.random.default_rng(11)
    shape = (ny + 2, nz + 2, nx + 2)
    with Channel(p, gy) as ch:
        for call in range(2):
            v = rng.standard_normal(shape)
            expect = np.zeros(shape)
            ch.fft_xz_to_fourier(v.copy(), expect)
            v_dev = torch.from_numpy(v).to(cuda_device)
            vv_dev = torch.zeros(shape, dtype=torch.float64, device=cuda_device)
            assert _noalloc(lib, p, v_dev, vv_dev) == _lib.OK
            torch.cuda.synchronize()
            got = vv_dev.cpu().numpy()
            assert rel_err(sig(p, got), sig(p, expect)) < TOL, call
            # in place, as the reference calls it (v == vv)
            w_dev = torch.from_numpy(v).to(cuda_device)
            assert _noalloc(lib, p, w_dev, w_dev) == _lib.OK
            torch.cuda.synchronize()
            assert rel_err(sig(p, w_dev.cpu().numpy()), sig(p, expect)) < TOL, call


def test_noalloc_rejects_grids_beyond_its_scratch(cuda_device):
    import torch
    lib = _lib.load()
    p = small_params(nx=256, ny=257, nz=256, n_th=0)
    # full reference-layout buffers (about 138 MB each): should the size
    # check ever regress, the transform stays inside them and the test fails
    # on the return code
    shape = (p.ny + 2, p.nz + 2, p.nx + 2)
    v = torch.zeros(shape, dtype=torch.float64, device=cuda_device)
    vv = torch.zeros(shape, dtype=torch.float64, device=cuda_device)
    assert _noalloc(lib, p, v, vv) == _lib.ERR_SIZE


def test_noalloc_rejects_host_arrays(cuda_device):
    # a Fortran caller passing host arrays gets an error code before anything
    # is queued on the GPU
    import torch
    lib = _lib.load()
    p = small_params(nx=32, ny=33, nz=24, n_th=0)
    shape = (p.ny + 2, p.nz + 2, p.nx + 2)
    h = np.zeros(shape)
    d = torch.zeros(shape, dtype=torch.float64, device=cuda_device)
    hp = ctypes.c_void_p(h.ctypes.data)
    dp = ctypes.c_void_p(d.data_ptr())
    assert lib.diablo_fft_xz_to_fourier_noalloc(p.nx, p.ny, p.nz, hp, dp, None) == _lib.ERR_ARG
    assert lib.diablo_fft_xz_to_fourier_noalloc(p.nx, p.ny, p.nz, dp, hp, None) == _lib.ERR_ARG
    assert _noalloc(lib, p, d, d) == _lib.OK
    torch.cuda.synchronize()


def test_noalloc_leaves_free_device_memory_unchanged(cuda_device):
    import torch
    lib = _lib.load()
    p = small_params(nx=64, ny=65, nz=64, n_th=0)
    shape = (p.ny + 2, p.nz + 2, p.nx + 2)
    v = torch.randn(shape, dtype=torch.float64, device=cuda_device)
    vv = torch.zeros_like(v)
    assert _noalloc(lib, p, v, vv) == _lib.OK   # set-up happens on the first call
    torch.cuda.synchronize()
    before = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert _noalloc(lib, p, v, vv) == _lib.OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == before
