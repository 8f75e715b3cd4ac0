"""A channel's state through the checkpoint layout and back on the device:
physical fields by the device inverse transform (WriteHDF5's
fft_xz_to_physical, for/phdf5.f90:1070-1075), the file datasets, ReadHDF5's
fields, uploaded with the forward transform (:1451-1457).  u1, u3, the
scalars and p come back to transform round-off; u2 at rows 2..Ny (rows 1 and
Ny+1 are ghost/wall rows that ReadHDF5 rewrites)."""
import numpy as np
import pytest

from diablo3_test_b200 import _lib, checkpoint as ck
from tests.helpers import small_params, grid_for, initial_fields, setup_gpu, gpu_state, rel_err

pytestmark = pytest.mark.gpu


def test_state_round_trip_through_checkpoint_layout(cuda_device):
    from diablo3_test_b200.channel import Channel
    p = small_params(nx=32, ny=33, nz=24, n_th=2, pr=[0.71, 1.0])
    gy = grid_for(p)
    a = setup_gpu(p, gy, initial_fields(p, gy, kind="turbulent", seed=12))
    try:
        a.step(2)
        get = lambda fid: a.download(fid, _lib.LAYOUT_PHYSICAL)
        ds = ck.file_datasets(p, get(_lib.U1), get(_lib.U2), get(_lib.U3),
                              [get(_lib.TH + n) for n in range(p.n_th)], get(_lib.P))
        fields = ck.fields_from_datasets(p, ds)
        with Channel(p, gy) as b:
            ids = [("u1", _lib.U1), ("u2", _lib.U2), ("u3", _lib.U3), ("p", _lib.P)] + \
                [(f"th{n}", _lib.TH + n) for n in range(p.n_th)]
            for name, fid in ids:
                b.upload(fid, np.ascontiguousarray(fields[name]), _lib.LAYOUT_PHYSICAL)
            sa, sb = gpu_state(a), gpu_state(b)
            ny = p.ny
            for k in sa:
                if k == "u2":
                    assert rel_err(sb[k][2:ny + 1], sa[k][2:ny + 1]) < 1e-12, k
                else:
                    assert rel_err(sb[k][1:ny + 1], sa[k][1:ny + 1]) < 1e-12, k
    finally:
        a.close()
