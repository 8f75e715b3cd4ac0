"""The checkpoint layout transform (diablo3_test_b200/checkpoint.py) against
the reference's own start-file writer (py/setup/start.py:37-62, golden
datasets captured by tests/golden/make_checkpoint_golden.py) and the
reference's WriteHDF5/ReadHDF5 pair (for/phdf5.f90:913-1559).  CPU only."""
import os

import numpy as np
import pytest

from diablo3_test_b200 import checkpoint as ck
from diablo3_test_b200.config import ChannelParams

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "start_h5.npz")


def _golden():
    g = np.load(GOLDEN)
    nx, ny, nz, nth = (int(v) for v in g["grid"])
    p = ChannelParams.with_scalars(nth, nx=nx, ny=ny, nz=nz)
    return p, g


def _state_from_start_inputs(p, g, wall_rows):
    """Reference-layout physical fields holding start.py's inputs: U, W, TH
    at GYF rows 1..Ny, V at GY rows 1..Ny+1."""
    nx, ny, nz = p.nx, p.ny, p.nz
    shape = (ny + 2, nz + 2, nx + 2)
    u1, u2, u3 = np.zeros(shape), np.zeros(shape), np.zeros(shape)
    u1[1:ny + 1, :nz, :nx] = np.transpose(g["in_U"], (1, 0, 2))
    u3[1:ny + 1, :nz, :nx] = np.transpose(g["in_W"], (1, 0, 2))
    v = np.array(g["in_V"])
    if wall_rows:
        # the wall rows the step leaves in u2: u2(1) = u2(2), u2(Ny+1) = u2(Ny)
        v[:, 0, :] = v[:, 1, :]
        v[:, ny, :] = v[:, ny - 1, :]
    u2[1:ny + 2, :nz, :nx] = np.transpose(v, (1, 0, 2))
    th = []
    for n in range(p.n_th):
        t = np.zeros(shape)
        t[1:ny + 1, :nz, :nx] = np.transpose(g["in_TH"][n], (1, 0, 2))
        th.append(t)
    return u1, u2, u3, th


def test_datasets_match_the_reference_start_writer():
    p, g = _golden()
    u1, u2, u3, th = _state_from_start_inputs(p, g, wall_rows=False)
    ds = ck.file_datasets(p, u1, u2, u3, th)
    assert np.array_equal(ds["U"], g["ds_U"])
    assert np.array_equal(ds["W"], g["ds_W"])
    for n in range(p.n_th):
        assert np.array_equal(ds[f"TH{n + 1}"], g[f"ds_TH{n + 1}"])
    # V: start.py interpolates the raw GY values; the Fortran writer first
    # sets v(1) = v(2) and v(Ny+1) = v(Ny) (g2gf).  The interior rows agree.
    assert ds["V"].shape == g["ds_V"].shape
    assert np.array_equal(ds["V"][:, 1:p.ny - 1, :], g["ds_V"][:, 1:p.ny - 1, :])


def test_datasets_match_for_wall_consistent_v():
    p, g = _golden()
    u1, u2, u3, th = _state_from_start_inputs(p, g, wall_rows=True)
    v = np.array(g["in_V"])
    v[:, 0, :] = v[:, 1, :]
    v[:, p.ny, :] = v[:, p.ny - 1, :]
    expect = (v[:, :-1, :] + v[:, 1:, :]) / 2   # start.py's interpolation
    assert np.array_equal(ck.file_datasets(p, u1, u2, u3, th)["V"], expect)


def test_attributes_match_the_reference_start_writer():
    p, g = _golden()
    fa, ga = ck.file_attributes(p, time=float(g["gattr_Time"]), time_step=int(g["gattr_Time_Step"]),
                                save_flow_time=float(g["gattr_Save_Flow_Time"]),
                                save_stats_time=float(g["gattr_Save_Stats_Time"]),
                                save_movie_time=float(g["gattr_Save_Movie_Time"]))
    assert np.array_equal(fa["Resolution"], g["attr_Resolution"])
    assert fa["Resolution"].dtype == g["attr_Resolution"].dtype
    for k in ck.TIME_ATTRS + ("Time_Step",):
        assert ga[k] == g[f"gattr_{k}"], k


def test_reading_the_reference_start_file():
    # ReadHDF5 on start.py's datasets: U, W, TH placed exactly; u2 recovered
    # at GY rows 2..Ny-1 by gf2g's recurrence, with the reference's ghost rows
    p, g = _golden()
    ny = p.ny
    f = ck.fields_from_datasets(p, {k[3:]: g[k] for k in g.files if k.startswith("ds_")})
    u1, u2, u3, th = _state_from_start_inputs(p, g, wall_rows=True)
    assert np.array_equal(f["u1"], u1) and np.array_equal(f["u3"], u3)
    for n in range(p.n_th):
        assert np.array_equal(f[f"th{n}"], th[n])
    vf = np.transpose(g["ds_V"], (1, 0, 2))     # [y][z][x], y = 1..Ny
    r = f["u2"][:, :p.nz, :p.nx]
    for y in range(2, ny):   # rows 1 and Ny+1 are overwritten by the ghost rows
        assert np.allclose(r[y] + r[y + 1], 2 * vf[y - 1], rtol=0, atol=1e-12), y
    assert np.array_equal(r[1], -r[2]) and np.array_equal(r[ny + 1], -r[ny])


def test_write_then_read_round_trip():
    rng = np.random.default_rng(9)
    p = ChannelParams.with_scalars(1, nx=16, ny=33, nz=12)
    nx, ny, nz = p.nx, p.ny, p.nz
    shape = (ny + 2, nz + 2, nx + 2)
    f = {k: rng.standard_normal(shape) for k in ("u1", "u2", "u3", "th0", "p")}
    ds = ck.file_datasets(p, f["u1"], f["u2"], f["u3"], [f["th0"]], f["p"])
    assert set(ds) == {"U", "V", "W", "TH1", "P"}
    assert all(d.shape == (nz, ny, nx) for d in ds.values())
    back = ck.fields_from_datasets(p, ds)
    box = (slice(1, ny + 1), slice(0, nz), slice(0, nx))
    for k in ("u1", "u3", "th0", "p"):
        assert np.array_equal(back[k][box], f[k][box]), k
        assert np.count_nonzero(back[k]) == np.count_nonzero(back[k][box])
    # u2: rows 2..Ny come back (the reference's own round trip), the ghost
    # rows become -u2(2) and -u2(Ny)
    u2, b2 = f["u2"][:, :nz, :nx], back["u2"][:, :nz, :nx]
    assert np.allclose(b2[2:ny + 1], u2[2:ny + 1], rtol=0, atol=1e-12 * np.abs(u2).max())
    assert np.array_equal(b2[1], -b2[2]) and np.array_equal(b2[ny + 1], -b2[ny])


def test_wrong_shape_is_rejected():
    p = ChannelParams.with_scalars(0, nx=16, ny=33, nz=12)
    with pytest.raises(ValueError):
        ck.fields_from_datasets(p, {"U": np.zeros((12, 32, 16)), "V": np.zeros((12, 33, 16)),
                                    "W": np.zeros((12, 33, 16))})


def test_hdf5_io_needs_h5py():
    try:
        import h5py  # noqa: F401
        pytest.skip("h5py is installed")
    except ImportError:
        pass
    with pytest.raises(ImportError, match="h5py"):
        ck.save_checkpoint("/nonexistent/x.h5", None)
