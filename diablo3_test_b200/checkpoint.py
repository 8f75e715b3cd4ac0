"""Checkpoint files in the reference's layout (start.h5 / end.h5 / out.*.h5).

The reference writes a checkpoint with WriteHDF5 and reads it with ReadHDF5
(for/phdf5.f90:913-1191 and :1195-1459); its Python tools write start files
with py/setup/start.py:37-62.  The file holds, per field, one dataset of the
physical field on the Nx x Ny x Nz interior points (Fortran dims (Nx, Ny, Nz),
so in C order an array [z, y, x]):

  /Timestep/U, /Timestep/W, /Timestep/TH1..THn   at GYF, y = 1..Ny
  /Timestep/V                                    u2 interpolated to GYF
  /Timestep/P                                    (checkpoints only)

with file attribute Resolution = [Nx, Ny, Nz] and group attributes Time,
Save_Flow_Time, Save_Stats_Time, Save_Movie_Time and Time_Step.

This module is the layout transform between those datasets and the
library's reference-layout physical buffers (Ny+2, Nz+2, Nx+2), including the
reference's wall-normal interpolation of u2 (g2gf, :1530-1547) and its
inverse on reading (gf2g, :1491-1527) with the same boundary rows.  Writing
and reading the HDF5 file itself needs h5py, which is optional: the
transforms work without it.
"""
from __future__ import annotations

import numpy as np

GROUP = "Timestep"
TIME_ATTRS = ("Time", "Save_Flow_Time", "Save_Stats_Time", "Save_Movie_Time")


def _swapzy(v, nx, ny, nz):
    """swapzy (for/phdf5.f90:1462-1475): reference layout [y][z][x] with
    ghosts -> dataset [z][y-1][x] of the interior points."""
    return np.ascontiguousarray(np.transpose(v[1:ny + 1, :nz, :nx], (1, 0, 2)))


def _swapyz(d, nx, ny, nz):
    """swapyz (:1477-1490): dataset [z][y-1][x] -> reference layout, every
    other entry zero."""
    out = np.zeros((ny + 2, nz + 2, nx + 2))
    out[1:ny + 1, :nz, :nx] = np.transpose(d, (1, 0, 2))
    return out


def g2gf(u2, ny):
    """g2gf at one y-rank (:1530-1547): the wall-normal velocity from GY to
    GYF, v(y) = (v(y) + v(y+1)) / 2 for y = 1..Ny after setting v(1) = v(2)
    and v(Ny+1) = v(Ny).  Returns a new array (the reference works in place
    and undoes it with gf2g)."""
    v = np.array(u2, dtype=np.float64, copy=True)
    v[1] = v[2]
    v[ny + 1] = v[ny]
    for y in range(1, ny + 1):
        v[y] = 0.5 * (v[y] + v[y + 1])
    return v


def gf2g(v, ny):
    """gf2g at one y-rank (:1491-1527), in place: v(Ny+1) = v(Ny), then
    v(y) = 2 v(y) - v(y+1) for y = Ny..1, and the zero-mass-flux ghost rows
    v(1) = -v(2), v(Ny+1) = -v(Ny)."""
    v[ny + 1] = v[ny]
    for y in range(ny, 0, -1):
        v[y] = 2 * v[y] - v[y + 1]
    v[1] = -v[2]
    v[ny + 1] = -v[ny]
    return v


def file_datasets(p, u1, u2, u3, th=(), pressure=None):
    """WriteHDF5's datasets from physical fields in the reference layout
    (Ny+2, Nz+2, Nx+2): {'U', 'V', 'W', 'TH1'.., ['P']} as [z][y][x] arrays."""
    nx, ny, nz = p.nx, p.ny, p.nz
    out = {"U": _swapzy(u1, nx, ny, nz), "V": _swapzy(g2gf(u2, ny), nx, ny, nz), "W": _swapzy(u3, nx, ny, nz)}
    for n, t in enumerate(th):
        out[f"TH{n + 1}"] = _swapzy(t, nx, ny, nz)
    if pressure is not None:
        out["P"] = _swapzy(pressure, nx, ny, nz)
    return out


def fields_from_datasets(p, ds):
    """ReadHDF5's fields from the datasets: reference-layout physical arrays
    {'u1', 'u2', 'u3', 'th0'.., ['p']}; u2 is brought back to GY by gf2g."""
    nx, ny, nz = p.nx, p.ny, p.nz
    for name, d in ds.items():
        if d.shape != (nz, ny, nx):
            raise ValueError(f"dataset {name} has shape {d.shape}, the grid needs {(nz, ny, nx)}")
    out = {"u1": _swapyz(ds["U"], nx, ny, nz), "u3": _swapyz(ds["W"], nx, ny, nz)}
    out["u2"] = gf2g(_swapyz(ds["V"], nx, ny, nz), ny)
    n = 1
    while f"TH{n}" in ds:
        out[f"th{n - 1}"] = _swapyz(ds[f"TH{n}"], nx, ny, nz)
        n += 1
    if "P" in ds:
        out["p"] = _swapyz(ds["P"], nx, ny, nz)
    return out


def file_attributes(p, time=0.0, time_step=0, save_flow_time=0.0, save_stats_time=0.0,
                    save_movie_time=0.0):
    """The file's Resolution attribute and the Timestep group's attributes."""
    return ({"Resolution": np.array([p.nx, p.ny, p.nz], dtype=np.int32)},
            {"Time": float(time), "Save_Flow_Time": float(save_flow_time),
             "Save_Stats_Time": float(save_stats_time), "Save_Movie_Time": float(save_movie_time),
             "Time_Step": np.int32(time_step)})


def _h5py():
    try:
        import h5py
    except ImportError as e:
        raise ImportError("reading or writing the HDF5 file needs h5py; the dataset transforms "
                          "(file_datasets, fields_from_datasets) work without it") from e
    return h5py


def save_checkpoint(path, channel, save_pressure=True, **times):
    """WriteHDF5 from a Channel: physical fields by the device inverse
    transform (fft_xz_to_physical semantics), then the file layout."""
    from diablo3_test_b200 import _lib
    h5py = _h5py()
    p = channel.params
    get = lambda fid: channel.download(fid, _lib.LAYOUT_PHYSICAL)
    ds = file_datasets(p, get(_lib.U1), get(_lib.U2), get(_lib.U3),
                       [get(_lib.TH + n) for n in range(p.n_th)],
                       get(_lib.P) if save_pressure else None)
    t, step, _ = channel.time
    fattr, gattr = file_attributes(p, time=t, time_step=step, **times)
    with h5py.File(path, "w") as f:
        for k, v in fattr.items():
            f.attrs[k] = v
        g = f.create_group(GROUP)
        for k, v in gattr.items():
            g.attrs[k] = v
        for k, v in ds.items():
            g.create_dataset(k, data=v)


def load_checkpoint(path, channel):
    """ReadHDF5 into a Channel: checks the resolution, uploads the physical
    fields (transformed on the device), sets the clock; returns whether the
    file held a pressure."""
    from diablo3_test_b200 import _lib
    h5py = _h5py()
    p = channel.params
    with h5py.File(path, "r") as f:
        res = [int(x) for x in f.attrs["Resolution"]]
        if res != [p.nx, p.ny, p.nz]:
            raise ValueError(f"file resolution {res} differs from the grid {[p.nx, p.ny, p.nz]}")
        g = f[GROUP]
        ds = {k: np.asarray(g[k]) for k in g.keys()}
        t = float(g.attrs["Time"])
        step = int(g.attrs["Time_Step"])
    fields = fields_from_datasets(p, ds)
    ids = [("u1", _lib.U1), ("u2", _lib.U2), ("u3", _lib.U3)] + \
        [(f"th{n}", _lib.TH + n) for n in range(p.n_th)] + [("p", _lib.P)]
    for name, fid in ids:
        if name in fields:
            channel.upload(fid, np.ascontiguousarray(fields[name]), _lib.LAYOUT_PHYSICAL)
    channel.set_time(t, step, p.delta_t)
    return "p" in fields
