"""Generate tests/golden/start_h5.npz from the reference's start-file writer.

Run in the build container with the read-only reference checkout as the
argument.  It imports py/setup/start.py, fills a start object with seeded
fields on a small grid, and runs its write_start_file() with dask.array,
h5py and the setup module stubbed so that the datasets and attributes it
would write are captured instead (start.py itself is not changed).  The GPU
box never runs this script; the tests read the committed .npz.

    python tests/golden/make_checkpoint_golden.py /path/to/reference
"""
import os
import sys
import types

import numpy as np


def main(ref_root):
    captured = {"datasets": {}, "attrs": {}, "group_attrs": {}}

    class _Attrs(dict):
        def create(self, name, value, dtype=None):
            self[name] = np.array(value, dtype=dtype)

    class _Group:
        def __init__(self):
            self.attrs = _Attrs()
            captured["group_attrs"] = self.attrs

    class _File:
        def __init__(self, path, mode):
            self.attrs = _Attrs()
            captured["attrs"] = self.attrs

        def __enter__(self):
            return self

        def __exit__(self, *exc):
            return False

        def create_group(self, name):
            assert name == "Timestep"
            return _Group()

    h5py = types.ModuleType("h5py")
    h5py.File = _File
    dask = types.ModuleType("dask")
    da = types.ModuleType("dask.array")
    da.empty = lambda shape: np.empty(shape)
    da.to_hdf5 = lambda path, variables: captured["datasets"].update(
        {k: np.asarray(v) for k, v in variables.items()})
    dask.array = da
    setup_mod = types.ModuleType("setup")
    setup_mod.setup = object
    sys.modules["h5py"] = h5py
    sys.modules["dask"] = dask
    sys.modules["dask.array"] = da
    sys.modules["setup"] = setup_mod
    sys.path.insert(0, os.path.join(ref_root, "py", "setup"))
    import start  # noqa: E402

    nx, ny, nz, nth = 16, 17, 12, 2
    rng = np.random.default_rng(42)
    st = types.SimpleNamespace(
        directory=".", NX=nx, NY=ny, NZ=nz, NTH=nth,
        x_grid=np.arange(nx) * 2 * np.pi / nx, z_grid=np.arange(nz) * np.pi / nz,
        G=np.linspace(-1, 1, ny + 1), GF=0.5 * (np.linspace(-1, 1, ny + 1)[1:] + np.linspace(-1, 1, ny + 1)[:-1]),
        output={"SAVE_FLOW_DT": 0.5, "SAVE_STATS_DT": 0.1, "SAVE_MOVIE_DT": 0.25})
    s = start.start(st)
    s.U = rng.standard_normal((nz, ny, nx))
    s.V = rng.standard_normal((nz, ny + 1, nx))
    s.W = rng.standard_normal((nz, ny, nx))
    s.TH = rng.standard_normal((nth, nz, ny, nx))
    s.write_start_file()
    out = {"grid": np.array([nx, ny, nz, nth]), "in_U": s.U, "in_V": s.V, "in_W": s.W, "in_TH": s.TH}
    for k, v in captured["datasets"].items():
        out["ds_" + k.split("/")[-1]] = v
    out["attr_Resolution"] = captured["attrs"]["Resolution"]
    for k, v in captured["group_attrs"].items():
        out["gattr_" + k] = v
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "start_h5.npz")
    np.savez(path, **out)
    print("wrote", path, sorted(out))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_checkpoint_golden.py <reference checkout>")
    main(sys.argv[1])
