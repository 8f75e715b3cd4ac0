"""Generate tests/golden/grids.npz from the reference's own grid tool.

Run in the build container (it imports py/setup/create_grid.py and
py/setup/grid_generators.py from the read-only reference checkout given as
the first argument; h5py and matplotlib, which only that tool's file writer
and plotter use, are stubbed).  The GPU box never runs this script; the tests
read the committed .npz.

    python tests/golden/make_golden.py /path/to/reference
"""
import os
import sys
import types

import numpy as np


def main(ref_root):
    sys.modules.setdefault("h5py", types.ModuleType("h5py"))
    mpl = types.ModuleType("matplotlib")
    mpl.pyplot = types.ModuleType("matplotlib.pyplot")
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", mpl.pyplot)
    sys.path.insert(0, os.path.join(ref_root, "py", "setup"))
    import create_grid as cg          # noqa: E402
    import grid_generators as gg      # noqa: E402
    cases = {
        # (N, H, type, CS): the benchmark grids plus every generator type
        "c1_193_tanh1.8": (193, 2.0, 5, 1.8),
        "c2_257_tanh2.0": (257, 2.0, 5, 2.0),
        "c3_129_tanh2.2": (129, 2.0, 5, 2.2),
        "c4_97_tanh1.8": (97, 2.0, 5, 1.8),
        "c5_33_tanh1.8": (33, 2.0, 5, 1.8),
        "c5_65_tanh1.8": (65, 2.0, 5, 1.8),
        "type1_33": (33, 1.0, 1, 1.5),
        "type2_33": (33, 1.0, 2, 1.5),
        "type3_33": (33, 20.0, 3, 1.5),
        "type4_49": (49, 3.0, 4, 1.7),
        "type6_49": (49, 2.0, 6, 2.5),
    }
    out = {}
    for name, (n, h, kind, cs) in cases.items():
        cls = gg.GRID_GENERATORS[kind]
        gen = cls(CS=cs) if issubclass(cls, gg.StretchedGridGenerator) else cls()
        G, GF = cg.create_grid(n, h, gen)
        out[name + "_G"] = G
        out[name + "_GF"] = GF
        out[name + "_spec"] = np.array([n, h, kind, cs])
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "grids.npz")
    np.savez(path, **out)
    print("wrote", path, len(cases), "grids")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference checkout>")
    main(sys.argv[1])
