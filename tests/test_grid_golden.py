"""Wall-normal grids against golden vectors produced by the reference's own
grid tool (py/setup/create_grid.py; fixture generator tests/golden/make_golden.py),
and the metric restatements of for/domain.f90 against each other."""
import os

import numpy as np
import pytest

from diablo3_test_b200.grid import create_grid, metrics
from oracle.channel import grid_metrics

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "grids.npz")


def _cases():
    g = np.load(GOLDEN)
    names = sorted({k[:-5] for k in g.files if k.endswith("_spec")})
    return [(n, g[n + "_spec"], g[n + "_G"], g[n + "_GF"]) for n in names]


@pytest.mark.parametrize("name,spec,G,GF", _cases())
def test_create_grid_matches_reference_tool(name, spec, G, GF):
    n, h, kind, cs = int(spec[0]), float(spec[1]), int(spec[2]), float(spec[3])
    g, gf = create_grid(n, h, kind, cs)
    assert g.shape == (n + 1,) and gf.shape == (n + 2,)
    np.testing.assert_array_equal(g, G)
    np.testing.assert_array_equal(gf, GF)


@pytest.mark.parametrize("name,spec,G,GF", _cases())
def test_metrics_agree_and_are_consistent(name, spec, G, GF):
    a = metrics(G)
    b = grid_metrics(G)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    gy, gyf, dy, dyf = a
    ny = G.size - 1
    # GYF(1..Ny) are midpoints of the base grid; the rescaling of the reference
    # tool puts GF(1) and GF(N) on the walls, i.e. gy(1) and gy(Ny+1)
    np.testing.assert_allclose(gyf[1:ny + 1], 0.5 * (gy[1:ny + 1] + gy[2:ny + 2]), rtol=0, atol=1e-15)
    assert np.all(dy[1:] > 0) and np.all(dyf[1:ny + 1] > 0)
    np.testing.assert_allclose(GF[1:ny + 1], gyf[1:ny + 1], rtol=0, atol=1e-12 * abs(G).max())
