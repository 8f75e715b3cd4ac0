"""Wall-normal grids of the channel.

``create_grid`` builds the base (G) grid the way the reference's setup tool does
(``py/setup/create_grid.py:22-72`` with the generators of
``py/setup/grid_generators.py:36-73``): points are generated at scaled indices
``J = (-1..N+1)/N``, the fractional grid is taken half-way between them, both
are rescaled so that GF[1] and GF[N] land on the walls, and G is trimmed to
its N+1 interior points.  The result is what the reference reads from
``grid.h5:/grids/y`` into ``gy(1:Ny+1)`` (``for/domain.f90:429-483``).

``metrics`` then derives ``gyf, dy, dyf`` the way ``ReadGridHDF5`` and
``create_grid_chan`` do at one y-rank (``for/domain.f90:230-248,501-527``).
"""
from __future__ import annotations

import numpy as np

# grid generator types, numbered as in py/setup/grid_generators.py:67-74
UNIFORM_POSITIVE = 1
UNIFORM_SYMMETRIC = 2
UNIFORM_NEGATIVE = 3
TANH_ENDS_POSITIVE = 4
TANH_ENDS_SYMMETRIC = 5
CUBIC_CENTRE_SYMMETRIC = 6


def _generate(kind: int, J: np.ndarray, cs: float) -> np.ndarray:
    if kind in (UNIFORM_POSITIVE, UNIFORM_NEGATIVE):
        return J - 1.0
    if kind == UNIFORM_SYMMETRIC:
        return J - 0.5
    if kind == TANH_ENDS_POSITIVE:
        return (np.tanh(cs * (2 * J - 1)) / np.tanh(cs) + 1) / 2
    if kind == TANH_ENDS_SYMMETRIC:
        return np.tanh(cs * (2 * J - 1.0)) / np.tanh(cs) / 2
    if kind == CUBIC_CENTRE_SYMMETRIC:
        return (cs * (2 * J - 1.0) ** 3 + 2 * J - 1.0) / (cs + 1) / 2
    raise ValueError(f"unknown grid type {kind}")


def create_grid(n: int, h: float = 2.0, kind: int = TANH_ENDS_SYMMETRIC,
                cs: float = 1.5):
    """Return ``(G, GF)``: G has n+1 points (gy(1..n+1)), GF has n+2."""
    J = np.arange(-1, n + 2, 1, dtype=np.float64) / n
    G = h * _generate(kind, J, cs)
    GF = (G[:-1] + G[1:]) / 2
    gf_low, gf_up = GF[1], GF[n]
    g_low, g_up = G[1], G[n + 1]
    GF = GF * (g_up - g_low) / (gf_up - gf_low)
    G = G * (g_up - g_low) / (gf_up - gf_low)
    shift = g_low - GF[1]
    GF = GF + shift
    G = G + shift
    return G[1:-1], GF


def metrics(gy_file: np.ndarray):
    """Grid metrics at one y-rank from the n+1 file points ``gy(1..n+1)``.

    Returns arrays indexed 0..Ny+1 (``gy, gyf, dy, dyf``).  ``gy(0)`` and
    ``dy(0)`` are never assigned by the reference (module storage, zero); the
    same zero is used here.
    """
    gy_file = np.asarray(gy_file, dtype=np.float64)
    ny = gy_file.size - 1
    gy = np.zeros(ny + 2)
    gy[1:] = gy_file
    gyf = np.zeros(ny + 2)
    gyf[1:ny + 1] = 0.5 * (gy[1:ny + 1] + gy[2:ny + 2])
    gyf[0] = 2.0 * gyf[1] - gyf[2]
    gyf[ny + 1] = 2.0 * gyf[ny] - gyf[ny - 1]
    dy = np.zeros(ny + 2)
    dy[1:ny + 2] = gyf[1:ny + 2] - gyf[0:ny + 1]
    dyf = np.zeros(ny + 2)
    dyf[1:ny + 1] = gy[2:ny + 2] - gy[1:ny + 1]
    dyf[0] = dyf[1]
    dyf[ny + 1] = dyf[ny]
    return gy, gyf, dy, dyf
