"""CPU model of the warp tridiagonal solver in csrc/kernels_solve.cuh
(lane-owned chunks, modified Thomas sweep, interface elimination, parallel
cyclic reduction over 32 lanes), checked against the reference's Thomas
algorithm (for/channel.f90:1335-1540) on the channel's own systems,
including the weakly diagonally dominant Neumann rows and the pinned
kx = kz = 0 pressure mode."""
import numpy as np
import pytest

from diablo3_test_b200.grid import create_grid, TANH_ENDS_SYMMETRIC
from oracle.channel import grid_metrics, OracleChannel

P = 32


def warp_tridiag(a, b, c, d, R):
    """Mirror of csolve::warp_tridiag; arrays of length 32*R, complex d."""
    a = a.reshape(P, R).copy(); b = b.reshape(P, R).copy()
    c = c.reshape(P, R).copy(); d = d.reshape(P, R).astype(complex).copy()
    for r in range(2):
        ib = 1.0 / b[:, r]
        a[:, r] *= ib; c[:, r] *= ib; d[:, r] *= ib
    for r in range(2, R):
        ib = 1.0 / (b[:, r] - a[:, r] * c[:, r - 1])
        d[:, r] = ib * (d[:, r] - a[:, r] * d[:, r - 1])
        a[:, r] = -ib * a[:, r] * a[:, r - 1]
        c[:, r] = ib * c[:, r]
    for r in range(R - 3, 0, -1):
        d[:, r] = d[:, r] - c[:, r] * d[:, r + 1]
        a[:, r] = a[:, r] - c[:, r] * a[:, r + 1]
        c[:, r] = -c[:, r] * c[:, r + 1]
    ib = 1.0 / (1.0 - c[:, 0] * a[:, 1])
    d[:, 0] = ib * (d[:, 0] - c[:, 0] * d[:, 1])
    a[:, 0] = ib * a[:, 0]
    c[:, 0] = -ib * c[:, 0] * c[:, 1]
    as_, gs, ds = a[:, 0], c[:, 0], d[:, 0]
    ae, ge, de = a[:, R - 1], c[:, R - 1], d[:, R - 1]
    sh = lambda x, s, fill: np.concatenate([np.full(s, fill, dtype=x.dtype), x[:-s]])   # from lane t-s
    shd = lambda x, s, fill: np.concatenate([x[s:], np.full(s, fill, dtype=x.dtype)])  # from lane t+s
    L = -as_ * sh(ae, 1, 0.0)
    D = 1.0 - as_ * sh(ge, 1, 0.0) - gs * ae
    U = -gs * ge
    Q = ds - as_ * sh(de, 1, 0.0) - gs * de
    s = 1
    while s < P:
        Lm, Dm, Um, Qm = sh(L, s, 0.0), sh(D, s, 1.0), sh(U, s, 0.0), sh(Q, s, 0.0)
        Lp, Dp, Up, Qp = shd(L, s, 0.0), shd(D, s, 1.0), shd(U, s, 0.0), shd(Q, s, 0.0)
        k1, k2 = L / Dm, U / Dp
        L, U, D, Q = -k1 * Lm, -k2 * Up, D - k1 * Um - k2 * Lp, Q - k1 * Qm - k2 * Qp
        s *= 2
    S = Q / D
    Sn = shd(S, 1, 0.0)
    E = de - ae * S - ge * Sn
    x = d.copy()
    x[:, 0] = S
    x[:, R - 1] = E
    for r in range(1, R - 1):
        x[:, r] = d[:, r] - a[:, r] * S - c[:, r] * E
    return x.reshape(-1)


def thomas(a, b, c, g):
    a, b, g = a.copy(), b.copy(), g.astype(complex).copy()
    n = len(b)
    for j in range(1, n):
        a[j] = -a[j] / b[j - 1]
        b[j] = b[j] + a[j] * c[j - 1]
        g[j] = g[j] + a[j] * g[j - 1]
    g[n - 1] /= b[n - 1]
    for j in range(n - 2, -1, -1):
        g[j] = (g[j] - c[j] * g[j + 1]) / b[j]
    return g


def pad(a, b, c, d, R):
    n = len(b)
    N = P * R
    A = np.zeros(N); B = np.ones(N); C = np.zeros(N); Dd = np.zeros(N, complex)
    A[:n], B[:n], C[:n], Dd[:n] = a, b, c, d
    return A, B, C, Dd


def systems(ny, cs=2.0):
    gy, _ = create_grid(ny, 2.0, TANH_ENDS_SYMMETRIC, cs)
    _, _, dy, dyf = grid_metrics(gy)
    n = ny + 2
    rng = np.random.default_rng(ny)
    out = []
    t1 = 0.5 * (1 / 180.) * (8 / 15.) * 5e-4
    # u1 with Dirichlet rows / theta with Neumann rows
    for neumann in (False, True):
        a = np.zeros(n); b = np.ones(n); c = np.zeros(n)
        for j in range(1, ny + 1):
            a[j] = -t1 / (dy[j] * dyf[j])
            b[j] = 1. + t1 / (dy[j + 1] * dyf[j]) + t1 / (dy[j] * dyf[j])
            c[j] = -t1 / (dy[j + 1] * dyf[j])
        if neumann:
            a[1], b[1], c[1] = 0., -1., 1.
            a[ny], b[ny], c[ny] = -1., 1., 0.
        else:
            a[1], b[1], c[1] = 0., 1., 0.
            a[ny], b[ny], c[ny] = 0., 1., 0.
        a[0], b[0], c[0] = 0., 1., 0.
        a[ny + 1], b[ny + 1], c[ny + 1] = 0., 1., 0.
        out.append((a, b, c, rng.standard_normal(n) + 1j * rng.standard_normal(n)))
    # pressure-correction Poisson, (0,0) mode and a high mode
    for k2 in (0.0, 25.0):
        a = np.zeros(n); b = np.ones(n); c = np.zeros(n)
        for j in range(1, ny + 1):
            a[j] = 1. / (dy[j] * dyf[j])
            b[j] = -k2 - 1. / (dy[j + 1] * dyf[j]) - 1. / (dy[j] * dyf[j])
            c[j] = 1. / (dy[j + 1] * dyf[j])
        a[1], b[1], c[1] = 0., 1., (0. if k2 == 0 else -1.)
        a[ny], b[ny], c[ny] = 1., -1., 0.
        d = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        d[0] = d[1] = d[ny] = d[ny + 1] = 0
        out.append((a, b, c, d))
    return out


@pytest.mark.parametrize("ny", [33, 65, 97, 129, 193, 257])
def test_partition_solver_matches_thomas(ny):
    n = ny + 2
    R = max(3, (n + 31) // 32)
    for a, b, c, d in systems(ny):
        ref = thomas(a, b, c, d)
        x = warp_tridiag(*pad(a, b, c, d, R), R)[:n]
        scale = np.abs(ref).max()
        assert np.abs(x - ref).max() / scale < 1e-11, ny
        # residual of the original system
        res = b * x + np.concatenate([[0], a[1:] * x[:-1]]) + np.concatenate([c[:-1] * x[1:], [0]]) - d
        assert np.abs(res).max() < 1e-9 * max(1.0, np.abs(d).max())


def test_oracle_thomas_is_the_reference_recurrence():
    """The oracle's vectorised Thomas reproduces the scalar recurrence."""
    for a, b, c, d in systems(65):
        A, B, G = a.copy()[:, None], b.copy()[:, None], d.real.copy()[:, None]
        OracleChannel.thomas_real(A, B, c.copy()[:, None], G, len(b) - 2)
        assert np.allclose(G[:, 0], thomas(a, b, c, d.real).real, rtol=1e-13, atol=1e-13)
