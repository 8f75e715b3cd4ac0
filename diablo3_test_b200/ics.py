"""Seeded synthetic initial conditions for the benchmark configurations.

The reference builds its initial fields in physical space (``for/ics.f90``)
and reads/writes them through ``start.h5``; neither is part of the step.  The
configurations here are the synthetic stand-ins the step is measured on.  Every
function returns physical fields in the reference layout (numpy shape
``(Ny+2, Nz+2, Nx+2)``, index ``[j, k, i]``) that a caller uploads with
``LAYOUT_PHYSICAL`` and then projects with ``pre_first_step``.
"""
from __future__ import annotations

import math

import numpy as np

from .config import ChannelParams
from .grid import create_grid, metrics, TANH_ENDS_SYMMETRIC


def _empty(p: ChannelParams):
    return np.zeros((p.ny + 2, p.nz + 2, p.nx + 2))


def _noise(rng, p: ChannelParams, amp, damp):
    """Gaussian noise with its plane mean removed, scaled by amp*damp(y)."""
    f = _empty(p)
    n = rng.standard_normal((p.ny + 2, p.nz, p.nx))
    n -= n.mean(axis=(1, 2), keepdims=True)
    f[:, :p.nz, :p.nx] = amp * damp[:, None, None] * n
    return f


def laminar_dns(p: ChannelParams, gy, seed: int = 1, amp: float = 0.01):
    """Laminar parabola u1 = 1.5(1 - y^2) plus seeded Gaussian noise of
    amplitude ``amp`` (plane mean removed) and scalar th_n = y."""
    _, gyf, _, _ = metrics(gy)
    rng = np.random.default_rng(seed)
    y = gyf
    fields = {}
    ones = np.ones_like(y)
    u1 = _noise(rng, p, amp, ones)
    u1[:, :p.nz, :p.nx] += (1.5 * (1.0 - y ** 2))[:, None, None]
    fields["u1"] = u1
    fields["u2"] = _noise(rng, p, amp, ones)
    fields["u3"] = _noise(rng, p, amp, ones)
    for n in range(p.n_th):
        t = _empty(p)
        t[:, :p.nz, :p.nx] = y[:, None, None]
        fields[f"th{n}"] = t
    return fields


def log_law_turbulent(p: ChannelParams, gy, seed: int = 2, amp: float = 0.1, re_tau: float = 180.0):
    """Log-law mean (u+ = y+ below y+ = 11, (1/0.41) ln y+ + 5.2 above) in
    wall units with u_tau = 1, plus seeded random perturbations of ``amp``
    times the centreline velocity, damped to zero at the walls; the projection
    in ``pre_first_step`` makes them divergence-free.  Scalars: th_0 = y,
    th_n = y^2 (n >= 1), each with 1% noise."""
    _, gyf, _, _ = metrics(gy)
    rng = np.random.default_rng(seed)
    y = gyf
    yp = np.clip((1.0 - np.abs(y)) * re_tau, 0.0, None)
    with np.errstate(divide="ignore"):
        ulog = np.where(yp < 11.0, yp, np.log(np.maximum(yp, 1e-30)) / 0.41 + 5.2)
    ucl = float(ulog.max())
    damp = np.clip(1.0 - y ** 2, 0.0, None)
    fields = {}
    u1 = _noise(rng, p, amp * ucl, damp)
    u1[:, :p.nz, :p.nx] += ulog[:, None, None]
    fields["u1"] = u1
    fields["u2"] = _noise(rng, p, amp * ucl, damp)
    fields["u3"] = _noise(rng, p, amp * ucl, damp)
    for n in range(p.n_th):
        t = _noise(rng, p, 0.01, damp)
        t[:, :p.nz, :p.nx] += (y if n == 0 else y ** 2)[:, None, None]
        fields[f"th{n}"] = t
    return fields


def config_c1(n_th: int = 1):
    """Plain FP64 DNS: 64 x 193 x 32, Lx = 2pi, Lz = pi, tanh 1.8, Re = 1000,
    Pr = 1, no-slip walls, zero-flux scalar, dt = 1e-3."""
    p = ChannelParams.with_scalars(
        n_th, nx=64, ny=193, nz=32, lx=2 * math.pi, lz=math.pi, ly=2.0, re=1000.0,
        delta_t=1e-3, grav_y=1.0, pr=[1.0] * n_th)
    gy, _ = create_grid(p.ny, 2.0, TANH_ENDS_SYMMETRIC, 1.8)
    return p, gy


def config_c2(precision: int = 0):
    """Turbulent channel at Re_tau = 180: 256 x 257 x 256, Lx = 4pi, Lz = 2pi,
    tanh 2.0, two passive scalars (Pr = 0.71, 1.0), constant pressure gradient
    px0 = -1 (f_type 1), dt = 5e-4."""
    p = ChannelParams.with_scalars(
        2, nx=256, ny=257, nz=256, lx=4 * math.pi, lz=2 * math.pi, ly=2.0, re=180.0,
        delta_t=5e-4, f_type=1, px0=-1.0, pr=[0.71, 1.0],
        th_bc_ymin=[0, 1], th_bc_ymax=[0, 1], th_bc_ymin_c1=[-1.0, 0.0], th_bc_ymax_c1=[1.0, 0.0],
        precision=precision)
    gy, _ = create_grid(p.ny, 2.0, TANH_ENDS_SYMMETRIC, 2.0)
    return p, gy


ENSEMBLE_SIZES = [(32, 33, 32), (64, 65, 64), (96, 97, 64), (128, 65, 128)]


def config_c5(n_members: int = 48, precision: int = 1, seed: int = 5):
    """Ensemble of independent channels with uneven grids: (Nx, Ny, Nz) cycles
    through ENSEMBLE_SIZES; Lx = 2pi, Lz = pi, tanh 1.8; one scalar (Pr 1,
    grav_y 0); Re drawn uniformly from [500, 3000]; dt = 1e-3, mixed precision
    by default.  Returns [(params, gy, physical fields)] with each member's
    own seeded perturbation on the laminar parabola."""
    rng = np.random.default_rng(seed)
    res = rng.uniform(500.0, 3000.0, n_members)
    out = []
    for i in range(n_members):
        nx, ny, nz = ENSEMBLE_SIZES[i % len(ENSEMBLE_SIZES)]
        p = ChannelParams.with_scalars(1, nx=nx, ny=ny, nz=nz, lx=2 * math.pi, lz=math.pi, ly=2.0,
                                       re=float(res[i]), delta_t=1e-3, grav_y=0.0, precision=precision)
        gy, _ = create_grid(ny, 2.0, TANH_ENDS_SYMMETRIC, 1.8)
        out.append((p, gy, laminar_dns(p, gy, seed=seed * 1000 + i, amp=0.05)))
    return out


def config_c4():
    """Adjoint sensitivity case: 64 x 97 x 64, Lx = 2pi, Lz = pi, tanh 1.8,
    Re = 2000, velocities only, dt = 1e-3, laminar parabola driven by the
    matching pressure gradient (f_type 1, px0 = -2/Re) plus seeded noise
    (seed 4)."""
    p = ChannelParams.with_scalars(0, nx=64, ny=97, nz=64, lx=2 * math.pi, lz=math.pi, ly=2.0, re=2000.0,
                                   delta_t=1e-3, f_type=1, px0=-2.0 / 2000.0, grav_y=0.0)
    gy, _ = create_grid(p.ny, 2.0, TANH_ENDS_SYMMETRIC, 1.8)
    return p, gy, laminar_dns(p, gy, seed=4, amp=0.05)


def _spectral_noise(rng, p: ChannelParams, amp, damp, slope=-5.0 / 3.0):
    """Random-phase field whose x-z energy spectrum follows k^slope (shell
    spectrum E(k) ~ k^slope, so |u_hat|^2 ~ k^(slope - 1) in two dimensions),
    zero mean per plane, rms amp * damp(y)."""
    f = _empty(p)
    kx = np.fft.rfftfreq(p.nx, 1.0 / p.nx)
    kz = np.fft.fftfreq(p.nz, 1.0 / p.nz)
    k = np.sqrt(kx[None, :] ** 2 + kz[:, None] ** 2)
    a = np.zeros_like(k)
    a[k > 0] = k[k > 0] ** ((slope - 1.0) / 2.0)
    for j in range(p.ny + 2):
        ph = rng.uniform(0.0, 2.0 * np.pi, k.shape)
        v = np.fft.irfft2(a * np.exp(1j * ph), s=(p.nz, p.nx))
        s = v.std()
        if s > 0:
            f[j, :p.nz, :p.nx] = amp * damp[j] * v / s
    return f


def config_c3(les_model_type: int = 2):
    """LES of a Re_tau = 1000 channel: 128 x 129 x 128, Lx = 2pi, Lz = pi,
    tanh 2.2, velocities only, constant pressure gradient px0 = -1 in wall
    units (Re = 1000), dt = 2e-4, dynamic Smagorinsky by default, started from a
    written state (create_new_flow = False, so the LES term acts from step 1).
    IC: log-law mean plus random-phase fluctuations with a k^-5/3 spectrum of
    10% of the centreline velocity (seed 3)."""
    p = ChannelParams.with_scalars(0, nx=128, ny=129, nz=128, lx=2 * math.pi, lz=math.pi, ly=2.0, re=1000.0,
                                   delta_t=2e-4, f_type=1, px0=-1.0, grav_y=0.0, use_les=True,
                                   les_model_type=les_model_type, create_new_flow=False)
    gy, _ = create_grid(p.ny, 2.0, TANH_ENDS_SYMMETRIC, 2.2)
    _, gyf, _, _ = metrics(gy)
    rng = np.random.default_rng(3)
    yp = np.clip((1.0 - np.abs(gyf)) * 1000.0, 0.0, None)
    with np.errstate(divide="ignore"):
        ulog = np.where(yp < 11.0, yp, np.log(np.maximum(yp, 1e-30)) / 0.41 + 5.2)
    ucl = float(ulog.max())
    damp = np.clip(1.0 - gyf ** 2, 0.0, None)
    fields = {q: _spectral_noise(rng, p, 0.1 * ucl, damp) for q in ("u1", "u2", "u3")}
    fields["u1"][:, :p.nz, :p.nx] += ulog[:, None, None]
    return p, gy, fields
