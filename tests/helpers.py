"""Shared test helpers: build matching GPU and oracle channels from one
seeded initial condition and compare their states."""
import numpy as np

from diablo3_test_b200 import _lib
from diablo3_test_b200.config import ChannelParams
from diablo3_test_b200.grid import create_grid, TANH_ENDS_SYMMETRIC
from diablo3_test_b200 import ics


def small_params(nx=32, ny=33, nz=24, n_th=1, **kw):
    base = dict(nx=nx, ny=ny, nz=nz, lx=2 * np.pi, lz=np.pi, re=200.0, delta_t=2e-3, grav_y=0.5)
    base.update(kw)
    th = {k: base.pop(k) for k in list(base) if k in (
        "pr", "ri", "th_bc_ymin", "th_bc_ymax", "th_bc_ymin_c1", "th_bc_ymax_c1", "dthdx", "dthdz",
        "filter_th", "filter_int")}
    return ChannelParams.with_scalars(n_th, **base, **th)


def grid_for(p, cs=1.8):
    gy, _ = create_grid(p.ny, 2.0, TANH_ENDS_SYMMETRIC, cs)
    return gy


def initial_fields(p, gy, kind="laminar", seed=1):
    if kind == "laminar":
        return ics.laminar_dns(p, gy, seed=seed, amp=0.05)
    return ics.log_law_turbulent(p, gy, seed=seed)


def field_ids(p):
    return [("u1", _lib.U1), ("u2", _lib.U2), ("u3", _lib.U3)] + \
        [(f"th{n}", _lib.TH + n) for n in range(p.n_th)]


def setup_oracle(p, gy, fields, workers=1):
    from oracle.channel import OracleChannel
    o = OracleChannel(p, gy, workers=workers)
    o.u1.r[:] = fields["u1"]
    o.u2.r[:] = fields["u2"]
    o.u3.r[:] = fields["u3"]
    for n in range(p.n_th):
        o.th[n].r[:] = fields[f"th{n}"]
    for f in [o.u1, o.u2, o.u3] + o.th:
        o.fft_xz_to_fourier(f)
    o.pre_first_step()
    return o


def setup_gpu(p, gy, fields):
    from diablo3_test_b200.channel import Channel
    ch = Channel(p, gy)
    for name, fid in field_ids(p):
        ch.upload(fid, np.ascontiguousarray(fields[name]), _lib.LAYOUT_PHYSICAL)
    ch.pre_first_step()
    return ch


def sig(p, buf):
    """Significant Fourier entries of a reference-layout buffer."""
    c = buf.view(np.complex128)
    return c[:, :2 * (p.nz // 3) + 1, :p.nx // 2]


def oracle_state(o):
    p = o.p
    st = {"u1": sig(p, o.u1.buf), "u2": sig(p, o.u2.buf), "u3": sig(p, o.u3.buf), "p": sig(p, o.p_.buf)}
    for n in range(p.n_th):
        st[f"th{n}"] = sig(p, o.th[n].buf)
    return st


def gpu_state(ch):
    p = ch.params
    st = {}
    for name, fid in field_ids(p) + [("p", _lib.P)]:
        st[name] = sig(p, ch.download(fid)).copy()
    return st


def rel_err(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
