"""The pure-torch FP64 step (oracle/torch_step.py, the reference gradient of
the adjoint tests) against the numpy restatement of rk_chan_1
(oracle/channel.py) on CPU: same initial Fourier state, two RK3 steps, every
field within 1e-11 relative.  The scalar case covers buoyancy in all three
directions (for/channel.f90:156-172), the background gradients (:240-249),
Dirichlet and Neumann scalar walls (:1797-1876) and two Prandtl numbers."""
import numpy as np
import pytest
import torch

from tests.helpers import small_params, grid_for, initial_fields, setup_oracle

CASES = {
    "velocity_only": dict(n_th=0, grav_y=0.0),
    "rotation_forcing": dict(n_th=0, grav_y=0.0, f_type=1, px0=-0.3, ro=3.0),
    "two_scalars": dict(n_th=2, grav_y=0.5, grav_x=0.2, grav_z=-0.1, pr=[0.71, 1.0],
                        dthdx=[0.3, 0.0], dthdz=[0.0, -0.2], th_bc_ymin=[1, 0], th_bc_ymax=[0, 1],
                        th_bc_ymin_c1=[0.1, 0.0], th_bc_ymax_c1=[0.0, 0.05]),
}


def _box(p):
    return slice(None), slice(0, 2 * (p.nz // 3) + 1), slice(0, p.nx // 3 + 1)


@pytest.mark.parametrize("case", sorted(CASES))
def test_torch_step_matches_numpy_oracle(case):
    from oracle.torch_step import TorchChannel
    kw = dict(CASES[case])
    p = small_params(nx=16, ny=17, nz=12, re=300.0, **kw)
    gy = grid_for(p)
    o = setup_oracle(p, gy, initial_fields(p, gy, kind="turbulent", seed=3))
    box = _box(p)
    fields = [o.u1, o.u2, o.u3, o.p_] + list(o.th)
    st = tuple(torch.tensor(f.c[box].copy()) for f in fields)
    tc = TorchChannel(p, gy)
    out = tc.step(st, 2)
    o.step(2)
    names = ["u1", "u2", "u3", "p"] + [f"th{n}" for n in range(p.n_th)]
    for name, a, f in zip(names, out, fields):
        ref = f.c[box]
        err = float(np.abs(a.numpy() - ref).max() / np.abs(ref).max())
        assert err < 1e-11, (case, name, err)
