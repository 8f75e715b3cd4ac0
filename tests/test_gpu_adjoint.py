"""The hand-written discrete adjoint of the channel step (diablo_adjoint_*,
through diablo3_test_b200.adjoint.ChannelSteps) against
  * torch autograd through a pure-torch FP64 restatement of the same step
    (oracle/torch_step.py) on a small grid: relative error <= 1e-9;
  * central finite differences (eps = 1e-6 relative) of the volume-averaged
    kinetic energy after 50 steps of the 64 x 97 x 64, Re = 2000 case along
    8 seeded random directions: relative error <= 1e-6.  The directions are
    complex Gaussian noise scaled entry by entry by |x0| (perturbations shaped
    like the state; white noise is nearly orthogonal to a gradient carried by
    the mean flow, and its directional derivative drowns in round-off), and
    J(x+) - J(x-) is formed from the difference of the final states.
"""
import numpy as np
import pytest
import torch

from diablo3_test_b200 import _lib, ics
from diablo3_test_b200.grid import metrics
from tests.helpers import small_params, grid_for, initial_fields, setup_gpu

pytestmark = pytest.mark.gpu

FIELDS = (_lib.U1, _lib.U2, _lib.U3, _lib.P)


def _box(p):
    return slice(None), slice(0, 2 * (p.nz // 3) + 1), slice(0, p.nx // 3 + 1)


def _cview(t, p):
    """Complex view (Ny+2, Nz+2, Nx/2+1) of a reference-layout real tensor."""
    return torch.view_as_complex(t.reshape(p.ny + 2, p.nz + 2, p.nx // 2 + 1, 2))


def _energy_torch(u1, u2, u3, p, dy, dyf):
    from oracle.torch_step import TorchChannel
    return TorchChannel.energy((u1, u2, u3), p, dy, dyf)


CASES = {
    "no_slip": dict(),
    "rotation_forcing": dict(f_type=1, px0=-0.3, ro=3.0),
    "neumann_walls": dict(u_bc_ymin=1, w_bc_ymax=1, u_bc_ymax_c1=0.1),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_adjoint_matches_torch_autograd(cuda_device, case):
    from diablo3_test_b200.adjoint import ChannelSteps
    from oracle.torch_step import TorchChannel
    p = small_params(nx=32, ny=33, nz=24, n_th=0, re=300.0, grav_y=0.0, **CASES[case])
    gy = grid_for(p)
    ch = setup_gpu(p, gy, initial_fields(p, gy, kind="turbulent", seed=9))
    _, _, dy, dyf = metrics(gy)
    dyt = torch.tensor(dy, dtype=torch.float64)
    dyft = torch.tensor(dyf, dtype=torch.float64)
    box = _box(p)
    nsteps, every = 3, 2
    try:
        x0 = [torch.tensor(ch.download(f), device="cuda") for f in FIELDS]
        # hand-written adjoint through the autograd Function
        xs = [x.clone().requires_grad_(True) for x in x0]
        out = ChannelSteps.apply(ch, nsteps, every, *xs)
        c = [_cview(o, p)[box] for o in out[:3]]
        J = _energy_torch(*c, p, dyt.cuda(), dyft.cuda())
        J.backward()
        g_gpu = [torch.view_as_complex(
            x.grad.reshape(p.ny + 2, p.nz + 2, p.nx // 2 + 1, 2))[box].cpu() for x in xs]
        # pure-torch FP64 step with autograd
        tc = TorchChannel(p, gy)
        leaves = [torch.view_as_real(_cview(x.cpu(), p)[box]).clone().requires_grad_(True) for x in x0]
        st = tc.step(tuple(torch.view_as_complex(l) for l in leaves), nsteps)
        for a, b in zip(st, out):
            ref = _cview(b.detach().cpu(), p)[box]
            assert float((a.detach() - ref).abs().max() / ref.abs().max()) < 1e-10
        Jr = _energy_torch(st[0], st[1], st[2], p, dyt, dyft)
        Jr.backward()
        assert abs(float(J.detach()) - float(Jr.detach())) < 1e-12 * abs(float(Jr.detach()))
        for name, l, g in zip(("u1", "u2", "u3", "p"), leaves, g_gpu):
            gr = torch.view_as_complex(l.grad)
            err = float((g - gr).abs().max() / gr.abs().max())
            assert err < 1e-9, (case, name, err)
    finally:
        ch.close()


def test_adjoint_finite_differences_c4(cuda_device):
    p, gy, fields = ics.config_c4()
    _, _, dy, dyf = metrics(gy)
    ch = setup_gpu(p, gy, fields)
    nsteps, every = 50, 10
    box = _box(p)
    try:
        x0 = [ch.download(f) for f in FIELDS]

        w = np.full(p.nx // 3 + 1, 2.0)
        w[0] = 1.0
        ly = dyf[1:p.ny + 1].sum()
        wy = [np.zeros(p.ny + 2) for _ in range(3)]
        wy[0][1:p.ny + 1] = dyf[1:p.ny + 1]
        wy[2][1:p.ny + 1] = dyf[1:p.ny + 1]
        wy[1][2:p.ny + 1] = dy[2:p.ny + 1]

        def final(xs):
            for f, x in zip(FIELDS, xs):
                ch.upload(f, x, _lib.LAYOUT_FOURIER)
            ch.step(nsteps)
            return [ch.download(f).view(np.complex128)[box].copy() for f in FIELDS[:3]]

        def dJ(a, b):
            # J(a) - J(b) = 1/2 sum w Re((a - b) conj(a + b)) / Ly
            return 0.5 * sum(float((wy[q][:, None, None] * w[None, None, :] *
                                    np.real((a[q] - b[q]) * np.conj(a[q] + b[q]))).sum())
                             for q in range(3)) / ly

        for f, x in zip(FIELDS, x0):
            ch.upload(f, x, _lib.LAYOUT_FOURIER)
        ch.adjoint_record(nsteps, every)
        xn = [ch.download(f) for f in FIELDS]
        # dJ/dx_N of J = 1/2 <u.u>: w(m) * metric weight * u / Ly, packed (dRe, dIm)
        lam = [np.zeros_like(x) for x in xn]
        for q in range(3):
            c = xn[q].view(np.complex128)[box]
            g = lam[q].view(np.complex128)
            g[box] = (wy[q][:, None, None] * w[None, None, :] / ly) * c
        ch.adjoint_run(lam)
        lam0 = [l.view(np.complex128)[box] for l in lam]
        rng = np.random.default_rng(4)
        xnorm = np.sqrt(sum(np.linalg.norm(x.view(np.complex128)[box]) ** 2 for x in x0[:3]))
        for _ in range(8):
            d = [(rng.standard_normal(lam0[0].shape) + 1j * rng.standard_normal(lam0[0].shape)) *
                 np.abs(x0[q].view(np.complex128)[box]) for q in range(3)]
            dn = np.sqrt(sum(np.linalg.norm(v) ** 2 for v in d))
            d = [v * (1e-6 * xnorm / dn) for v in d]
            xp = [x.copy() for x in x0]
            xm = [x.copy() for x in x0]
            for q in range(3):
                xp[q].view(np.complex128)[box] += d[q]
                xm[q].view(np.complex128)[box] -= d[q]
            fd = dJ(final(xp), final(xm)) / 2.0
            ad = sum(float(np.real(np.vdot(lam0[q], d[q]))) for q in range(3))
            rel = abs(fd - ad) / abs(ad)
            assert rel < 1e-6, (fd, ad, rel)
    finally:
        ch.close()


def test_adjoint_rejects_unsupported_and_stale(cuda_device):
    p = small_params(n_th=1)
    gy = grid_for(p)
    ch = setup_gpu(p, gy, initial_fields(p, gy))
    try:
        with pytest.raises(_lib.DiabloError) as e:
            ch.adjoint_record(2, 1)
        assert e.value.status == _lib.ERR_UNSUPPORTED
    finally:
        ch.close()
    p = small_params(n_th=0, grav_y=0.0)
    ch = setup_gpu(p, gy, initial_fields(p, gy))
    try:
        ch.adjoint_record(2, 1)
        ch.step(1)
        lam = [np.zeros((p.ny + 2, p.nz + 2, p.nx + 2)) for _ in range(4)]
        with pytest.raises(_lib.DiabloError) as e:
            ch.adjoint_run(lam)
        assert e.value.status == _lib.ERR_STATE
    finally:
        ch.close()
