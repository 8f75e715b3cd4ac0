"""The hand-written discrete adjoint of the channel step (diablo_adjoint_*,
through diablo3_test_b200.adjoint.ChannelSteps) against
  * torch autograd through a pure-torch FP64 restatement of the same step
    (oracle/torch_step.py) on a small grid: relative error <= 1e-9, with and
    without scalars (buoyancy in x, y and z, background gradients, Dirichlet
    and Neumann scalar walls; the objective then adds 1/2 <th^2>);
  * central finite differences along seeded directions with two scalars on a
    small grid: relative error <= 1e-6;
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


SCALARS = dict(grav_y=0.5, grav_x=0.2, grav_z=-0.1, pr=[0.71, 1.0], dthdx=[0.3, 0.0],
               dthdz=[0.0, -0.2], th_bc_ymin=[1, 0], th_bc_ymax=[0, 1], th_bc_ymin_c1=[0.1, 0.0],
               th_bc_ymax_c1=[0.0, 0.05])

CASES = {
    "no_slip": dict(n_th=0, grav_y=0.0),
    "rotation_forcing": dict(n_th=0, grav_y=0.0, f_type=1, px0=-0.3, ro=3.0),
    "neumann_walls": dict(n_th=0, grav_y=0.0, u_bc_ymin=1, w_bc_ymax=1, u_bc_ymax_c1=0.1),
    "one_scalar_buoyancy": dict(n_th=1, grav_y=0.8),
    "two_scalars": dict(n_th=2, **SCALARS),
}


def _state_fields(p):
    return list(FIELDS) + [_lib.TH + n for n in range(p.n_th)]


@pytest.mark.parametrize("case", sorted(CASES))
def test_adjoint_matches_torch_autograd(cuda_device, case):
    from diablo3_test_b200.adjoint import ChannelSteps
    from oracle.torch_step import TorchChannel
    p = small_params(nx=32, ny=33, nz=24, re=300.0, **CASES[case])
    gy = grid_for(p)
    ch = setup_gpu(p, gy, initial_fields(p, gy, kind="turbulent", seed=9))
    _, _, dy, dyf = metrics(gy)
    dyt = torch.tensor(dy, dtype=torch.float64)
    dyft = torch.tensor(dyf, dtype=torch.float64)
    box = _box(p)
    nsteps, every = 3, 2
    fids = _state_fields(p)
    # the objective: kinetic energy plus 1/2 <th^2> of every scalar
    obj = lambda st: TorchChannel.energy(st, p, dyt.to(st[0].device), dyft.to(st[0].device))
    try:
        x0 = [torch.tensor(ch.download(f), device="cuda") for f in fids]
        # hand-written adjoint through the autograd Function
        xs = [x.clone().requires_grad_(True) for x in x0]
        out = ChannelSteps.apply(ch, nsteps, every, *xs)
        c = [_cview(o, p)[box] for o in out[:3]] + [_cview(o, p)[box] for o in out[4:]]
        J = obj(c)
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
        Jr = obj(list(st[:3]) + list(st[4:]))
        Jr.backward()
        assert abs(float(J.detach()) - float(Jr.detach())) < 1e-12 * abs(float(Jr.detach()))
        names = ["u1", "u2", "u3", "p"] + [f"th{n}" for n in range(p.n_th)]
        for name, l, g in zip(names, leaves, g_gpu):
            gr = torch.view_as_complex(l.grad)
            err = float((g - gr).abs().max() / gr.abs().max())
            assert err < 1e-9, (case, name, err)
    finally:
        ch.close()


FD_VARIANTS = {
    "plain": {},
    "filtered": dict(filter_th=[True, True], filter_int=[2, 4]),
    "front": dict(flavor="Front", ro=4.0, delta=0.8),
}


@pytest.mark.parametrize("variant", sorted(FD_VARIANTS))
def test_adjoint_finite_differences_scalars(cuda_device, variant):
    """Two scalars with buoyancy and background gradients, 48 x 65 x 32,
    20 steps with checkpoints every 5: the directional derivative of
    J = 1/2 <u.u> + 1/2 <th.th> from the adjoint against central finite
    differences along 4 seeded directions (perturbing velocities and
    scalars).  "filtered": filter_scalars filters the scalars every 2 and 4
    steps (for/advance.f90:161-173); 20 is a multiple of both, so every
    evaluation meets the filter at the same steps of its run.  "front": the
    'Front' flavor's thermal-wind advection of velocities and scalars
    (for/forcing.f90:37-113) with rotation."""
    p = small_params(nx=48, ny=65, nz=32, re=500.0, delta_t=1e-3, n_th=2, **SCALARS,
                     **FD_VARIANTS[variant])
    gy = grid_for(p)
    _, _, dy, dyf = metrics(gy)
    ch = setup_gpu(p, gy, initial_fields(p, gy, kind="turbulent", seed=6))
    nsteps, every = 20, 5
    box = _box(p)
    fids = _state_fields(p)
    nq = 3 + p.n_th       # differentiated fields: u1, u2, u3, th..
    qf = [0, 1, 2] + [4 + n for n in range(p.n_th)]
    try:
        x0 = [ch.download(f) for f in fids]
        w = np.full(p.nx // 3 + 1, 2.0)
        w[0] = 1.0
        ly = dyf[1:p.ny + 1].sum()
        wy = []
        for q in range(nq):
            v = np.zeros(p.ny + 2)
            if q == 1:
                v[2:p.ny + 1] = dy[2:p.ny + 1]
            else:
                v[1:p.ny + 1] = dyf[1:p.ny + 1]
            wy.append(v)

        def final(xs):
            for f, x in zip(fids, xs):
                ch.upload(f, x, _lib.LAYOUT_FOURIER)
            ch.step(nsteps)
            return [ch.download(fids[i]).view(np.complex128)[box].copy() for i in qf]

        def dJ(a, b):
            return 0.5 * sum(float((wy[q][:, None, None] * w[None, None, :] *
                                    np.real((a[q] - b[q]) * np.conj(a[q] + b[q]))).sum())
                             for q in range(nq)) / ly

        for f, x in zip(fids, x0):
            ch.upload(f, x, _lib.LAYOUT_FOURIER)
        ch.adjoint_record(nsteps, every)
        xn = [ch.download(f) for f in fids]
        lam = [np.zeros_like(x) for x in xn]
        for q, i in enumerate(qf):
            c = xn[i].view(np.complex128)[box]
            lam[i].view(np.complex128)[box] = (wy[q][:, None, None] * w[None, None, :] / ly) * c
        ch.adjoint_run(lam)
        lam0 = [lam[i].view(np.complex128)[box] for i in qf]
        rng = np.random.default_rng(11)
        xnorm = np.sqrt(sum(np.linalg.norm(x0[i].view(np.complex128)[box]) ** 2 for i in qf))
        for _ in range(4):
            d = [(rng.standard_normal(lam0[0].shape) + 1j * rng.standard_normal(lam0[0].shape)) *
                 np.abs(x0[i].view(np.complex128)[box]) for i in qf]
            dn = np.sqrt(sum(np.linalg.norm(v) ** 2 for v in d))
            d = [v * (1e-6 * xnorm / dn) for v in d]
            xp = [x.copy() for x in x0]
            xm = [x.copy() for x in x0]
            for q, i in enumerate(qf):
                xp[i].view(np.complex128)[box] += d[q]
                xm[i].view(np.complex128)[box] -= d[q]
            fd = dJ(final(xp), final(xm)) / 2.0
            ad = sum(float(np.real(np.vdot(lam0[q], d[q]))) for q in range(nq))
            rel = abs(fd - ad) / abs(ad)
            assert rel < 1e-6, (fd, ad, rel)
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
    from diablo3_test_b200.config import MIXED
    p = small_params(n_th=1)
    gy = grid_for(p)
    ch = setup_gpu(p, gy, initial_fields(p, gy))
    try:
        ch.set_precision(MIXED)
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


def test_adjoint_run_repeats_bit_identically(cuda_device):
    """The record keeps the last segment's substep inputs, so the first run
    recomputes every segment but that one; a second run over the same record
    recomputes all of them.  Both must give the same gradient, bit for bit,
    with one segment and with several."""
    p = small_params(nx=32, ny=33, nz=24, re=300.0, n_th=1, grav_y=0.5)
    gy = grid_for(p)
    ch = setup_gpu(p, gy, initial_fields(p, gy, kind="turbulent", seed=2))
    try:
        rng = np.random.default_rng(3)
        shape = (p.ny + 2, p.nz + 2, p.nx + 2)
        for nsteps, every in ((5, 2), (3, 3)):
            x0 = [ch.download(f) for f in _state_fields(p)]
            ch.adjoint_record(nsteps, every)
            lam0 = [rng.standard_normal(shape) for _ in x0]
            a = [l.copy() for l in lam0]
            b = [l.copy() for l in lam0]
            ch.adjoint_run(a)
            ch.adjoint_run(b)
            for q in range(len(a)):
                assert np.array_equal(a[q], b[q]), (nsteps, every, q)
            for f, x in zip(_state_fields(p), x0):
                ch.upload(f, x, _lib.LAYOUT_FOURIER)
    finally:
        ch.close()
