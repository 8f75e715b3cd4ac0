"""Ensembles through the C ABI (diablo_ensemble_*): members of uneven grids,
parameters and precisions advanced by one CUDA graph launch per step must end
bit-identical to the same channels stepped one at a time, also after a member
is stepped on its own in between (the graphs are then captured again)."""
import numpy as np
import pytest

from diablo3_test_b200 import _lib
from diablo3_test_b200.config import MIXED, LES_SMAGORINSKY
from tests.helpers import small_params, grid_for, initial_fields, setup_gpu, gpu_state

pytestmark = pytest.mark.gpu

MEMBERS = [
    dict(nx=32, ny=33, nz=32, n_th=1, re=500.0),
    dict(nx=64, ny=33, nz=48, n_th=0, re=1500.0, f_type=1, px0=-0.2),
    dict(nx=48, ny=17, nz=16, n_th=2, re=900.0, precision=MIXED),
    dict(nx=32, ny=33, nz=24, n_th=1, re=400.0, use_les=True, create_new_flow=False,
         les_model_type=LES_SMAGORINSKY),
]


def _build(kw):
    kw = dict(kw)
    n_th = kw.pop("n_th")
    prec = kw.pop("precision", None)
    p = small_params(n_th=n_th, **kw)
    gy = grid_for(p)
    fields = initial_fields(p, gy, kind="turbulent", seed=p.nx + p.nz)
    out = []
    for _ in range(2):
        ch = setup_gpu(p, gy, fields)
        if prec is not None:
            ch.set_precision(prec)
        out.append(ch)
    return out


def _same(a, b):
    sa, sb = gpu_state(a), gpu_state(b)
    return all(np.array_equal(sa[k], sb[k]) for k in sa)


def test_ensemble_matches_members_run_singly(cuda_device):
    from diablo3_test_b200.channel import Ensemble
    pairs = [_build(kw) for kw in MEMBERS]
    try:
        with Ensemble([p[0] for p in pairs]) as ens:
            l0 = [p[0].kernel_launches() for p in pairs]
            ens.step(3)
            ens.synchronize()
            for a, b in pairs:
                b.step(3)
            for i, (a, b) in enumerate(pairs):
                assert _same(a, b), i
                assert a.kernel_launches() > l0[i]
                assert a.time[1] == b.time[1] == 3
            # one member on its own: the buffer parity no longer matches the graphs
            pairs[0][0].step(1)
            pairs[0][1].step(1)
            ens.step(2)
            ens.synchronize()
            for a, b in pairs:
                b.step(2)
            for i, (a, b) in enumerate(pairs):
                assert _same(a, b), i
                assert a.check_finite()
    finally:
        for a, b in pairs:
            a.close()
            b.close()


def test_ensemble_rejects_per_step_arguments(cuda_device):
    from diablo3_test_b200.channel import Ensemble
    p = small_params(n_th=0, f_type=2, px0=-0.2, amp_omega0=0.3, omega0=40.0)
    gy = grid_for(p)
    ch = setup_gpu(p, gy, initial_fields(p, gy))
    try:
        with pytest.raises(_lib.DiabloError) as e:
            Ensemble([ch])
        assert e.value.status == _lib.ERR_UNSUPPORTED
    finally:
        ch.close()


def test_autotune_keeps_results_and_caches(cuda_device):
    from diablo3_test_b200.config import MIXED
    kw = dict(MEMBERS[2])
    a, b = _build(kw)
    try:
        t1 = a.autotune()
        assert len(t1) == 4 and all(v > 0 for v in t1)
        t2 = b.autotune()            # same size and precision: from the cache
        assert t1 == t2
        a.step(3)
        c = _build(kw)
        try:
            c[0].step(3)             # default tiles
            assert _same(a, c[0])
        finally:
            for ch in c:
                ch.close()
    finally:
        a.close()
        b.close()


def test_ensemble_autotune_restores_states(cuda_device):
    from diablo3_test_b200.channel import Ensemble
    pairs = [_build(kw) for kw in MEMBERS[:3]]
    try:
        with Ensemble([p[0] for p in pairs]) as ens:
            ens.step(2)
            for a, b in pairs:
                b.step(2)
            tiles = ens.autotune(2)
            assert len(tiles) == 3
            for i, (a, b) in enumerate(pairs):
                assert _same(a, b), i
                assert a.time[1] == 2
            ens.step(2)
            ens.synchronize()
            for a, b in pairs:
                b.step(2)
            for i, (a, b) in enumerate(pairs):
                assert _same(a, b), i
    finally:
        for a, b in pairs:
            a.close()
            b.close()


# members without LES: the persistent mode (the column steps of every member
# of a rows-per-lane class in one launch per substep); Ny = 97 gives a second
# class (four rows per lane) beside the three-row members
PERSISTENT_MEMBERS = MEMBERS[:3] + [dict(nx=32, ny=97, nz=24, n_th=1, re=700.0, precision=MIXED)]


def test_persistent_ensemble_matches_members_run_singly(cuda_device):
    from diablo3_test_b200.channel import Ensemble
    pairs = [_build(kw) for kw in PERSISTENT_MEMBERS]
    try:
        with Ensemble([p[0] for p in pairs]) as ens:
            assert ens.mode == _lib.ENSEMBLE_PERSISTENT
            ens.step(3)
            ens.synchronize()
            for a, b in pairs:
                b.step(3)
            for i, (a, b) in enumerate(pairs):
                assert _same(a, b), i
            # a member stepped on its own, then the branches mode and back
            pairs[1][0].step(1)
            pairs[1][1].step(1)
            ens.mode = _lib.ENSEMBLE_BRANCHES
            ens.step(1)
            ens.mode = _lib.ENSEMBLE_PERSISTENT
            ens.step(2)
            ens.synchronize()
            for a, b in pairs:
                b.step(3)
            for i, (a, b) in enumerate(pairs):
                assert _same(a, b), i
                assert a.check_finite()
    finally:
        for a, b in pairs:
            a.close()
            b.close()


def test_persistent_ensemble_wait_times_out_and_recovers(cuda_device):
    """One member withholds an arrival (failure injected from the host): its
    projection tasks' bounded waits give up, the launch returns on its own
    and the ensemble reports DIABLO_ERR_TIMEOUT; with the bound restored and
    the member's state reloaded the ensemble steps bit-identically again."""
    from diablo3_test_b200.channel import Ensemble
    pairs = [_build(kw) for kw in PERSISTENT_MEMBERS[:2]]
    try:
        with Ensemble([p[0] for p in pairs]) as ens:
            assert ens.mode == _lib.ENSEMBLE_PERSISTENT
            victim = pairs[1][0]
            assert victim.lib.diablo_set_wait_bound(victim.ctx, 2000, 1) == _lib.OK
            ens.step(1)
            with pytest.raises(_lib.DiabloError) as e:
                ens.synchronize()
            assert e.value.status == _lib.ERR_TIMEOUT
            ens.synchronize()                    # the record was read and cleared
            assert victim.lib.diablo_set_wait_bound(victim.ctx, 1 << 24, 0) == _lib.OK
            pairs[0][1].step(1)
            ref = pairs[1][1]
            ref.step(1)
            fids = [_lib.U1, _lib.U2, _lib.U3, _lib.P] + [_lib.TH + n for n in range(ref.params.n_th)]
            for fid in fids:
                victim.upload(fid, ref.download(fid), _lib.LAYOUT_FOURIER)
            t, n, dt = ref.time
            victim.set_time(t, n, dt)
            ens.step(2)
            ens.synchronize()
            for a, b in pairs:
                b.step(2)
            for i, (a, b) in enumerate(pairs):
                assert _same(a, b), i
    finally:
        for a, b in pairs:
            a.close()
            b.close()
