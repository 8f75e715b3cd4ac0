"""Benchmark of the channel step on the Re_tau = 180 workload (256 x 257 x 256,
three velocities + two scalars), Mpoint-steps/s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm runs the mixed-precision and FP64 steps through the C ABI with the
state resident in HBM (the state, ~1 GB, is larger than L2), times K steps
with CUDA events on the context's stream between barriers, and reports
mixed precision as `value` with FP64 beside it, the mixed-vs-FP64 error, the
dominant kernel's live roofline, an end-to-end figure through the C ABI with
host buffers, the CPU-oracle baseline and the SM clocks seen.  Under torchrun
every rank runs an independent replica (the step does not shard).

The reference arm (`--impl reference`) times the CPU restatement of the
reference's step (the Fortran cannot be built on this image) on all host
cores: whole RK3 steps of the same workload restricted to 33 of its 257
wall-normal planes per timed step, with one full-size substep beside it as a
calibration of the per-point rate (kept out of the value).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mpoint-steps/s on 1 B200: FP64 vs mixed at ≤1e-6 rel err; adjoint/forward cost"
UNIT = "Mpoint-steps/s"
WORKLOAD = "Re_tau=180 channel 256x257x256, 3 velocities + 2 scalars (Pr 0.71, 1.0), dt=5e-4"
SAMPLE_NY = 33


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            pk = json.load(fh)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clocks and clock-event (throttle) reasons of this process's GPU,
    read through NVML every 10 ms on a background thread (nvidia-smi every
    200 ms when NVML is unavailable).  Read-only: no setting is changed."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.thread = None
        self.samples = []
        self.reasons = set()

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            pr = torch.cuda.get_device_properties(self.index)
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        import threading
        try:
            nv, h = self._nvml_handle()
        except Exception:
            nv = None
        if nv is None:
            try:
                self.proc = subprocess.Popen(
                    ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200",
                     "-i", str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            except Exception:
                self.proc = None
            return
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        self.stop_flag = threading.Event()

        def run():
            while not self.stop_flag.is_set():
                try:
                    self.samples.append(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.reasons.update(k for k, b in bits.items() if r & b)
                except Exception:
                    pass
                self.stop_flag.wait(0.01)
        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()

    def stop(self):
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                    "sm_max_mhz": self.max_mhz, "samples": len(self.samples),
                    "reasons": sorted(self.reasons), "source": "nvml, 10 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, mx, reasons = [], [], set()
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(self.NAMES, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "samples": len(sm),
                "reasons": sorted(reasons), "source": "nvidia-smi, 200 ms"}


# ---------------------------------------------------------------------------
def kernel_bytes(p, nf, mixed):
    """Algorithmic HBM bytes per launch of each step kernel: every input read
    once and every output written once (state FP64; step scratch FP32 in mixed
    precision).  Fourier fields hold (Nkx+1)(2Nkz+1) modes per plane, x-spectral
    fields (Nkx+1)Nz, physical fields NxNz."""
    cs = 8 if mixed else 16
    rs = cs // 2
    nyp2, ny = p.ny + 2, p.ny
    four = (p.nx // 3 + 1) * (2 * (p.nz // 3) + 1)
    xsp = (p.nx // 3 + 1) * p.nz
    phys = p.nx * p.nz
    nth = p.n_th
    return {
        "z_inverse": nf * nyp2 * (four * 16 + xsp * cs),
        "x_inverse_c2r": nf * nyp2 * (xsp * cs + phys * rs),
        "products_x_forward_r2c": nf * nyp2 * phys * rs + 2 * nf * ny * xsp * cs,
        # mixed: the u1 equation's NL is FP64 and takes the mean epilogue
        # (state u1, u3, u2 on two planes read; 8 more bytes written per mode)
        "z_forward_combine": 2 * nf * ny * xsp * cs + nf * ny * four * cs
                             + (ny * four * (4 * 16 + 8) if mixed else 0),
        # field solves: every field in and its solved value out, the pressure
        # in (once), NL in, cf in on 2 of 3 substeps and out on 2 of 3
        "column_solve": nyp2 * four * (2 * nf * 16 + 16 + nf * cs + (16 - cs if mixed else 0)
                                       + 2 * (2.0 / 3.0) * nf * 16),
        # projection: solved u1, u2, u3 and p in, projected u1, u2, u3 and p out
        "projection": nyp2 * four * (4 * 16 * 2),
    }


def setup_channel(p, gy, fields, precision):
    from diablo3_test_b200 import _lib
    from diablo3_test_b200.channel import Channel
    ch = Channel(p, gy)
    ch.set_precision(precision)
    ids = [("u1", _lib.U1), ("u2", _lib.U2), ("u3", _lib.U3)] + \
        [(f"th{n}", _lib.TH + n) for n in range(p.n_th)]
    for name, fid in ids:
        ch.upload(fid, np.ascontiguousarray(fields[name]), _lib.LAYOUT_PHYSICAL)
    ch.pre_first_step()
    ch.synchronize()
    return ch


def state_sig(ch, scalars=False):
    from diablo3_test_b200 import _lib
    p = ch.params
    out = {}
    ids = [("u1", _lib.U1), ("u2", _lib.U2), ("u3", _lib.U3)]
    if scalars:
        ids += [(f"th{n}", _lib.TH + n) for n in range(p.n_th)]
    for name, fid in ids:
        c = ch.download(fid).view(np.complex128)
        out[name] = c[:, :2 * (p.nz // 3) + 1, :p.nx // 2].copy()
    return out


def accuracy_report(sm, sd, p, gy):
    """Mixed (sm) against FP64 (sd) states: per-field relative L2 error of the
    significant Fourier modes, relative error of the mean wall shear dU1/dy at
    both walls, and relative L2 error of the streamwise energy spectrum
    E(kx) = sum over y and kz of |u_hat|^2 per velocity component."""
    from diablo3_test_b200.grid import metrics
    _, _, dy, _ = metrics(gy)
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    out = {"field_rel_l2": {k: rel(sm[k], sd[k]) for k in sm}}
    ny = p.ny
    shear = {}
    for tag, (ja, jb, jd) in {"lower": (1, 2, 2), "upper": (ny - 1, ny, ny)}.items():
        tm = (sm["u1"][jb, 0, 0].real - sm["u1"][ja, 0, 0].real) / dy[jd]
        td = (sd["u1"][jb, 0, 0].real - sd["u1"][ja, 0, 0].real) / dy[jd]
        shear[tag] = float(abs(tm - td) / abs(td))
    out["wall_shear_rel"] = shear
    spec = {}
    for k in ("u1", "u2", "u3"):
        w = np.full(sm[k].shape[2], 2.0)
        w[0] = 1.0
        em = (np.abs(sm[k][1:ny + 1]) ** 2).sum(axis=(0, 1)) * w
        ed = (np.abs(sd[k][1:ny + 1]) ** 2).sum(axis=(0, 1)) * w
        spec[k] = rel(em, ed)
    out["spectrum_kx_rel_l2"] = spec
    vel = max(out["field_rel_l2"][k] for k in ("u1", "u2", "u3"))
    out["max_velocity_rel_l2"] = vel
    out["within_1e-6"] = bool(vel <= 1e-6)
    return out


def max_over_ranks(vals, torch, dist=None, device="cuda"):
    """Element-wise maximum of per-rank timings over every rank (identity
    without a process group).  `device` is where the reduction tensor lives:
    "cuda" for NCCL, "cpu" for gloo."""
    if dist is None:
        return [float(v) for v in vals]
    t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def aggregate_rate(points_per_step, world, steps, ms):
    """Whole-job Mpoint-steps/s: every rank advanced its own replica of
    `points_per_step` points `steps` times in `ms` milliseconds (the maximum
    over ranks)."""
    return points_per_step * world * steps / (ms * 1e-3) / 1e6


def timed_steps(ch, torch, stream, k, dist=None):
    """K steps between barriers, CUDA events on the context's stream."""
    ch.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ch.step(k)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    return e0.elapsed_time(e1)


def _oracle_slice(ny, cores):
    import dataclasses
    from diablo3_test_b200 import ics
    from diablo3_test_b200.grid import create_grid, TANH_ENDS_SYMMETRIC
    from tests.helpers import setup_oracle
    p, _ = ics.config_c2()
    p = dataclasses.replace(p, ny=ny)
    gy, _ = create_grid(p.ny, 2.0, TANH_ENDS_SYMMETRIC, 2.0)
    fields = ics.log_law_turbulent(p, gy)
    return p, setup_oracle(p, gy, fields, workers=cores)


def cpu_baseline(steps=1, warmup=1):
    """The CPU oracle on all host cores: whole RK3 steps (three substeps) of
    the benchmark workload restricted to SAMPLE_NY wall-normal planes."""
    cores = os.cpu_count() or 1
    p, o = _oracle_slice(SAMPLE_NY, cores)
    times = []
    for s in range(warmup + steps):
        t = time.perf_counter()
        o.step(1)
        dt = time.perf_counter() - t
        if s >= warmup:
            times.append(dt)
    t_step = sum(times) / len(times)
    value = p.nx * p.ny * p.nz / t_step / 1e6
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"oracle RK3 steps (3 substeps each) of the workload on {SAMPLE_NY} of 257 "
                      f"planes (256x{SAMPLE_NY}x256), mean of {steps} after {warmup} warm-up",
            "s_per_step": t_step}


def cpu_calibration(cores):
    """One RK substep of the full 257-plane workload on the CPU oracle, to
    check the slice's per-point rate (not part of any reported value)."""
    p, o = _oracle_slice(257, cores)
    o.rk_step = 1
    t = time.perf_counter()
    o.rk_chan_1()
    dt = time.perf_counter() - t
    return {"full_planes_substep_s": dt,
            "full_planes_rate": p.nx * p.ny * p.nz / 3.0 / dt / 1e6, "unit": UNIT}


def read_traffic():
    """Per-launch DRAM bytes of each profiled kernel from the committed ncu
    summaries (profiles/*.md lines 'traffic_per_launch <kernel> <bytes>
    <how the figure was obtained>'): {kernel: (bytes, source)}.  These are
    captured offline, not in this run."""
    out = {}
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return out
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith(".md"):
            continue
        for line in open(os.path.join(pdir, fn)):
            m = re.match(r"\s*traffic_per_launch\s+(\S+)\s+(\d+)\s*(.*)$", line)
            if m:
                out[m.group(1)] = (int(m.group(2)), f"profiles/{fn}: {m.group(3).strip()}")
    return out


def ensemble_bench(torch, k, warmup=3):
    """The uneven-grid ensemble (48 mixed-precision members cycling four grid
    sizes, 23.5 M points per ensemble step): one graph launch per step for all
    members, in the persistent mode (every member's column step of a substep
    in one persistent launch per rows-per-lane class) and in the branches mode
    (each member's whole step on its own graph branch), against the same
    members run one at a time on one stream.  All are timed with CUDA events;
    the final states are compared."""
    from diablo3_test_b200 import _lib
    from diablo3_test_b200 import ics
    from diablo3_test_b200.channel import Ensemble
    from diablo3_test_b200.config import MIXED
    cfg = ics.config_c5()
    pts = sum(p.nx * p.ny * p.nz for p, _, _ in cfg)
    ens_m = [setup_channel(p, gy, f, MIXED) for p, gy, f in cfg]
    one_m = [setup_channel(p, gy, f, MIXED) for p, gy, f in cfg]
    s1 = torch.cuda.Stream()
    for ch in one_m:
        ch.set_stream(s1.cuda_stream)
    ens = Ensemble(ens_m)
    ens.step(warmup)
    for ch in one_m:
        ch.step(warmup)
    ens.synchronize()
    torch.cuda.synchronize()
    es = torch.cuda.ExternalStream(ens.stream_handle)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def time_graph():
        e0.record(es)
        ens.step(k)
        e1.record(es)
        ens.synchronize()
        return e0.elapsed_time(e1)

    ms_default = time_graph()
    # autotuned tiles per member size, scored on this graph (states restored)
    tiles = {}
    for (p, _, _), t in zip(cfg, ens.autotune(5)):
        tiles[f"{p.nx}x{p.ny}x{p.nz}"] = list(t)
    ens.step(1)
    ens.synchronize()
    mode = ens.mode
    ms_graph = time_graph()
    # the other mode on the same members
    ens.mode = _lib.ENSEMBLE_BRANCHES if mode == _lib.ENSEMBLE_PERSISTENT else _lib.ENSEMBLE_PERSISTENT
    ens.step(1)
    ens.synchronize()
    ms_other = time_graph()
    other_mode = ens.mode
    ens.mode = mode
    # the members run singly catch up to the same step count, then are timed
    for ch in one_m:
        ch.step(2 * k + 2)
    torch.cuda.synchronize()
    e0.record(s1)
    for ch in one_m:
        ch.step(k)
    e1.record(s1)
    torch.cuda.synchronize()
    ms_one = e0.elapsed_time(e1)
    diff = 0.0
    for a, b in zip(ens_m, one_m):
        sa, sb = state_sig(a), state_sig(b)
        for key in sa:
            nb = np.linalg.norm(sb[key])
            diff = max(diff, float(np.linalg.norm(sa[key] - sb[key]) / (nb if nb > 0 else 1.0)))
    launches = sum(ch.kernel_launches() for ch in ens_m)
    ens.close()
    for ch in ens_m + one_m:
        ch.close()
    return {"workload": "48 independent channels, (Nx,Ny,Nz) cycling (32,33,32), (64,65,64), (96,97,64), "
                        "(128,65,128); Re ~ U[500,3000] (seed 5); mixed precision; dt=1e-3",
            "points_per_step": pts, "steps": k, "warmup": warmup,
            "value": pts * k / (ms_graph * 1e-3) / 1e6, "unit": UNIT, "ms_per_step": ms_graph / k,
            "singly": {"value": pts * k / (ms_one * 1e-3) / 1e6, "ms_per_step": ms_one / k},
            "speedup_vs_singly": ms_one / ms_graph,
            "default_tiles": {"value": pts * k / (ms_default * 1e-3) / 1e6, "ms_per_step": ms_default / k},
            "tiles": tiles,
            "tiles_meaning": "z inverse sequences/block, x inverse rows/block, x forward rows/block, "
                             "z forward sequences/block (0 = default), tuned per size on the graph",
            "max_rel_diff_vs_singly": diff,
            "mode": "persistent" if mode == _lib.ENSEMBLE_PERSISTENT else "branches",
            "other_mode": {"mode": "persistent" if other_mode == _lib.ENSEMBLE_PERSISTENT else "branches",
                           "value": pts * k / (ms_other * 1e-3) / 1e6, "ms_per_step": ms_other / k},
            "graph": "one CUDA graph launch per ensemble step; persistent: per substep the members' "
                     "transforms on parallel branches, then one k_column_step_ens launch per "
                     "rows-per-lane class walking the member table; branches: one branch per member",
            "kernel_launches_total": launches}


def c1_bench(torch, k=200, warmup=5, cpu_steps=2):
    """Config 1, plain FP64 DNS at the reference test-case shape (64 x 193 x 32,
    one scalar, Re 1000, dt 1e-3, laminar parabola plus seeded 1% noise):
    k steps on the GPU (CUDA events on the context's stream), and the CPU
    oracle on all host cores for cpu_steps whole steps after one warm-up."""
    from diablo3_test_b200 import ics
    from diablo3_test_b200.config import FP64
    from tests.helpers import setup_oracle
    p, gy = ics.config_c1()
    fields = ics.laminar_dns(p, gy, seed=1, amp=0.01)
    ch = setup_channel(p, gy, fields, FP64)
    stream = torch.cuda.Stream()
    ch.set_stream(stream.cuda_stream)
    ch.step(warmup)
    ms = timed_steps(ch, torch, stream, k)
    ch.close()
    pts = p.nx * p.ny * p.nz
    cores = os.cpu_count() or 1
    o = setup_oracle(p, gy, fields, workers=cores)
    o.step(1)
    t = time.perf_counter()
    o.step(cpu_steps)
    t_cpu = (time.perf_counter() - t) / cpu_steps
    return {"workload": "plain FP64 DNS 64x193x32, one scalar, Re 1000, Pr 1, dt 1e-3, tanh 1.8, "
                        "laminar parabola + 1% seeded noise",
            "steps": k, "value": pts * k / (ms * 1e-3) / 1e6, "unit": UNIT, "ms_per_step": ms / k,
            "cpu_oracle": {"value": pts / t_cpu / 1e6, "unit": UNIT, "cores": cores, "s_per_step": t_cpu,
                           "steps": cpu_steps, "kind": "port"}}


def les_bench(torch, k=5, warmup=2):
    """LES workload (config 3: dynamic Smagorinsky, 128 x 129 x 128, Re_tau =
    1000, k^-5/3 random-phase start, LES active from step 1) in FP64 and in
    mixed precision (LES model and its transforms FP32; solves, projection and
    state FP64), with the mixed-vs-FP64 error of the velocity and of nu_t after
    the same steps; the reference's constant-Smagorinsky model beside it.
    CUDA events on the context's stream."""
    from diablo3_test_b200 import ics
    from diablo3_test_b200.config import FP64, MIXED
    out = {}
    for name, model in (("dynamic_smagorinsky", 2), ("constant_smagorinsky", 1)):
        p, gy, fields = ics.config_c3(model)
        pts = p.nx * p.ny * p.nz
        res = {}
        chans = {}
        for prec_name, prec in (("fp64", FP64), ("mixed", MIXED)):
            ch = setup_channel(p, gy, fields, prec)
            s = torch.cuda.Stream()
            ch.set_stream(s.cuda_stream)
            ch.step(warmup)
            ms = timed_steps(ch, torch, s, k)
            nt = ch.download_nu_t()[:, :p.nz, :p.nx].copy()
            res[prec_name] = {"value": pts * k / (ms * 1e-3) / 1e6, "unit": UNIT, "ms_per_step": ms / k,
                              "nu_t_max": float(nt.max()), "nu_t_mean": float(nt.mean()),
                              "nu_t_positive_fraction": float((nt > 0).mean()),
                              "finite": bool(ch.check_finite())}
            chans[prec_name] = (ch, nt)
        sd, sm = state_sig(chans["fp64"][0]), state_sig(chans["mixed"][0])
        rel = lambda x, y: float(np.linalg.norm(x - y) / np.linalg.norm(y))
        res["mixed_vs_fp64"] = {"steps": warmup + k, "velocity_rel_l2": {q: rel(sm[q], sd[q]) for q in sd},
                                "nu_t_rel_l2": rel(chans["mixed"][1], chans["fp64"][1])}
        res["mixed_speedup_vs_fp64"] = res["fp64"]["ms_per_step"] / res["mixed"]["ms_per_step"]
        for ch, _ in chans.values():
            ch.close()
        out[name] = res
    out["workload"] = ("Re_tau=1000 channel LES 128x129x128, tanh 2.2, dt=2e-4, log-law mean + "
                       "k^-5/3 random-phase fluctuations (seed 3), LES active from step 1")
    return out


def adjoint_bench(torch, nsteps=50, every=10):
    """Cost of the hand-written discrete adjoint on the 64 x 97 x 64,
    Re = 2000 velocity-only case: 50 FP64 steps forward (diablo_step) against
    the checkpointed forward (diablo_adjoint_record, a checkpoint every 10
    steps) and the backward sweep (diablo_adjoint_run: segment recompute +
    adjoint substeps), all timed with CUDA events on the context's stream."""
    from diablo3_test_b200 import ics, _lib
    from diablo3_test_b200.config import FP64
    p, gy, fields = ics.config_c4()
    ch = setup_channel(p, gy, fields, FP64)
    s = torch.cuda.Stream()
    ch.set_stream(s.cuda_stream)
    ids = (_lib.U1, _lib.U2, _lib.U3, _lib.P)
    x0 = [torch.tensor(ch.download(f), device="cuda") for f in ids]
    lam = [torch.zeros_like(x0[0]) for _ in ids]

    def timed(fn):
        for f, x in zip(ids, x0):
            ch.upload(f, x, _lib.LAYOUT_FOURIER)
        ch.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        fn()
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1)

    timed(lambda: ch.step(nsteps))                     # warm-up
    t_fwd = min(timed(lambda: ch.step(nsteps)) for _ in range(3))
    timed(lambda: ch.adjoint_record(nsteps, every))    # first call allocates the checkpoints
    # one untimed backward sweep first: it allocates the adjoint work arrays
    # and loads the adjoint kernels
    for l in lam:
        l.normal_()
    ch.adjoint_run([l.clone() for l in lam])
    t_rec = timed(lambda: ch.adjoint_record(nsteps, every))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    ch.adjoint_run(lam)
    e1.record(s)
    e1.synchronize()
    t_run = e0.elapsed_time(e1)
    ch.close()
    return {"workload": "64x97x64, Re=2000, velocities only, FP64, 50 steps, dt=1e-3, checkpoints every 10",
            "forward_ms": t_fwd, "record_ms": t_rec, "adjoint_run_ms": t_run,
            "adjoint_over_forward": t_run / t_fwd,
            "record_plus_adjoint_over_forward": (t_rec + t_run) / t_fwd,
            "note": "adjoint_run includes recomputing every segment but the last from its checkpoint (the record keeps the last segment's substep inputs)"}


def stats_bench(ch, p, peak, reps=5):
    """save_stats_chan on the workload state (diablo_stats): the device time of
    the statistics kernels (Parseval plane sums, compute_BPE and y* binning
    histograms, per-launch events; the FP64 inverse transforms that feed the
    histograms are not in it) and the whole call (wall values, transforms,
    kernels, partial sums to the host, the host finish)."""
    import time
    ch.stats()   # first call allocates the partial-sum and field buffers
    ch.set_profiling(True)
    t0 = time.perf_counter()
    for _ in range(reps):
        ch.stats()
    wall_ms = (time.perf_counter() - t0) / reps * 1e3
    ms, n = ch.kernel_times().get("other", (0.0, 0))
    ch.set_profiling(False)
    nkx1, nk2 = p.nx // 3 + 1, 2 * (p.nz // 3) + 1
    return {"kernels_device_ms": ms / reps, "launches_per_call": n / reps, "call_ms": wall_ms,
            "parseval_alg_bytes": (3 + p.n_th) * 16 * (p.ny + 2) * nkx1 * nk2,
            "note": "x-homogeneous save_stats_chan with compute_BPE and the y* binning"}


def e2e_round_trip(ch, torch, k, stream, dist=None, world=1):
    """End to end through the C ABI with pinned host buffers: each step
    uploads the state (u1, u2, u3, p, scalars) from the host in the reference
    layout, advances one step and downloads the state into the same host
    arrays.  The value is diablo_step_host, which overlaps each field's
    download with the next step's upload of the field before it (the two link
    directions at once); beside it, the same round trip as separate
    diablo_upload_state / diablo_step / diablo_download_state calls.  The work
    is ordered on the context's stream, so CUDA events on that stream bracket
    the copies and the steps; under torchrun every rank runs its replica
    between barriers and the time is the maximum over ranks."""
    from diablo3_test_b200 import _lib
    p = ch.params
    ids = [_lib.U1, _lib.U2, _lib.U3, _lib.P] + [_lib.TH + n for n in range(p.n_th)]
    shape = (p.ny + 2, p.nz + 2, p.nx + 2)
    bufs = [torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy() for _ in ids]
    for b, fid in zip(bufs, ids):
        ch.download(fid, out=b)
    ch.synchronize()
    # bytes a field moves each way: its rows k <= 2Nkz of every plane, with
    # each row's pad entry (Nx/2 + 1 complex)
    rows = (p.ny + 2) * (2 * (p.nz // 3) + 1)
    h2d = d2h = rows * (p.nx // 2 + 1) * 16
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def timed(fn):
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        ch.synchronize()
        return max_over_ranks([e0.elapsed_time(e1)], torch, dist)[0]

    ch.step_host(bufs, 1)          # warm-up: the copy streams and staging arrays

    def per_call():
        for _ in range(k):
            for b, fid in zip(bufs, ids):
                ch.upload(fid, b)
            ch.step(1)
            for b, fid in zip(bufs, ids):
                ch.download(fid, out=b)

    ms = timed(lambda: ch.step_host(bufs, k))
    ms_calls = timed(per_call)
    if dist is not None:
        dist.barrier()
    pts = p.nx * p.ny * p.nz
    return {"value": aggregate_rate(pts, world, k, ms), "unit": UNIT,
            "h2d_bytes_per_step": h2d * len(ids) * world,
            "d2h_bytes_per_step": d2h * len(ids) * world, "ms_per_step": ms / k,
            "path": f"diablo_step_host (host, pinned; {len(ids)} fields up and down per step, "
                    "each field's download overlapping the next step's upload of the field before it)",
            "separate_calls": {"value": aggregate_rate(pts, world, k, ms_calls), "ms_per_step": ms_calls / k,
                               "path": f"diablo_upload_state x{len(ids)} + diablo_step + "
                                       f"diablo_download_state x{len(ids)}"},
            "timing": "CUDA events on the context's stream, max over ranks"}


def profile_other(args, torch):
    """Profiling runs (no JSON line), for launch lists and ncu sections, at
    --grid: the adjoint with the adjoint workload's parameters (FP64;
    diablo_adjoint_record over --steps steps, a checkpoint every step, then
    diablo_adjoint_run; with --adjoint-scalars N, N scalars with buoyancy and
    background gradients), the statistics (diablo_stats --steps times) on the
    Re_tau = 180 workload's state, and the 48-member ensemble (--steps
    ensemble steps in its default mode)."""
    import dataclasses
    from diablo3_test_b200 import ics, _lib
    from diablo3_test_b200.config import FP64, MIXED, ChannelParams
    from diablo3_test_b200.grid import create_grid, TANH_ENDS_SYMMETRIC
    if args.profile_ensemble:
        from diablo3_test_b200.channel import Ensemble
        members = [setup_channel(p, gy, f, MIXED) for p, gy, f in ics.config_c5()]
        ens = Ensemble(members)
        ens.step(args.warmup)
        ens.synchronize()
        t0 = time.perf_counter()
        ens.step(args.steps)
        ens.synchronize()
        print(f"profiling run ensemble (mode {ens.mode}): {time.perf_counter() - t0:.3f} s")
        ens.close()
        for ch in members:
            ch.close()
        return
    if args.profile_adjoint:
        p, gy, _ = ics.config_c4()      # velocity-only FP64 parameters
        if args.adjoint_scalars:
            kw = {f.name: getattr(p, f.name) for f in dataclasses.fields(p)
                  if f.name not in ("n_th", "pr", "ri", "th_bc_ymin", "th_bc_ymax", "th_bc_ymin_c1",
                                    "th_bc_ymax_c1", "dthdx", "dthdz", "filter_th", "filter_int")}
            kw.update(grav_y=0.5, grav_x=0.2)
            p = ChannelParams.with_scalars(args.adjoint_scalars, **kw)
    else:
        p, gy = ics.config_c2()
    if args.grid:
        p = dataclasses.replace(p, nx=args.grid[0], ny=args.grid[1], nz=args.grid[2])
        gy, _ = create_grid(p.ny, 2.0, TANH_ENDS_SYMMETRIC, 1.8 if args.profile_adjoint else 2.0)
    fields = ics.laminar_dns(p, gy, seed=4, amp=0.05) if args.profile_adjoint else ics.log_law_turbulent(p, gy)
    ch = setup_channel(p, gy, fields, FP64 if args.profile_adjoint else MIXED)
    stream = torch.cuda.Stream()
    ch.set_stream(stream.cuda_stream)
    ch.step(args.warmup)
    t0 = time.perf_counter()
    if args.profile_adjoint:
        ids = (_lib.U1, _lib.U2, _lib.U3, _lib.P) + tuple(_lib.TH + n for n in range(p.n_th))
        lam = [torch.randn(ch.shape_phys, dtype=torch.float64, device="cuda") for _ in ids]
        ch.adjoint_record(args.steps, 1)
        ch.adjoint_run(lam)
    else:
        for _ in range(args.steps):
            ch.stats()
    ch.synchronize()
    what = "adjoint" if args.profile_adjoint else "statistics"
    print(f"profiling run {what} {p.nx}x{p.ny}x{p.nz}: {time.perf_counter() - t0:.3f} s")
    ch.close()


# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    from diablo3_test_b200 import ics, _lib
    from diablo3_test_b200.config import FP64, MIXED
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)
    torch.cuda.init()
    if args.profile_adjoint or args.profile_stats or args.profile_ensemble:
        profile_other(args, torch)
        return
    if args.profile_les:
        # profiling run of the dynamic-LES workload (128 x 129 x 128), no JSON line
        p, gy, fields = ics.config_c3(2)
        ch = setup_channel(p, gy, fields, FP64 if args.precision == "fp64" else MIXED)
        stream = torch.cuda.Stream()
        ch.set_stream(stream.cuda_stream)
        ch.step(args.warmup)
        ms = timed_steps(ch, torch, stream, args.steps)
        print(f"profiling run LES 128x129x128 dynamic: {ms / max(args.steps, 1):.3f} ms/step")
        ch.close()
        return
    p, gy = ics.config_c2()
    if args.grid:
        import dataclasses
        from diablo3_test_b200.grid import create_grid, TANH_ENDS_SYMMETRIC
        p = dataclasses.replace(p, nx=args.grid[0], ny=args.grid[1], nz=args.grid[2])
        gy, _ = create_grid(p.ny, 2.0, TANH_ENDS_SYMMETRIC, 2.0)
    fields = ics.log_law_turbulent(p, gy)
    nf = 3 + p.n_th
    pts = p.nx * p.ny * p.nz
    stream = torch.cuda.Stream()
    if args.grid or args.precision != "both":
        # profiling run: one precision, no JSON line
        ch = setup_channel(p, gy, fields, MIXED if args.precision != "fp64" else FP64)
        ch.set_stream(stream.cuda_stream)
        ch.step(args.warmup)
        ms = timed_steps(ch, torch, stream, args.steps)
        print(f"profiling run {p.nx}x{p.ny}x{p.nz} {args.precision}: {ms / max(args.steps, 1):.3f} ms/step")
        ch.close()
        return
    chm = setup_channel(p, gy, fields, MIXED)
    chd = setup_channel(p, gy, fields, FP64)
    tiles = {}
    for name, ch in (("mixed", chm), ("fp64", chd)):
        ch.set_stream(stream.cuda_stream)
        if not args.no_autotune:
            tiles[name] = list(ch.autotune())
    # warm-up
    chm.step(args.warmup)
    chd.step(args.warmup)
    sampler = ClockSampler(local)
    sampler.start()
    chm.set_profiling(True)
    l0 = chm.kernel_launches()
    ms_mixed = timed_steps(chm, torch, stream, args.steps, dist)
    launches = chm.kernel_launches() - l0
    ktimes = chm.kernel_times()
    chm.set_profiling(False)
    # the FP64 step is timed the same way (per-kernel events on), so the two
    # carry the same event overhead
    chd.set_profiling(True)
    ms_fp64 = timed_steps(chd, torch, stream, args.steps, dist)
    ktimes64 = chd.kernel_times()
    chd.set_profiling(False)
    clocks = sampler.stop()
    ms_mixed, ms_fp64 = max_over_ranks([ms_mixed, ms_fp64], torch, dist)
    # mixed vs FP64 after the same W+K steps from the same state
    sm, sd = state_sig(chm), state_sig(chd)
    err = {k: float(np.linalg.norm(sm[k] - sd[k]) / np.linalg.norm(sd[k])) for k in sm}
    # both continued (untimed) to the workload's 100 steps
    acc = None
    done = args.warmup + args.steps
    if args.acc_steps > done:
        chm.step(args.acc_steps - done)
        chd.step(args.acc_steps - done)
        acc = accuracy_report(state_sig(chm, True), state_sig(chd, True), p, gy)
        acc["steps"] = args.acc_steps
    e2e = None
    if not args.no_e2e:
        e2e = e2e_round_trip(chm, torch, max(2, min(args.steps, 5)), stream, dist, world)
    if rank != 0:
        chm.close()
        chd.close()
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return
    peak, peak_kind = _peaks()
    kb = kernel_bytes(p, nf, mixed=True)
    per_kernel = {}
    for name, (ms, n) in ktimes.items():
        if n and name in kb:
            avg = ms / n
            per_kernel[name] = {"launches": n, "avg_ms": avg, "share": ms / max(ms_mixed, 1e-9),
                                "alg_bytes": kb[name], "achieved_gbs": kb[name] / (avg * 1e-3) / 1e9}
    dom = max(per_kernel, key=lambda k: per_kernel[k]["avg_ms"] * per_kernel[k]["launches"])
    traffic, traffic_src = read_traffic().get(dom, (None, None))
    achieved = per_kernel[dom]["achieved_gbs"]
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": f"{peak_kind} hbm_gbs",
                "traffic_source": traffic_src}
    # whole-step roofline against the 3*(8NF+9)*s bytes-per-point-step model
    alg64 = 3 * (8 * nf + 9) * 8
    value = aggregate_rate(pts, world, args.steps, ms_mixed)
    v64 = aggregate_rate(pts, world, args.steps, ms_fp64)
    # the mixed step as a whole: algorithmic bytes of every timed kernel launch
    # per step over the step's own time
    mixed_bytes = sum(v["launches"] * v["alg_bytes"] for v in per_kernel.values()) / args.steps
    # The 4-pass model counts only state arrays, which are FP64 in both
    # precisions here (mixed precision keeps its FP32 arrays inside the
    # transforms), so the model's bytes per point-step are the same for both.
    step_roof = {"model_bytes_per_point_step_fp64": alg64,
                 "fp64_frac": alg64 * pts / (ms_fp64 / args.steps * 1e-3) / 1e9 / peak,
                 "mixed_model_frac": alg64 * pts / (ms_mixed / args.steps * 1e-3) / 1e9 / peak,
                 "mixed_alg_bytes_per_step": mixed_bytes,
                 "mixed_achieved_gbs": mixed_bytes / (ms_mixed / args.steps * 1e-3) / 1e9,
                 "mixed_frac": mixed_bytes / (ms_mixed / args.steps * 1e-3) / 1e9 / peak}
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_mixed / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 FFT/nonlinear + f64 solves/state (mixed)",
        "data": "synthetic (seeded log-law mean + 10% perturbations, projected)",
        "config": {"workload": WORKLOAD, "grid": [p.nx, p.ny, p.nz], "n_th": p.n_th,
                   "precision": "mixed", "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "state (~1 GB FP64 Fourier + scratch) larger than the 126 MB L2; no flush"},
        "fp64": {"value": v64, "unit": UNIT, "ms_per_step": ms_fp64 / args.steps,
                 "kernels_avg_ms": {k: ms / n for k, (ms, n) in ktimes64.items() if n},
                 "dtype": "f64"},
        "mixed_speedup_vs_fp64": ms_fp64 / ms_mixed,
        "mixed_vs_fp64_rel_err": err,
        "rel_err_steps": args.warmup + args.steps,
        "mixed_accuracy": acc,
        "roofline": roofline,
        "step_roofline": step_roof,
        "kernels": per_kernel,
        "gpu_launches": launches,
        "tiles": tiles,
        "clocks": clocks,
    }
    if e2e is not None:
        out["e2e"] = e2e
    out["stats"] = stats_bench(chm, p, peak)
    chm.close()
    chd.close()
    if world == 1 and not args.no_c1:
        out["c1"] = c1_bench(torch)
    if world == 1 and not args.no_les:
        out["les"] = les_bench(torch)
    if world == 1 and not args.no_adjoint:
        out["adjoint"] = adjoint_bench(torch)
    if world == 1 and args.ensemble_steps > 0:
        out["ensemble"] = ensemble_bench(torch, args.ensemble_steps)
    if world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    print(json.dumps(out))


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cb = cpu_baseline(steps=args.steps, warmup=args.warmup)
    cal = cpu_calibration(cb["cores"])
    out = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": cb["s_per_step"] * 1e3, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "impl": "reference",
           "data": "synthetic (seeded log-law mean + 10% perturbations, projected)",
           "config": {"workload": WORKLOAD + f"; timed on its 256x{SAMPLE_NY}x256 slice "
                                             f"({SAMPLE_NY} of 257 wall-normal planes), whole RK3 steps",
                      "precision": "fp64",
                      "sample": f"256x{SAMPLE_NY}x256 slice of the workload, one whole RK3 step per timed step"},
           "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
           "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "calibration": dict(cal, note="one full 257-plane substep, outside the timed steps and the value"),
           "note": "reference Fortran (gfortran+MPI+FFTW+HDF5+toml-f) cannot be built on this image; "
                   "the CPU restatement of its step (oracle/) is timed instead"}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint-cost section")
    ap.add_argument("--no-les", action="store_true", help="skip the LES section")
    ap.add_argument("--no-c1", action="store_true", help="skip the 64x193x32 FP64 DNS section")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default transform tiles")
    ap.add_argument("--ensemble-steps", type=int, default=20,
                    help="timed steps of the 48-member ensemble section (0: skip)")
    ap.add_argument("--acc-steps", type=int, default=100,
                    help="steps after which mixed and FP64 states are compared (untimed)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grid", type=int, nargs=3, metavar=("NX", "NY", "NZ"), default=None,
                    help="profiling: run a smaller grid of the same workload (no JSON contract)")
    ap.add_argument("--precision", choices=["both", "mixed", "fp64"], default="both",
                    help="profiling: run one precision only")
    ap.add_argument("--profile-les", action="store_true",
                    help="profiling: time the dynamic-LES workload instead (mixed unless --precision fp64)")
    ap.add_argument("--profile-adjoint", action="store_true",
                    help="profiling: record and run the adjoint on the --grid workload (velocities, FP64)")
    ap.add_argument("--profile-ensemble", action="store_true",
                    help="profiling: --steps steps of the 48-member ensemble")
    ap.add_argument("--adjoint-scalars", type=int, default=0,
                    help="profiling: scalars in the --profile-adjoint case")
    ap.add_argument("--profile-stats", action="store_true",
                    help="profiling: save_stats_chan on the --grid workload state")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
