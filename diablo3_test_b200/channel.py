"""Python front end of libdiablo_gpu, mirroring the reference's step surface.

``Channel`` owns one device context.  Its methods keep the reference's
routine names and argument meaning:

* ``fft_xz_to_fourier(v, vv)`` / ``fft_xz_to_physical(vv, v)``
  (``for/fft.f90:247,319``) take arrays in the reference layout; passing the
  same array twice reproduces the reference's in-place aliasing.
* ``rk_chan_1(rk_step)`` (``for/channel.f90:10``), ``step(n)``
  (``for/diablo.f90:104-108``), ``pre_first_step`` (``for/advance.f90:17``)
  and ``apply_bc_post`` (``for/boundary.f90:824-855``).

Arrays are numpy (host) arrays in the reference's Fortran memory order: a
physical field has numpy shape ``(Ny+2, Nz+2, Nx+2)`` float64 (index
``[j, k, i]``) and a Fourier field the complex128 view of the same bytes,
shape ``(Ny+2, Nz+2, Nx/2+1)``.  Torch CUDA tensors of those shapes may be
passed instead; their device pointers are used directly.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .config import ChannelParams


def _ptr(a):
    """Data pointer of a contiguous numpy array or torch tensor."""
    if isinstance(a, np.ndarray):
        if not a.flags.c_contiguous:
            raise ValueError("array must be C-contiguous (the reference's Fortran order)")
        return a.ctypes.data_as(ctypes.c_void_p)
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return ctypes.c_void_p(a.data_ptr())
    raise TypeError(f"unsupported array type {type(a)!r}")


# mean.h5 dataset each statistic is written to (for/statistics.f90:176-273,
# 490-520, 702, 1066, 1268, 2116; for/les.f90:1074): the reference's y is
# the wall-normal direction internally but its files label it z, so v and w
# swap.  Scalar profiles take the scalar number (1-based, two digits).
MEAN_H5_NAMES = {
    "ume": "ume", "vme": "wme", "wme": "vme", "mke": "mke", "urms": "urms", "vrms": "wrms",
    "wrms": "vrms", "uv": "uw", "uw": "uv", "wv": "wv", "uu_dudx": "uu_dudx",
    "vv_dvdy": "ww_dwdz", "wu_dwdx": "vu_dvdx", "vu_dvdx": "wu_dwdx", "uv_dudy": "uw_dudz",
    "wv_dwdy": "vw_dvdz", "dudy": "dudz", "dwdy": "dvdz", "cp": "cp", "shear": "shear",
    "omega_x": "omega_x", "omega_y": "omega_z", "omega_z": "omega_y", "epsilon": "epsilon",
    "epsilon_m": "epsilon_m", "nu_sgs": "nu_sgs", "eps_sgs2": "eps_sgs2",
    "thme": "thme{:02d}", "dthdy": "dthdz{:02d}", "thrms": "thrms{:02d}", "thv": "thw{:02d}",
    "thv_m": "thw{:02d}_m", "pe_diss": "pe_diss{:02d}", "kappa_sgs": "kappa_sgs", "spectrum": "FTx_uu",
    "u1y_left_b": "u1z_x0", "time": "time", "bpe": "BPE", "th1_pdf": "th1PDF",
    "th1_bin": "th1bin", "zstar": "<name>_zstar",
}


class Channel:
    def __init__(self, params: ChannelParams, gy):
        self.params = params
        self.lib = _lib.load()
        self._c = params.to_c()
        gy = np.ascontiguousarray(gy, dtype=np.float64)
        if gy.size != params.ny + 1:
            raise ValueError(f"gy must hold Ny+1 = {params.ny + 1} points")
        self._gy = gy
        st = ctypes.c_int(0)
        self.ctx = self.lib.diablo_create(ctypes.byref(self._c), gy.ctypes.data_as(ctypes.c_void_p),
                                          ctypes.byref(st))
        if not self.ctx:
            raise _lib.DiabloError(st.value, "diablo_create")
        self.shape_phys = (params.ny + 2, params.nz + 2, params.nx + 2)
        self.shape_four = (params.ny + 2, params.nz + 2, params.nx // 2 + 1)

    # -- lifetime ------------------------------------------------------
    def close(self):
        if getattr(self, "ctx", None):
            self.lib.diablo_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- arrays --------------------------------------------------------
    def new_field(self) -> np.ndarray:
        """A zeroed reference-layout buffer (physical view)."""
        return np.zeros(self.shape_phys, dtype=np.float64)

    def upload(self, field: int, buf, layout: int = _lib.LAYOUT_FOURIER):
        _lib.check(self.lib.diablo_upload_state(self.ctx, field, _ptr(buf), layout), "upload_state")

    def download(self, field: int, layout: int = _lib.LAYOUT_FOURIER, out=None) -> np.ndarray:
        if out is None:
            out = self.new_field()
        _lib.check(self.lib.diablo_download_state(self.ctx, field, _ptr(out), layout), "download_state")
        return out

    def tiles_in_use(self):
        """The context's current transform tiles (0 = default)."""
        t = (ctypes.c_int * 4)()
        _lib.check(self.lib.diablo_tiles(self.ctx, t), "tiles")
        return tuple(t)

    def autotune(self):
        """Time the transform tile shapes for this grid and precision and keep
        the fastest; returns (z inverse S, x inverse KT, x forward KT, z forward S)."""
        t = (ctypes.c_int * 4)()
        _lib.check(self.lib.diablo_autotune(self.ctx, t), "autotune")
        return tuple(t)

    def step_host(self, bufs, nsteps: int = 1):
        """nsteps host round trips (diablo_step_host): upload the state from
        the host arrays bufs (u1, u2, u3, p, then one per scalar; reference
        Fourier layout, pinned for the full link rate), step, download into
        the same arrays; field downloads overlap the next uploads."""
        ns = 4 + self.params.n_th
        if len(bufs) != ns:
            raise ValueError(f"{ns} host arrays: u1, u2, u3, p and one per scalar")
        arr = (ctypes.c_void_p * ns)(*[_ptr(b) for b in bufs])
        _lib.check(self.lib.diablo_step_host(self.ctx, arr, nsteps), "step_host")

    def adjoint_record(self, nsteps: int, every: int):
        """Advance nsteps steps, keeping checkpoints every `every` steps for
        adjoint_run (DNS with velocities and scalars in FP64)."""
        _lib.check(self.lib.diablo_adjoint_record(self.ctx, nsteps, every), "adjoint_record")

    def adjoint_run(self, lam):
        """lam: 4 + N_th reference-layout Fourier arrays (numpy or torch)
        holding dJ/d(u1, u2, u3, p, th_0, ..) of the recorded final state;
        overwritten with dJ/d of the recorded initial state."""
        ns = 4 + self.params.n_th
        if len(lam) != ns:
            raise ValueError(f"{ns} arrays: u1, u2, u3, p and one per scalar")
        arr = (ctypes.c_void_p * ns)(*[_ptr(a) for a in lam])
        _lib.check(self.lib.diablo_adjoint_run(self.ctx, arr), "adjoint_run")

    def download_nu_t(self, out=None) -> np.ndarray:
        """Eddy viscosity of the last LES substep, reference physical layout."""
        if out is None:
            out = self.new_field()
        _lib.check(self.lib.diablo_download_nu_t(self.ctx, _ptr(out)), "download_nu_t")
        return out

    def stats(self, homogeneous_x: bool = True) -> dict:
        """Plane statistics of save_stats_chan (for/statistics.f90:44-712);
        ``homogeneous_x`` is the reference's homogeneousX (False for IC types
        5-8).  Applies the wall values to the state first, as the reference
        does.  Returns ``{"profiles": {name: (Ny,)},
        "th": [{name: (Ny,)} per scalar], "spectrum": (Nx/2,), "scalars":
        {name: float}}`` with the reference's internal names (MEAN_H5_NAMES
        gives the dataset each one is written to); with scalars also
        "th1_pdf" and "th1_bin" (Nx,) of compute_BPE, scalars["bpe"], and
        "zstar": {shear2, thw, chi, epsilon, TKE, KE: (Nx,)} bin means."""
        p = self.params
        n = self.lib.diablo_stats_size(self.ctx)
        if n < 0:
            _lib.check(n, "stats_size")
        out = np.zeros(n)
        _lib.check(self.lib.diablo_stats(self.ctx, 1 if homogeneous_x else 0,
                                         out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n), "stats")
        ny, npf, ntp = p.ny, len(_lib.STAT_PROFILES), len(_lib.STAT_TH_PROFILES)
        prof = {k: out[q * ny:(q + 1) * ny].copy() for q, k in enumerate(_lib.STAT_PROFILES)}
        th = []
        for t in range(p.n_th):
            b = (npf + t * ntp) * ny
            th.append({k: out[b + r * ny:b + (r + 1) * ny].copy() for r, k in enumerate(_lib.STAT_TH_PROFILES)})
        b = (npf + p.n_th * ntp) * ny
        spec = out[b:b + p.nx // 2].copy()
        b += p.nx // 2
        res = {"profiles": prof, "th": th, "spectrum": spec}
        if p.n_th > 0:   # compute_BPE's PDF of th_1 and its lower bin edges
            res["th1_pdf"] = out[b:b + p.nx].copy()
            res["th1_bin"] = out[b + p.nx:b + 2 * p.nx].copy()
            b += 2 * p.nx
            # Bin_Ystar_and_Write's bin means on the same th_1 bins
            res["zstar"] = {k: out[b + q * p.nx:b + (q + 1) * p.nx].copy()
                            for q, k in enumerate(_lib.STAT_ZSTAR)}
            b += len(_lib.STAT_ZSTAR) * p.nx
        res["scalars"] = {k: float(v) for k, v in zip(_lib.STAT_SCALARS, out[b:])}
        if p.n_th == 0:
            del res["scalars"]["bpe"]
        return res

    def les_eps_sgs1(self) -> np.ndarray:
        """eps_sgs1 of les_chan (for/les.f90:924-1068), (Ny,) on GY points:
        requested by :meth:`stats` on an LES channel and formed at the first
        substep of the next step, as the reference's flag_save_LES does.
        Raises DiabloError (DIABLO_ERR_STATE) when no step has run since the
        request."""
        out = np.zeros(self.params.ny)
        _lib.check(self.lib.diablo_les_eps_sgs1(self.ctx, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                out.size), "les_eps_sgs1")
        return out

    # -- reference surface ---------------------------------------------
    def fft_xz_to_fourier(self, v, vv):
        _lib.check(self.lib.diablo_fft_xz_to_fourier(self.ctx, _ptr(v), _ptr(vv)), "fft_xz_to_fourier")

    def fft_xz_to_physical(self, vv, v):
        _lib.check(self.lib.diablo_fft_xz_to_physical(self.ctx, _ptr(vv), _ptr(v)), "fft_xz_to_physical")

    def rk_chan_1(self, rk_step: int):
        _lib.check(self.lib.diablo_rk_substep(self.ctx, rk_step), "rk_substep")

    def step(self, nsteps: int = 1):
        _lib.check(self.lib.diablo_step(self.ctx, nsteps), "step")

    def pre_first_step(self, compute_pressure: bool = False):
        _lib.check(self.lib.diablo_pre_first_step(self.ctx, int(compute_pressure)), "pre_first_step")

    def apply_bc_post(self):
        _lib.check(self.lib.diablo_apply_bc_post(self.ctx), "apply_bc_post")

    def set_precision(self, precision: int):
        _lib.check(self.lib.diablo_set_precision(self.ctx, precision), "set_precision")

    def synchronize(self):
        _lib.check(self.lib.diablo_synchronize(self.ctx), "synchronize")

    def check_finite(self) -> bool:
        st = self.lib.diablo_check_finite(self.ctx)
        if st == _lib.ERR_NONFINITE:
            return False
        _lib.check(st, "check_finite")
        return True

    @property
    def time(self):
        t = ctypes.c_double(0)
        n = ctypes.c_int(0)
        dt = ctypes.c_double(0)
        _lib.check(self.lib.diablo_get_time(self.ctx, ctypes.byref(t), ctypes.byref(n), ctypes.byref(dt)),
                   "get_time")
        return t.value, n.value, dt.value

    def set_time(self, time: float, time_step: int, delta_t: float):
        _lib.check(self.lib.diablo_set_time(self.ctx, time, time_step, delta_t), "set_time")

    def kernel_launches(self) -> int:
        return int(self.lib.diablo_kernel_launches(self.ctx))

    def set_profiling(self, enable: bool):
        _lib.check(self.lib.diablo_set_profiling(self.ctx, int(enable)), "set_profiling")

    def kernel_times(self) -> dict:
        """{kernel name: (total device ms, launches)} since profiling was enabled."""
        out = {}
        for s in range(self.lib.diablo_kernel_slots()):
            ms = ctypes.c_double(0)
            n = ctypes.c_longlong(0)
            _lib.check(self.lib.diablo_kernel_times(self.ctx, s, ctypes.byref(ms), ctypes.byref(n)),
                       "kernel_times")
            out[self.lib.diablo_kernel_name(s).decode()] = (ms.value, n.value)
        return out

    def set_stream(self, stream_handle: int):
        """Order the context's work on an existing cudaStream_t (0 = own stream)."""
        _lib.check(self.lib.diablo_set_stream(self.ctx, ctypes.c_void_p(stream_handle or None)),
                   "set_stream")


class Ensemble:
    """Independent channels (any mix of grids, parameters and precisions)
    stepped together: one CUDA graph launch per step for all members
    (``diablo_ensemble_*`` of the C ABI).  In the persistent mode (the
    default when every member qualifies) each substep's column steps of all
    members run in one persistent launch per rows-per-lane class after the
    members' transforms, which run on parallel branches; in the branches mode
    each member's whole step is one branch.  The members stay usable on their
    own and must outlive the ensemble."""

    def __init__(self, members, autotune: bool = False):
        self.lib = _lib.load()
        self.members = list(members)
        # tile shapes per member size (cached across members of one size)
        self.tiles = [m.autotune() for m in self.members] if autotune else None
        arr = (ctypes.c_void_p * len(self.members))(*[m.ctx for m in self.members])
        st = ctypes.c_int(0)
        self.e = self.lib.diablo_ensemble_create(arr, len(self.members), ctypes.byref(st))
        _lib.check(st.value, "ensemble_create")

    def step(self, nsteps: int = 1):
        _lib.check(self.lib.diablo_ensemble_step(self.e, nsteps), "ensemble_step")

    def synchronize(self):
        _lib.check(self.lib.diablo_ensemble_synchronize(self.e), "ensemble_synchronize")

    @property
    def mode(self) -> int:
        """_lib.ENSEMBLE_PERSISTENT or _lib.ENSEMBLE_BRANCHES."""
        return self.lib.diablo_ensemble_mode(self.e)

    @mode.setter
    def mode(self, mode: int):
        _lib.check(self.lib.diablo_ensemble_set_mode(self.e, mode), "ensemble_set_mode")

    def autotune(self, steps_per_trial: int = 5):
        """Tune each member size's transform tiles on the ensemble's own graph
        (the members' states are restored); returns the tiles per member."""
        _lib.check(self.lib.diablo_ensemble_autotune(self.e, steps_per_trial), "ensemble_autotune")
        return [tuple(m.tiles_in_use()) for m in self.members]

    @property
    def stream_handle(self) -> int:
        """cudaStream_t the ensemble's graphs run on (for device timing)."""
        return int(self.lib.diablo_ensemble_stream(self.e) or 0)

    def close(self):
        if self.e:
            self.lib.diablo_ensemble_destroy(self.e)
            self.e = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
