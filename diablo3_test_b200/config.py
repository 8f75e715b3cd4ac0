"""Run parameters of one channel, mirroring the reference's ``parameters`` module.

The fields are the ones ``rk_chan_1`` and its callees read
(``for/parameters.f90:22-82``), under the reference's own names, plus the
grid sizes that the reference bakes in at compile time (``grid_def``:
``Nx, Ny, Nz, N_th``).  ``ChannelParams.to_c()`` packs them into the
``diablo_params`` struct declared in ``include/diablo_gpu.h``.

Velocity boundary-condition names follow the reference's internal variables:
``u_bc_*`` is u1 (streamwise), ``v_bc_*`` is u2 (wall-normal) and ``w_bc_*``
is u3 (spanwise), as used by ``apply_BC_1/2/3_*`` (``for/channel.f90:1545-1792``).
``read_input_toml`` reproduces the reference's label swap for TOML input,
where the file's ``V_BC_*`` keys feed ``w_BC_*`` and ``W_BC_*`` feed ``v_BC_*``
(``for/parameters.f90:371-382``).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field, fields
from typing import List

MAX_TH = 8  # scalars a context supports; DIABLO_MAX_TH in include/diablo_gpu.h

# precision modes (DIABLO_FP64 / DIABLO_MIXED)
FP64 = 0
MIXED = 1

# LES model types handled by les_chan (for/les.f90:94-850); 2 = dynamic
# Smagorinsky has no reference implementation (for/les.f90:272-277).
LES_NONE = 0
LES_SMAGORINSKY = 1
LES_DYNAMIC_SMAGORINSKY = 2
LES_AMD_ROZEMA = 4
LES_AMD_VERSTAPPEN = 5


@dataclass
class ChannelParams:
    nx: int
    ny: int
    nz: int
    n_th: int = 0
    lx: float = 2 * math.pi
    ly: float = 2.0
    lz: float = math.pi
    re: float = 1000.0
    nu_v_scale: float = 1.0
    beta: float = 1.0
    ro: float = math.inf
    delta: float = 1.0
    grav_x: float = 0.0
    grav_y: float = 0.0
    grav_z: float = 0.0
    delta_t: float = 1e-3
    f_type: int = 0
    ubulk0: float = 0.0
    px0: float = 0.0
    omega0: float = 0.0
    amp_omega0: float = 0.0
    force_start: float = 0.0
    u_bc_ymin: int = 0
    v_bc_ymin: int = 0
    w_bc_ymin: int = 0
    u_bc_ymax: int = 0
    v_bc_ymax: int = 0
    w_bc_ymax: int = 0
    u_bc_ymin_c1: float = 0.0
    v_bc_ymin_c1: float = 0.0
    w_bc_ymin_c1: float = 0.0
    u_bc_ymax_c1: float = 0.0
    v_bc_ymax_c1: float = 0.0
    w_bc_ymax_c1: float = 0.0
    pr: List[float] = field(default_factory=list)
    ri: List[float] = field(default_factory=list)
    th_bc_ymin: List[int] = field(default_factory=list)
    th_bc_ymax: List[int] = field(default_factory=list)
    th_bc_ymin_c1: List[float] = field(default_factory=list)
    th_bc_ymax_c1: List[float] = field(default_factory=list)
    dthdx: List[float] = field(default_factory=list)
    dthdz: List[float] = field(default_factory=list)
    use_les: bool = False
    les_model_type: int = LES_NONE
    create_new_flow: bool = True
    variable_dt: bool = False
    cfl: float = 0.5
    update_dt: int = 1
    max_dt: float = 1.0
    precision: int = FP64
    flavor: str = "Basic"
    filter_th: List[bool] = field(default_factory=list)
    filter_int: List[int] = field(default_factory=list)

    # ------------------------------------------------------------------
    # quantities derived exactly as the reference derives them
    @property
    def nu(self) -> float:
        """``nu = 1/Re`` (for/parameters.f90:101)."""
        return 1.0 / self.re

    @property
    def ro_inv(self) -> float:
        """``Ro_inv = 1/Ro`` (for/parameters.f90:102); Ro = inf gives 0."""
        return 0.0 if math.isinf(self.ro) else 1.0 / self.ro

    @property
    def nxp(self) -> int:
        """``Nxp = Nx/(2*NprocZ)`` at one rank (for/domain.f90:13)."""
        return self.nx // 2

    @property
    def nkx(self) -> int:
        return self.nx // 3  # for/domain.f90:18

    @property
    def nkz(self) -> int:
        return self.nz // 3  # for/domain.f90:19

    @property
    def nyp(self) -> int:
        return self.ny  # Nyp = (Ny-1)/NprocY + 1 at NprocY = 1 (for/domain.f90:12)

    @property
    def jstart(self) -> int:
        """Row range of u1/u3 updates at one y-rank (for/domain.f90:284-292)."""
        return 1 if self.u_bc_ymin == 1 else 2

    @property
    def jend(self) -> int:
        return self.ny  # rankY == 0 branch, for/domain.f90:285

    def jstart_th(self, n: int) -> int:
        return 1 if self.th_bc_ymin[n] == 1 else 2  # for/domain.f90:294-303

    def jend_th(self, n: int) -> int:
        return self.ny

    def validate(self) -> None:
        if self.nx % 2 or self.nx < 8:
            raise ValueError("nx must be even and >= 8")
        if self.nz < 4:
            raise ValueError("nz must be >= 4")
        if self.ny < 4:
            raise ValueError("ny must be >= 4")
        if not 0 <= self.n_th <= MAX_TH:
            raise ValueError(f"n_th must be in [0, {MAX_TH}]")
        for name in ("pr", "ri", "th_bc_ymin", "th_bc_ymax", "th_bc_ymin_c1",
                     "th_bc_ymax_c1", "dthdx", "dthdz"):
            if len(getattr(self, name)) != self.n_th:
                raise ValueError(f"{name} must have n_th={self.n_th} entries")

    @classmethod
    def with_scalars(cls, n_th: int, **kw) -> "ChannelParams":
        """Build a parameter set with ``n_th`` scalars and per-scalar defaults
        (Pr = 1, Ri = 0, zero-flux Neumann walls, no background gradient)."""
        per = dict(pr=[1.0] * n_th, ri=[0.0] * n_th, th_bc_ymin=[1] * n_th,
                   th_bc_ymax=[1] * n_th, th_bc_ymin_c1=[0.0] * n_th,
                   th_bc_ymax_c1=[0.0] * n_th, dthdx=[0.0] * n_th,
                   dthdz=[0.0] * n_th, filter_th=[False] * n_th, filter_int=[1] * n_th)
        for k in list(per):
            if k in kw:
                per[k] = list(kw.pop(k))
        p = cls(n_th=n_th, **per, **kw)
        p.validate()
        return p

    # ------------------------------------------------------------------
    def to_c(self) -> "CParams":
        self.validate()
        c = CParams()
        for f in fields(self):
            v = getattr(self, f.name)
            if f.name == "flavor":
                c.flavor_front = 1 if v == "Front" else 0
                continue
            if isinstance(v, list):
                arr = getattr(c, f.name)
                for i, x in enumerate(v):
                    arr[i] = x
            else:
                setattr(c, f.name, v)
        c.struct_size = ctypes.sizeof(CParams)
        return c


_TH = ctypes.c_double * MAX_TH
_THI = ctypes.c_int * MAX_TH


class CParams(ctypes.Structure):
    """ctypes image of ``diablo_params`` (include/diablo_gpu.h)."""
    _fields_ = [
        ("struct_size", ctypes.c_int),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("n_th", ctypes.c_int),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("re", ctypes.c_double), ("nu_v_scale", ctypes.c_double),
        ("beta", ctypes.c_double), ("ro", ctypes.c_double),
        ("delta", ctypes.c_double),
        ("grav_x", ctypes.c_double), ("grav_y", ctypes.c_double),
        ("grav_z", ctypes.c_double),
        ("delta_t", ctypes.c_double),
        ("f_type", ctypes.c_int),
        ("ubulk0", ctypes.c_double), ("px0", ctypes.c_double),
        ("omega0", ctypes.c_double), ("amp_omega0", ctypes.c_double),
        ("force_start", ctypes.c_double),
        ("u_bc_ymin", ctypes.c_int), ("v_bc_ymin", ctypes.c_int),
        ("w_bc_ymin", ctypes.c_int), ("u_bc_ymax", ctypes.c_int),
        ("v_bc_ymax", ctypes.c_int), ("w_bc_ymax", ctypes.c_int),
        ("u_bc_ymin_c1", ctypes.c_double), ("v_bc_ymin_c1", ctypes.c_double),
        ("w_bc_ymin_c1", ctypes.c_double), ("u_bc_ymax_c1", ctypes.c_double),
        ("v_bc_ymax_c1", ctypes.c_double), ("w_bc_ymax_c1", ctypes.c_double),
        ("pr", _TH), ("ri", _TH),
        ("th_bc_ymin", _THI), ("th_bc_ymax", _THI),
        ("th_bc_ymin_c1", _TH), ("th_bc_ymax_c1", _TH),
        ("dthdx", _TH), ("dthdz", _TH),
        ("use_les", ctypes.c_int), ("les_model_type", ctypes.c_int),
        ("create_new_flow", ctypes.c_int),
        ("variable_dt", ctypes.c_int), ("cfl", ctypes.c_double),
        ("update_dt", ctypes.c_int), ("max_dt", ctypes.c_double),
        ("precision", ctypes.c_int),
        ("flavor_front", ctypes.c_int),
        ("filter_th", ctypes.c_int * MAX_TH), ("filter_int", ctypes.c_int * MAX_TH),
    ]


def read_input_toml(path: str, nx: int, ny: int, nz: int, n_th: int) -> ChannelParams:
    """Read a reference ``input.toml`` (VERSION 3.5) into ``ChannelParams``.

    Follows ``read_input_toml`` (for/parameters.f90:287-403) including the
    V/W velocity-BC label swap (:371-382) and ``set_parameters``'s
    front-IC adjustments of w_BC and dTHdX (for/parameters.f90:241-281).
    """
    import tomllib
    with open(path, "rb") as fh:
        t = tomllib.load(fh)
    if t.get("VERSION") != "3.5":
        raise ValueError("Wrong input version")  # for/parameters.f90:307-308
    sch, phy, ts = t["SCHEME"], t["PHYSICAL"], t["TIMESTEPPING"]
    ic, frc, vb = t["INITIAL_CONDITIONS"], t["FORCING"], t["VELOCITY_BCS"]
    scal = t.get("SCALARS", [])
    if len(scal) != n_th:
        raise ValueError(f"{n_th} scalars defined but {len(scal)} scalars found in input.toml")
    g = phy["GRAV"]
    p = ChannelParams(
        nx=nx, ny=ny, nz=nz, n_th=n_th,
        lx=float(phy["LX"]), ly=float(phy["LY"]), lz=float(phy["LZ"]),
        re=float(phy["RE"]), nu_v_scale=float(phy["NU_V_SCALE"]),
        beta=float(sch["BETA"]), ro=float(phy["RO"]), delta=float(phy["DELTA"]),
        grav_x=float(g[0]), grav_y=float(g[1]), grav_z=float(g[2]),
        delta_t=float(ts["DELTA_T"]), variable_dt=bool(ts["VARIABLE_DT"]),
        cfl=float(ts["CFL"]), update_dt=int(ts["UPDATE_DT"]),
        f_type=int(frc["F_TYPE"]), ubulk0=float(frc["UBULK0"]),
        px0=float(frc["PX0"]), omega0=float(frc["OMEGA0"]),
        amp_omega0=float(frc["AMP_OMEGA0"]), force_start=float(frc["FORCE_START"]),
        u_bc_ymin=int(vb["U_BC_YMIN"]), u_bc_ymin_c1=float(vb["U_BC_YMIN_C1"]),
        w_bc_ymin=int(vb["V_BC_YMIN"]), w_bc_ymin_c1=float(vb["V_BC_YMIN_C1"]),
        v_bc_ymin=int(vb["W_BC_YMIN"]), v_bc_ymin_c1=float(vb["W_BC_YMIN_C1"]),
        u_bc_ymax=int(vb["U_BC_YMAX"]), u_bc_ymax_c1=float(vb["U_BC_YMAX_C1"]),
        w_bc_ymax=int(vb["V_BC_YMAX"]), w_bc_ymax_c1=float(vb["V_BC_YMAX_C1"]),
        v_bc_ymax=int(vb["W_BC_YMAX"]), v_bc_ymax_c1=float(vb["W_BC_YMAX_C1"]),
        pr=[float(s["PR"]) for s in scal], ri=[float(s["RI"]) for s in scal],
        th_bc_ymin=[int(s["TH_BC_YMIN"]) for s in scal],
        th_bc_ymax=[int(s["TH_BC_YMAX"]) for s in scal],
        th_bc_ymin_c1=[float(s["TH_BC_YMIN_C1"]) for s in scal],
        th_bc_ymax_c1=[float(s["TH_BC_YMAX_C1"]) for s in scal],
        dthdx=[0.0] * n_th, dthdz=[0.0] * n_th,
        use_les=bool(sch["USE_LES"]), les_model_type=int(sch["LES_MODEL_TYPE"]),
        create_new_flow=bool(ic["CREATE_NEW_FLOW"]),
        flavor=str(sch.get("FLAVOUR", "Basic")) or "Basic",
        filter_th=[bool(s.get("FILTER_TH", False)) for s in scal],
        filter_int=[int(s.get("FILTER_INT", 1)) for s in scal],
    )
    ic_type = int(ic["IC_TYPE"])
    if n_th:
        if ic_type in (4, 5):
            if p.w_bc_ymin == 1:
                p.w_bc_ymin_c1 -= 1.0
            if p.w_bc_ymax == 1:
                p.w_bc_ymax_c1 -= 1.0
            p.dthdx[0] = p.ro_inv / p.delta
        elif ic_type in (6, 7, 8):
            if p.w_bc_ymin == 1:
                p.w_bc_ymin_c1 -= 2.0 * p.delta / p.lx
            if p.w_bc_ymax == 1:
                p.w_bc_ymax_c1 -= 2.0 * p.delta / p.lx
            p.dthdx[0] = 2.0 / p.lx * p.ro_inv
    p.validate()
    return p
