"""Host-side particle state in the reference's in-memory layout.

``HostState`` holds what the reference's ``DEM`` object keeps between
``readbin`` and ``startTime`` (``src/sphere.h:30-95``): array-of-structs
``Float4`` rows of four doubles per particle (``src/datatypes.h:17-33``), the
contact bookkeeping of ``NC`` = 32 slots per particle, bonds and walls.  It is
the layout the C-ABI (``include/sphk.h``) uploads and downloads, so no
repacking happens at the library boundary.

``from_spherebin`` performs the initialisation of ``DEM::DEM`` +
``allocateGlobalDeviceMemory`` + ``transferToGlobalDeviceMemory``
(``src/sphere.cpp:16-77``, ``src/device.cu:233-324,394-488``): ``vel0 := vel``
and ``angvel0 := angvel`` (``device.cu:413-414,423-424``), zero ``acc`` and
``angacc`` (``device.cu:242-248``), every contact slot empty (``np``,
``device.cu:293-297``) with zero history, and each wall's half-step velocity
taken from its velocity (``device.cu:461-464``).  ``to_spherebin`` is the
inverse used before ``writebin``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .spherebin import Spherebin

NC = 32
MAXWALLS = 6

PARAM_NAMES = ("k_n", "k_t", "k_r", "gamma_n", "gamma_t", "gamma_r", "mu_s", "mu_d", "mu_r",
               "gamma_wn", "gamma_wt", "mu_ws", "mu_wd", "rho", "kappa", "db", "V_b",
               "lambda_bar", "sigma_b", "tau_b", "devs_A", "devs_f")


@dataclass
class SceneConfig:
    """Static scene description: grid, time step, physical parameters."""
    np: int
    nw: int
    nb0: int
    num: np.ndarray
    periodic: int
    contactmodel: int
    dt: float
    origo: np.ndarray
    L: np.ndarray
    g: np.ndarray
    params: dict
    wmode: np.ndarray

    @property
    def ncells(self) -> int:
        return int(self.num[0]) * int(self.num[1]) * int(self.num[2])


@dataclass
class HostState:
    """Dynamic state, reference host layout (all C-contiguous)."""
    x: np.ndarray          # (np, 4) x, y, z, radius
    xysum: np.ndarray      # (np, 2)
    vel: np.ndarray        # (np, 4) vx, vy, vz, fixvel
    vel0: np.ndarray       # (np, 4)
    acc: np.ndarray        # (np, 4)
    force: np.ndarray      # (np, 4)
    angpos: np.ndarray     # (np, 4)
    angvel: np.ndarray     # (np, 4)
    angvel0: np.ndarray    # (np, 4)
    angacc: np.ndarray     # (np, 4)
    torque: np.ndarray     # (np, 4)
    es_dot: np.ndarray     # (np,)
    es: np.ndarray
    ev_dot: np.ndarray
    ev: np.ndarray
    p: np.ndarray
    contacts: np.ndarray   # (np, NC) uint32, np = empty
    distmod: np.ndarray    # (np, NC, 4)
    delta_t: np.ndarray    # (np, NC, 4)
    bonds: np.ndarray      # (nb0, 2) uint32
    bonds_delta: np.ndarray  # (nb0, 4) tangential xyz, normal w
    bonds_omega: np.ndarray  # (nb0, 4)
    walls_nx: np.ndarray   # (nw, 4) normal xyz, position w
    walls_mvfd: np.ndarray  # (nw, 4) mass, velocity, force, deviatoric stress
    walls_vel0: np.ndarray  # (nw,)
    t_current: float = 0.0
    extra: dict = field(default_factory=dict)

    def copy(self) -> "HostState":
        kw = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self.__dict__.items()}
        kw["extra"] = dict(self.extra)
        return HostState(**kw)


def _c(a, dtype=np.float64):
    # always a fresh array: a HostState must never alias its Spherebin
    return np.array(a, dtype=dtype, copy=True, order="C")


def config_from_spherebin(sb: Spherebin) -> SceneConfig:
    params = {k: float(getattr(sb, k)) for k in PARAM_NAMES if k not in ("devs_A", "devs_f")}
    params["devs_A"] = float(sb.w_devs_A)
    params["devs_f"] = float(sb.w_devs_f)
    wmode = np.zeros(MAXWALLS, dtype=np.int32)
    wmode[: sb.nw] = np.asarray(sb.wmode, dtype=np.int32)
    return SceneConfig(np=int(sb.np), nw=int(sb.nw), nb0=int(sb.nb0),
                       num=_c(sb.num, np.uint32), periodic=int(sb.periodic),
                       contactmodel=int(sb.contactmodel), dt=float(sb.time_dt),
                       origo=_c(sb.origo), L=_c(sb.L), g=_c(sb.g), params=params, wmode=wmode)


def state_from_spherebin(sb: Spherebin) -> HostState:
    n, nw, nb0 = int(sb.np), int(sb.nw), int(sb.nb0)

    def f4(v3, w=None):
        out = np.zeros((n, 4))
        out[:, :3] = v3
        if w is not None:
            out[:, 3] = w
        return out

    vel = f4(sb.vel, sb.fixvel)
    angvel = f4(sb.angvel)
    walls_nx = np.zeros((nw, 4))
    walls_mvfd = np.zeros((nw, 4))
    if nw:
        walls_nx[:, :3] = sb.w_n
        walls_nx[:, 3] = sb.w_x
        walls_mvfd[:] = np.column_stack([sb.w_m, sb.w_vel, sb.w_force, sb.w_devs])
    bd = np.zeros((nb0, 4))
    bo = np.zeros((nb0, 4))
    if nb0:
        bd[:, :3] = sb.bonds_delta_t
        bd[:, 3] = sb.bonds_delta_n
        bo[:, :3] = sb.bonds_omega_t
        bo[:, 3] = sb.bonds_omega_n
    return HostState(
        x=f4(sb.x, sb.radius), xysum=_c(sb.xysum), vel=vel, vel0=vel.copy(),
        acc=np.zeros((n, 4)), force=f4(sb.force), angpos=f4(sb.angpos), angvel=angvel,
        angvel0=angvel.copy(), angacc=np.zeros((n, 4)), torque=f4(sb.torque),
        es_dot=_c(sb.es_dot), es=_c(sb.es), ev_dot=_c(sb.ev_dot), ev=_c(sb.ev), p=_c(sb.p),
        contacts=np.full((n, NC), n, dtype=np.uint32), distmod=np.zeros((n, NC, 4)),
        delta_t=np.zeros((n, NC, 4)), bonds=_c(sb.bonds, np.uint32).reshape(nb0, 2),
        bonds_delta=bd, bonds_omega=bo, walls_nx=walls_nx, walls_mvfd=walls_mvfd,
        walls_vel0=_c(walls_mvfd[:, 1]) if nw else np.zeros(0), t_current=float(sb.time_current))


def to_spherebin(sb_template: Spherebin, st: HostState) -> Spherebin:
    """A copy of ``sb_template`` carrying the state ``st`` (what
    ``transferFromGlobalDeviceMemory`` + ``writebin`` put on disk)."""
    sb = Spherebin.from_bytes(sb_template.to_bytes(), sid=sb_template.sid)
    sb.x = st.x[:, :3].copy()
    sb.radius = st.x[:, 3].copy()
    sb.xysum = st.xysum.copy()
    sb.vel = st.vel[:, :3].copy()
    sb.fixvel = st.vel[:, 3].copy()
    sb.force = st.force[:, :3].copy()
    sb.angpos = st.angpos[:, :3].copy()
    sb.angvel = st.angvel[:, :3].copy()
    sb.torque = st.torque[:, :3].copy()
    sb.es_dot, sb.es, sb.ev_dot, sb.ev, sb.p = (a.copy() for a in (st.es_dot, st.es, st.ev_dot, st.ev, st.p))
    if sb.nw:
        sb.w_n = st.walls_nx[:, :3].copy()
        sb.w_x = st.walls_nx[:, 3].copy()
        sb.w_m, sb.w_vel, sb.w_force, sb.w_devs = (st.walls_mvfd[:, k].copy() for k in range(4))
    if sb.nb0:
        sb.bonds = st.bonds.copy()
        sb.bonds_delta_t = st.bonds_delta[:, :3].copy()
        sb.bonds_delta_n = st.bonds_delta[:, 3].copy()
        sb.bonds_omega_t = st.bonds_omega[:, :3].copy()
        sb.bonds_omega_n = st.bonds_omega[:, 3].copy()
    sb.time_current = float(st.t_current)
    return sb
