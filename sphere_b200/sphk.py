"""ctypes binding of libsphk (include/sphk.h) and the host-side ``Simulation``.

``Simulation`` is the in-process counterpart of what the reference's ``DEM``
object does between ``readbin`` and ``writebin`` (``src/sphere.h:244-273``):
it owns one device context, uploads a ``HostState`` in the reference's host
layout, runs time steps on the GPU and downloads the state.  There is no
CPU fallback: constructing a ``Simulation`` without the built library or
without a CUDA device raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path

import numpy as np

from .state import NC, HostState, SceneConfig

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libsphk.so"
HEADER = PKG.parent / "include" / "sphk.h"

SPH_OK = 0
ERRORS = {
    -1: "SPH_ERR_CUDA", -2: "SPH_ERR_NC_OVERFLOW", -3: "SPH_ERR_OUT_OF_GRID",
    -4: "SPH_ERR_TIMEOUT", -5: "SPH_ERR_BAD_INPUT", -6: "SPH_ERR_BOND_ALIAS", -7: "SPH_ERR_NOMEM",
    -8: "SPH_ERR_TOO_LARGE", -9: "SPH_ERR_UNSTABLE",
}
OPT_RELAYOUT_EVERY = 1
OPT_GRAPH_STEPS = 2
OPT_PROFILE = 3
OPT_VERLET_SKIN = 4
OPT_BLOCK_SHAPES = 5
OPT_TOPO_SPAN = 6
PHASES = ("cells", "bonds", "topo", "force", "walls", "darcy", "contact")

_dp = C.POINTER(C.c_double)
_up = C.POINTER(C.c_uint32)


class SphConfig(C.Structure):
    _fields_ = [
        ("np", C.c_uint32), ("nw", C.c_uint32), ("nb0", C.c_uint32), ("contactmodel", C.c_uint32),
        ("periodic", C.c_int32), ("num", C.c_uint32 * 3),
        ("origo", C.c_double * 3), ("L", C.c_double * 3), ("dt", C.c_double),
        ("g", C.c_double * 3),
        ("k_n", C.c_double), ("k_t", C.c_double), ("k_r", C.c_double),
        ("gamma_n", C.c_double), ("gamma_t", C.c_double), ("gamma_r", C.c_double),
        ("mu_s", C.c_double), ("mu_d", C.c_double), ("mu_r", C.c_double),
        ("gamma_wn", C.c_double), ("gamma_wt", C.c_double), ("mu_ws", C.c_double),
        ("mu_wd", C.c_double), ("rho", C.c_double), ("kappa", C.c_double), ("db", C.c_double),
        ("V_b", C.c_double), ("lambda_bar", C.c_double), ("sigma_b", C.c_double),
        ("tau_b", C.c_double), ("devs_A", C.c_double), ("devs_f", C.c_double),
        ("wmode", C.c_int32 * 6), ("device", C.c_int32),
    ]


class SphHostState(C.Structure):
    _fields_ = [(n, _dp) for n in ("x", "xysum", "vel", "vel0", "acc", "force", "angpos", "angvel",
                                   "angvel0", "angacc", "torque", "es_dot", "es", "ev_dot", "ev", "p")]
    _fields_ += [("contacts", _up), ("distmod", _dp), ("delta_t", _dp), ("bonds", _up),
                 ("bonds_delta", _dp), ("bonds_omega", _dp), ("walls_nx", _dp), ("walls_mvfd", _dp),
                 ("walls_vel0", _dp), ("t_current", C.c_double)]


class SphDarcyState(C.Structure):
    _fields_ = [(n, _dp) for n in ("H", "H_new", "V", "dH", "K", "T", "Ss", "W", "phi", "dphi")]


class SphRenderOpts(C.Structure):
    _fields_ = [("method", C.c_int32), ("maxval", C.c_float), ("lower_cutoff", C.c_float),
                ("width", C.c_uint32), ("height", C.c_uint32)]


# colour-map methods of the reference's command line (src/main.cpp:97-118)
RENDER_METHODS = {"normal": 0, "pres": 1, "vel": 2, "angvel": 3, "xdisp": 4, "angpos": 5}


class SphStats(C.Structure):
    _fields_ = [("active_contacts", C.c_uint64), ("steps", C.c_uint64),
                ("relayouts", C.c_uint64), ("device_bytes", C.c_uint64),
                ("cell_rebuilds", C.c_uint64)]


class SphError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def exported_symbols():
    """Function names declared in include/sphk.h."""
    return re.findall(r"^\s*(?:int|const char \*)\s*(sph_\w+)\s*\(", HEADER.read_text(), re.M)


def load_library(path: os.PathLike | None = None):
    """Load libsphk.so; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is not built; run `python -m sphere_b200.build`")
    lib = C.CDLL(str(p))
    vp = C.c_void_p
    sig = {
        "sph_version": ([], C.c_int),
        "sph_create": ([C.POINTER(SphConfig), C.POINTER(vp)], C.c_int),
        "sph_batch_create": ([C.POINTER(SphConfig), C.c_uint32, C.POINTER(vp)], C.c_int),
        "sph_set_option": ([vp, C.c_int, C.c_int64], C.c_int),
        "sph_upload": ([vp, C.POINTER(SphHostState)], C.c_int),
        "sph_step": ([vp, C.c_uint64, vp], C.c_int),
        "sph_sync": ([vp], C.c_int),
        "sph_download": ([vp, C.POINTER(SphHostState)], C.c_int),
        "sph_get_contacts": ([vp, _up, _dp, _dp], C.c_int),
        "sph_get_cells": ([vp, _up, _up, _up, _up], C.c_int),
        "sph_get_wall_forces": ([vp, _dp], C.c_int),
        "sph_get_stats": ([vp, C.POINTER(SphStats)], C.c_int),
        "sph_relayout": ([vp], C.c_int),
        "sph_get_profile": ([vp, _dp, C.POINTER(C.c_uint64), C.c_int], C.c_int),
        "sph_last_error": ([vp], C.c_char_p),
        "sph_destroy": ([vp], C.c_int),
        "sph_cell_list_noalloc": ([C.POINTER(SphConfig), vp, vp, vp, vp, vp, vp], C.c_int),
        "sph_diff_begin": ([vp, _dp, C.c_uint32], C.c_int),
        "sph_diff_backward": ([vp, _dp, _dp, _dp, _dp, _dp, _dp], C.c_int),
        "sph_diff_end": ([vp], C.c_int),
        "sph_darcy_init": ([C.POINTER(SphConfig), C.c_double, _dp, C.POINTER(SphDarcyState), _dp],
                           C.c_int),
        "sph_darcy_upload": ([vp, C.c_double, C.POINTER(SphDarcyState)], C.c_int),
        "sph_darcy_download": ([vp, C.POINTER(SphDarcyState)], C.c_int),
        "sph_render": ([vp, C.POINTER(SphRenderOpts), C.POINTER(C.c_uint8)], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    if path is None:
        _lib = lib
    return lib


def make_config(cfg: SceneConfig, device: int = 0) -> SphConfig:
    c = SphConfig()
    c.np, c.nw, c.nb0, c.contactmodel = cfg.np, cfg.nw, cfg.nb0, cfg.contactmodel
    c.periodic = cfg.periodic
    c.num[:] = [int(v) for v in cfg.num]
    c.origo[:] = [float(v) for v in cfg.origo]
    c.L[:] = [float(v) for v in cfg.L]
    c.dt = cfg.dt
    c.g[:] = [float(v) for v in cfg.g]
    for k, v in cfg.params.items():
        setattr(c, k, float(v))
    c.wmode[:] = [int(v) for v in cfg.wmode]
    c.device = int(device)
    return c


def _ptr(a, dtype, keep):
    if a is None:
        return None
    assert a.dtype == dtype and a.flags.c_contiguous, (a.dtype, a.flags.c_contiguous)
    if a.size == 0:
        a = np.zeros(1, dtype)
        keep.append(a)
    return a.ctypes.data_as(_dp if dtype == np.float64 else _up)


def _host_struct(st: HostState, keep) -> SphHostState:
    h = SphHostState()
    for n in ("x", "xysum", "vel", "vel0", "acc", "force", "angpos", "angvel", "angvel0", "angacc",
              "torque", "es_dot", "es", "ev_dot", "ev", "p", "distmod", "delta_t", "bonds_delta",
              "bonds_omega", "walls_nx", "walls_mvfd", "walls_vel0"):
        setattr(h, n, _ptr(getattr(st, n), np.float64, keep))
    h.contacts = _ptr(st.contacts, np.uint32, keep)
    h.bonds = _ptr(st.bonds, np.uint32, keep)
    h.t_current = float(st.t_current)
    return h


def _darcy_struct(state, keep) -> SphDarcyState:
    d = SphDarcyState()
    for name, _ in SphDarcyState._fields_:
        setattr(d, name, _ptr(getattr(state, name), np.float64, keep))
    return d


def darcy_init(cfg: SceneConfig, nu: float, x, state, device: int = 0) -> float:
    """The reference's host-side Darcy initialisation (DEM::initDarcy) into
    `state`: storativity, recharge, porosity from the particle rows `x`
    (np x 4), conductivity and transmissivity.  Returns the stability
    criterion; raises SphError(SPH_ERR_UNSTABLE) above 0.5, where the
    reference exits."""
    lib = load_library()
    keep = []
    c = make_config(cfg, device)
    xa = np.ascontiguousarray(x, dtype=np.float64)
    value = C.c_double(0.0)
    rc = lib.sph_darcy_init(C.byref(c), float(nu), xa.ctypes.data_as(_dp),
                            C.byref(_darcy_struct(state, keep)), C.byref(value))
    if rc != SPH_OK:
        raise SphError(rc, f"Darcy initialisation (stability criterion {value.value:.6g})")
    return float(value.value)


class Simulation:
    """One DEM simulation resident on a GPU."""

    def __init__(self, cfg: SceneConfig, device: int = 0, graph_steps: int | None = None,
                 relayout_every: int | None = None, verlet_skin: float | None = None,
                 block_shapes: int | None = None, topo_span: int | None = None):
        """``verlet_skin``: Verlet-list skin as a fraction of the largest radius
        (default 0.1; 0 sweeps the full stencil every step).  ``block_shapes``:
        0 or 1, the compiled block shapes of the contact kernels to use.
        ``topo_span``: list decisions per thread of the contact search (0:
        chosen from the particle count; 1, 2 or 4)."""
        self.lib = load_library()
        self.cfg = cfg
        self._ctx = C.c_void_p()
        conf = make_config(cfg, device)
        rc = self.lib.sph_create(C.byref(conf), C.byref(self._ctx))
        self._check(rc)
        if graph_steps is not None:
            self._check(self.lib.sph_set_option(self._ctx, OPT_GRAPH_STEPS, int(graph_steps)))
        if relayout_every is not None:
            self._check(self.lib.sph_set_option(self._ctx, OPT_RELAYOUT_EVERY, int(relayout_every)))
        if verlet_skin is not None:
            self._check(self.lib.sph_set_option(self._ctx, OPT_VERLET_SKIN,
                                                int(round(verlet_skin * 1000))))
        if block_shapes is not None:
            self._check(self.lib.sph_set_option(self._ctx, OPT_BLOCK_SHAPES, int(block_shapes)))
        if topo_span is not None:
            self._check(self.lib.sph_set_option(self._ctx, OPT_TOPO_SPAN, int(topo_span)))

    def _check(self, rc):
        if rc != SPH_OK:
            msg = self.lib.sph_last_error(self._ctx) if self._ctx else b""
            raise SphError(rc, (msg or b"").decode())

    def upload(self, st: HostState):
        keep = []
        h = _host_struct(st, keep)
        self._check(self.lib.sph_upload(self._ctx, C.byref(h)))

    def step(self, nsteps: int, stream=None):
        """Enqueue nsteps steps (asynchronous); ``stream`` is a raw cudaStream_t."""
        s = C.c_void_p(stream) if stream else None
        self._check(self.lib.sph_step(self._ctx, int(nsteps), s))

    def sync(self):
        self._check(self.lib.sph_sync(self._ctx))

    def download(self, st: HostState | None = None) -> HostState:
        if st is None:
            st = empty_state(self.cfg)
        keep = []
        h = _host_struct(st, keep)
        self._check(self.lib.sph_download(self._ctx, C.byref(h)))
        st.t_current = h.t_current
        return st

    def contacts(self):
        n = self.cfg.np
        c = np.zeros((n, NC), np.uint32)
        dm = np.zeros((n, NC, 4))
        dt = np.zeros((n, NC, 4))
        self._check(self.lib.sph_get_contacts(self._ctx, c.ctypes.data_as(_up),
                                              dm.ctypes.data_as(_dp), dt.ctypes.data_as(_dp)))
        return c, dm, dt

    def cells(self):
        n, ncell = self.cfg.np, self.cfg.ncells
        cs = np.zeros(n, np.uint32)
        pm = np.zeros(n, np.uint32)
        st = np.zeros(ncell, np.uint32)
        en = np.zeros(ncell, np.uint32)
        self._check(self.lib.sph_get_cells(self._ctx, *(a.ctypes.data_as(_up) for a in (cs, pm, st, en))))
        return cs, pm, st, en

    def wall_forces(self):
        out = np.zeros(self.cfg.np)
        self._check(self.lib.sph_get_wall_forces(self._ctx, out.ctypes.data_as(_dp)))
        return out

    def stats(self) -> dict:
        s = SphStats()
        self._check(self.lib.sph_get_stats(self._ctx, C.byref(s)))
        return {k: int(getattr(s, k)) for k, _ in SphStats._fields_}

    def set_profile(self, on: bool):
        self._check(self.lib.sph_set_option(self._ctx, OPT_PROFILE, 1 if on else 0))

    def profile(self, reset=False) -> dict:
        ms = (C.c_double * len(PHASES))()
        n = C.c_uint64()
        self._check(self.lib.sph_get_profile(self._ctx, ms, C.byref(n), 1 if reset else 0))
        out = {p: float(ms[i]) for i, p in enumerate(PHASES)}
        out["steps"] = int(n.value)
        return out

    def relayout(self):
        self._check(self.lib.sph_relayout(self._ctx))

    # ---- ray tracer (sph_render) -----------------------------------------------
    def render(self, method=0, maxval=1.0e3, lower_cutoff=0.0, width=800, height=800):
        """DEM::render of the current state: a (height, width, 4) uint8 image
        (alpha 0).  `method` is 0-5 or one of RENDER_METHODS' names."""
        if isinstance(method, str):
            method = RENDER_METHODS[method]
        o = SphRenderOpts(int(method), float(maxval), float(lower_cutoff), int(width), int(height))
        img = np.zeros((int(height), int(width), 4), np.uint8)
        self._check(self.lib.sph_render(self._ctx, C.byref(o),
                                        img.ctypes.data_as(C.POINTER(C.c_uint8))))
        return img

    # ---- Darcy flow (sph_darcy_*) ------------------------------------------
    def darcy_upload(self, state, nu: float):
        """Run the Darcy flow in every following step, starting from `state`
        (a ``sphere_b200.darcy.DarcyState``), with dynamic viscosity `nu`."""
        keep = []
        self._check(self.lib.sph_darcy_upload(self._ctx, float(nu), C.byref(_darcy_struct(state, keep))))

    def darcy_download(self, state=None):
        """The Darcy grid after the last step (into `state` when given)."""
        from .darcy import DarcyState
        st = state if state is not None else DarcyState.zeros(self.cfg.num)
        keep = []
        self._check(self.lib.sph_darcy_download(self._ctx, C.byref(_darcy_struct(st, keep))))
        return st

    # ---- differentiable step (sph_diff_*) ----------------------------------
    def diff_begin(self, mu=None, checkpoint_every: int = 100):
        """Switch to the differentiable step: exact FP64 lengths, per-particle
        friction ``mu`` (np values; None: the configuration's mu_s)."""
        m = None if mu is None else np.ascontiguousarray(mu, dtype=np.float64)
        self._diff_keep = m
        ptr = None if m is None else m.ctypes.data_as(_dp)
        self._check(self.lib.sph_diff_begin(self._ctx, ptr, int(checkpoint_every)))

    def diff_backward(self, x_bar=None, v_bar=None) -> dict:
        """Adjoint of every step since diff_begin, seeded with dL/dx and dL/dv
        of the current state ((np, 3) each).  Returns the gradients with
        respect to k_n, k_t, gamma_n, per-particle friction and the starting
        positions and velocities."""
        n = self.cfg.np
        xb = None if x_bar is None else np.ascontiguousarray(x_bar, dtype=np.float64).reshape(n, 3)
        vb = None if v_bar is None else np.ascontiguousarray(v_bar, dtype=np.float64).reshape(n, 3)
        gp = np.zeros(3)
        gmu = np.zeros(n)
        x0 = np.zeros((n, 3))
        v0 = np.zeros((n, 3))
        P = lambda a: None if a is None else a.ctypes.data_as(_dp)
        self._check(self.lib.sph_diff_backward(self._ctx, P(xb), P(vb), P(gp), P(gmu), P(x0), P(v0)))
        return {"k_n": gp[0], "k_t": gp[1], "gamma_n": gp[2], "mu": gmu, "x0": x0, "v0": v0}

    def diff_end(self):
        self._check(self.lib.sph_diff_end(self._ctx))

    def close(self):
        if self._ctx:
            self.lib.sph_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


PARTICLE_FIELDS = ("x", "xysum", "vel", "vel0", "acc", "force", "angpos", "angvel", "angvel0",
                   "angacc", "torque", "es_dot", "es", "ev_dot", "ev", "p", "contacts",
                   "distmod", "delta_t")


def pack_states(states) -> HostState:
    """Scenes end to end, as a batched context takes them: per-particle rows
    of scene 0, then scene 1, ...; contact partners stay scene-local."""
    first = states[0]
    kw = {}
    for f in PARTICLE_FIELDS:
        parts = [getattr(st, f) for st in states]
        kw[f] = None if any(a is None for a in parts) else np.ascontiguousarray(np.concatenate(parts))
    kw.update(bonds=np.zeros((0, 2), np.uint32), bonds_delta=np.zeros((0, 4)),
              bonds_omega=np.zeros((0, 4)), walls_nx=np.zeros((0, 4)), walls_mvfd=np.zeros((0, 4)),
              walls_vel0=np.zeros(0))
    st = HostState(**kw)
    st.t_current = first.t_current
    return st


def split_state(st: HostState, nps) -> list:
    """Inverse of pack_states."""
    out, off = [], 0
    for n in nps:
        kw = {f: (None if getattr(st, f) is None else getattr(st, f)[off:off + n].copy())
              for f in PARTICLE_FIELDS}
        kw.update(bonds=np.zeros((0, 2), np.uint32), bonds_delta=np.zeros((0, 4)),
                  bonds_omega=np.zeros((0, 4)), walls_nx=np.zeros((0, 4)),
                  walls_mvfd=np.zeros((0, 4)), walls_vel0=np.zeros(0))
        part = HostState(**kw)
        part.t_current = st.t_current
        out.append(part)
        off += n
    return out


class BatchSimulation(Simulation):
    """Many independent scenes stepped together by one context
    (sph_batch_create): every kernel launch covers all of them.  Each scene
    keeps its own grid, parameters and time step, and its results are those
    of a Simulation of that scene alone."""

    def __init__(self, cfgs, device: int = 0, graph_steps: int | None = None,
                 relayout_every: int | None = None, verlet_skin: float | None = None,
                 block_shapes: int | None = None, topo_span: int | None = None):
        self.lib = load_library()
        self.cfgs = list(cfgs)
        self.nps = [c.np for c in self.cfgs]
        # the context-wide sizes (cells() reports the context-wide cell list)
        total = SceneConfig(**{**self.cfgs[0].__dict__})
        total.np = sum(self.nps)
        total.num = np.array([sum(int(c.ncells) for c in self.cfgs), 1, 1], np.uint32)
        self.cfg = total
        self._ctx = C.c_void_p()
        arr = (SphConfig * len(self.cfgs))(*[make_config(c, device) for c in self.cfgs])
        self._check(self.lib.sph_batch_create(arr, len(self.cfgs), C.byref(self._ctx)))
        if graph_steps is not None:
            self._check(self.lib.sph_set_option(self._ctx, OPT_GRAPH_STEPS, int(graph_steps)))
        if relayout_every is not None:
            self._check(self.lib.sph_set_option(self._ctx, OPT_RELAYOUT_EVERY, int(relayout_every)))
        if verlet_skin is not None:
            self._check(self.lib.sph_set_option(self._ctx, OPT_VERLET_SKIN,
                                                int(round(verlet_skin * 1000))))
        if block_shapes is not None:
            self._check(self.lib.sph_set_option(self._ctx, OPT_BLOCK_SHAPES, int(block_shapes)))
        if topo_span is not None:
            self._check(self.lib.sph_set_option(self._ctx, OPT_TOPO_SPAN, int(topo_span)))

    def upload(self, states):
        super().upload(pack_states(states))

    def download_all(self) -> list:
        """The state of every scene, in the order they were given."""
        return split_state(self.download(), self.nps)


def empty_state(cfg: SceneConfig) -> HostState:
    n, nw, nb0 = cfg.np, cfg.nw, cfg.nb0
    z4 = lambda: np.zeros((n, 4))
    return HostState(x=z4(), xysum=np.zeros((n, 2)), vel=z4(), vel0=z4(), acc=z4(), force=z4(),
                     angpos=z4(), angvel=z4(), angvel0=z4(), angacc=z4(), torque=z4(),
                     es_dot=np.zeros(n), es=np.zeros(n), ev_dot=np.zeros(n), ev=np.zeros(n),
                     p=np.zeros(n), contacts=np.zeros((n, NC), np.uint32),
                     distmod=np.zeros((n, NC, 4)), delta_t=np.zeros((n, NC, 4)),
                     bonds=np.zeros((nb0, 2), np.uint32), bonds_delta=np.zeros((nb0, 4)),
                     bonds_omega=np.zeros((nb0, 4)), walls_nx=np.zeros((nw, 4)),
                     walls_mvfd=np.zeros((nw, 4)), walls_vel0=np.zeros(nw))
