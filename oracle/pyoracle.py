"""ctypes binding of the CPU oracles (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/liborc.so`` (the plain-C restatement, ``kind == 1``) or
``oracle/_ref/libref.so`` (the reference's kernel bodies, ``kind == 2``) and
steps a ``sphere_b200.state.HostState`` in place.  Only tests/, the smoke
check and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_ORC = HERE / "liborc.so"
LIB_REF = HERE / "_ref" / "libref.so"
# the reference checkout's src/: SPHERE_REF_SRC, or a checkout named
# `reference` beside this repository
REF_SRC = Path(os.environ.get("SPHERE_REF_SRC", str(HERE.parent.parent / "reference" / "src")))

ERR_NC_OVERFLOW = 1
ERR_OUT_OF_GRID = 2
ERR_BAD_INPUT = 4

_dp = C.POINTER(C.c_double)
_up = C.POINTER(C.c_uint32)


class OrcScene(C.Structure):
    _fields_ = [
        ("np", C.c_uint32), ("nw", C.c_uint32), ("nb0", C.c_uint32), ("contactmodel", C.c_uint32),
        ("periodic", C.c_int32), ("num", C.c_uint32 * 3),
        ("origo", C.c_double * 3), ("L", C.c_double * 3),
        ("dt", C.c_double), ("t_current", C.c_double),
        ("g", C.c_double * 3),
        ("k_n", C.c_double), ("k_t", C.c_double), ("k_r", C.c_double),
        ("gamma_n", C.c_double), ("gamma_t", C.c_double), ("gamma_r", C.c_double),
        ("mu_s", C.c_double), ("mu_d", C.c_double), ("mu_r", C.c_double),
        ("gamma_wn", C.c_double), ("gamma_wt", C.c_double), ("mu_ws", C.c_double),
        ("mu_wd", C.c_double), ("rho", C.c_double), ("kappa", C.c_double), ("db", C.c_double),
        ("V_b", C.c_double), ("lambda_bar", C.c_double), ("sigma_b", C.c_double),
        ("tau_b", C.c_double), ("devs_A", C.c_double), ("devs_f", C.c_double),
        ("wmode", C.c_int32 * 6),
        ("x", _dp), ("vel", _dp), ("vel0", _dp), ("acc", _dp), ("force", _dp), ("angpos", _dp),
        ("angvel", _dp), ("angvel0", _dp), ("angacc", _dp), ("torque", _dp), ("xysum", _dp),
        ("es_dot", _dp), ("es", _dp), ("ev_dot", _dp), ("ev", _dp), ("p", _dp),
        ("contacts", _up), ("distmod", _dp), ("delta_t", _dp),
        ("bonds", _up), ("bonds_delta", _dp), ("bonds_omega", _dp),
        ("walls_nx", _dp), ("walls_mvfd", _dp), ("walls_vel0", _dp),
        ("cell_sorted", _up), ("perm", _up), ("cell_start", _up), ("cell_end", _up),
        ("wall0_force", _dp),
        ("nu", C.c_double), ("darcy", C.c_int32), ("iteration", C.c_uint32),
        ("d_factor", C.c_double), ("d_Hbuf", _dp * 2), ("d_hsel", C.c_uint32),
        ("d_V", _dp), ("d_dH", _dp), ("d_T", _dp),
        ("d_K", _dp), ("d_Ss", _dp), ("d_W", _dp), ("d_phi", _dp), ("d_dphi", _dp),
    ]


def build(ref: bool = True) -> None:
    """Build the oracle libraries with oracle/Makefile (``ref`` needs the
    reference checkout; it is skipped when that is absent)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "orc"], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF_SRC={REF_SRC}"], check=False)


def load(kind: str = "orc"):
    path = LIB_ORC if kind == "orc" else LIB_REF
    if not path.exists():
        raise FileNotFoundError(f"oracle library {path} is not built (run make -C oracle)")
    lib = C.CDLL(str(path))
    lib.orc_step.argtypes = [C.POINTER(OrcScene), C.c_uint64, C.c_int]
    lib.orc_step.restype = C.c_int
    lib.orc_kind.restype = C.c_int
    lib.orc_threads.argtypes = [C.c_int]
    lib.orc_threads.restype = C.c_int
    return lib


class OracleRun:
    """Owns the scratch/output arrays of one oracle scene.  With ``darcy`` (a
    ``sphere_b200.darcy.DarcyState``), each step also runs the Darcy flow
    block with dynamic viscosity ``nu`` and grain-size factor ``d_factor``;
    the state's arrays are updated in place (``H``/``H_new`` swap roles as
    the reference swaps its pointers)."""

    def __init__(self, lib, cfg, st, darcy=None, nu=0.0, d_factor=0.0):
        self.lib, self.cfg, self.st = lib, cfg, st
        n = cfg.np
        self.cell_sorted = np.zeros(n, np.uint32)
        self.perm = np.zeros(n, np.uint32)
        self.cell_start = np.zeros(cfg.ncells, np.uint32)
        self.cell_end = np.zeros(cfg.ncells, np.uint32)
        self.wall0_force = np.zeros(n)
        self._keep = []
        s = OrcScene()
        s.np, s.nw, s.nb0, s.contactmodel = cfg.np, cfg.nw, cfg.nb0, cfg.contactmodel
        s.periodic = cfg.periodic
        s.num[:] = [int(v) for v in cfg.num]
        s.origo[:] = [float(v) for v in cfg.origo]
        s.L[:] = [float(v) for v in cfg.L]
        s.dt = cfg.dt
        s.g[:] = [float(v) for v in cfg.g]
        for k, v in cfg.params.items():
            setattr(s, k, float(v))
        s.wmode[:] = [int(v) for v in cfg.wmode]
        for name in ("x", "vel", "vel0", "acc", "force", "angpos", "angvel", "angvel0", "angacc",
                     "torque", "xysum", "es_dot", "es", "ev_dot", "ev", "p", "distmod", "delta_t",
                     "bonds_delta", "bonds_omega", "walls_nx", "walls_mvfd", "walls_vel0"):
            setattr(s, name, self._ptr(getattr(st, name), np.float64))
        for name in ("contacts", "bonds"):
            setattr(s, name, self._ptr(getattr(st, name), np.uint32))
        s.cell_sorted = self._ptr(self.cell_sorted, np.uint32)
        s.perm = self._ptr(self.perm, np.uint32)
        s.cell_start = self._ptr(self.cell_start, np.uint32)
        s.cell_end = self._ptr(self.cell_end, np.uint32)
        s.wall0_force = self._ptr(self.wall0_force, np.float64)
        self.darcy = darcy
        if darcy is not None:
            s.darcy, s.nu, s.d_factor, s.iteration = 1, float(nu), float(d_factor), 0
            for name in ("V", "dH", "T", "K", "Ss", "W", "phi", "dphi"):
                setattr(s, "d_" + name, self._ptr(getattr(darcy, name), np.float64))
            self._bind_pressure(s)
        self.scene = s

    def _bind_pressure(self, s=None):
        s = s if s is not None else self.scene
        s.d_Hbuf[0] = self._ptr(self.darcy.H, np.float64)
        s.d_Hbuf[1] = self._ptr(self.darcy.H_new, np.float64)
        s.d_hsel = 0

    def _ptr(self, a, dtype):
        assert a.dtype == dtype and a.flags.c_contiguous, (a.dtype, a.flags)
        if a.size == 0:
            a = np.zeros(1, dtype)
            self._keep.append(a)
        return a.ctypes.data_as(_dp if dtype == np.float64 else _up)

    def step(self, nsteps: int, nthreads: int = 0) -> int:
        self.scene.t_current = self.st.t_current
        rc = self.lib.orc_step(C.byref(self.scene), nsteps, nthreads)
        self.st.t_current = self.scene.t_current
        if self.darcy is not None and self.scene.d_hsel == 1:
            self.darcy.H, self.darcy.H_new = self.darcy.H_new, self.darcy.H
            self._bind_pressure()
        return rc


# ---- ray tracer ---------------------------------------------------------------

class OrcRender(C.Structure):
    _fields_ = [("np", C.c_uint32), ("x", _dp), ("vel", _dp), ("values", _dp),
                ("L", C.c_double * 3), ("method", C.c_int32), ("maxval", C.c_float),
                ("lower_cutoff", C.c_float), ("width", C.c_uint32), ("height", C.c_uint32)]


class OrcCamera(C.Structure):
    _fields_ = [("u", C.c_float * 3), ("v", C.c_float * 3), ("w", C.c_float * 3),
                ("eye", C.c_float * 3), ("light", C.c_float * 3), ("imgplane", C.c_float * 4),
                ("d", C.c_float)]


def render_values(lib_orc, method, st):
    """DEM::render's colour-map values of a HostState (restatement)."""
    n = st.x.shape[0]
    out = np.zeros(n)
    f = lib_orc.orc_render_values
    f.argtypes = [C.c_int, C.c_uint32, _dp, _dp, _dp, _dp, _dp, _dp]
    f(int(method), n, *(np.ascontiguousarray(a).ctypes.data_as(_dp)
                         for a in (st.vel, st.angvel, st.angpos, st.xysum, st.p)),
      out.ctypes.data_as(_dp))
    return out


def render(lib, lib_orc, st, L, method=0, maxval=1.0e3, lower_cutoff=0.0, width=800,
           height=800, nthreads=0, values=None, rows=None):
    """One image (height, width, 4) uint8 of HostState `st` through `lib`'s
    kernels, with the camera of the restatement `lib_orc`."""
    r = OrcRender()
    x = np.ascontiguousarray(st.x, np.float64)
    vel = np.ascontiguousarray(st.vel, np.float64)
    r.np = x.shape[0]
    r.x, r.vel = x.ctypes.data_as(_dp), vel.ctypes.data_as(_dp)
    if method > 0 and values is None:
        values = render_values(lib_orc, method, st)
    vals = None if values is None else np.ascontiguousarray(values, np.float64)
    r.values = vals.ctypes.data_as(_dp) if vals is not None else None
    r.L[:] = [float(v) for v in L]
    r.method, r.maxval, r.lower_cutoff = int(method), float(maxval), float(lower_cutoff)
    r.width, r.height = int(width), int(height)
    cam = OrcCamera()
    lib_orc.orc_render_camera.argtypes = [C.POINTER(OrcRender), C.POINTER(OrcCamera)]
    lib_orc.orc_render_camera(C.byref(r), C.byref(cam))
    img = np.zeros((height, width, 4), np.uint8)
    row0, nrows = (0, height) if rows is None else rows
    lib.orc_render_rows.argtypes = [C.POINTER(OrcRender), C.POINTER(OrcCamera),
                                    C.POINTER(C.c_uint8), C.c_uint32, C.c_uint32, C.c_int]
    rc = lib.orc_render_rows(C.byref(r), C.byref(cam), img.ctypes.data_as(C.POINTER(C.c_uint8)),
                             int(row0), int(nrows), int(nthreads))
    if rc != 0:
        raise RuntimeError(f"orc_render_image failed ({rc})")
    return img, cam
