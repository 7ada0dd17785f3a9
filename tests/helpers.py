"""Shared helpers of the test suite: run a scene on an oracle or on the GPU
and compare states field by field."""
from __future__ import annotations

import numpy as np

from sphere_b200.state import (NC, HostState, config_from_spherebin, state_from_spherebin)

STATE_FIELDS = ("x", "vel", "angvel", "angpos", "xysum", "es", "ev", "vel0", "angvel0")
OUTPUT_FIELDS = ("force", "torque", "es_dot", "ev_dot", "p")
WALL_FIELDS = ("walls_nx", "walls_mvfd", "walls_vel0")
BOND_FIELDS = ("bonds", "bonds_delta", "bonds_omega")


def run_oracle(lib, sb, nsteps, nthreads=0, st=None, cfg=None):
    import pyoracle
    cfg = cfg or config_from_spherebin(sb)
    st = st if st is not None else state_from_spherebin(sb)
    run = pyoracle.OracleRun(lib, cfg, st)
    rc = run.step(nsteps, nthreads)
    return rc, st, run


def bits_equal(a, b) -> bool:
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and a.tobytes() == b.tobytes()


def mismatches(a: HostState, b: HostState, fields, active_only_distmod=True):
    bad = []
    for f in fields:
        A, B = getattr(a, f), getattr(b, f)
        if f in ("acc", "angacc"):
            A, B = A[:, :3], B[:, :3]
        if not bits_equal(A, B):
            diff = np.abs(np.asarray(A, float) - np.asarray(B, float))
            bad.append((f, float(np.nanmax(diff)) if diff.size else 0.0, int(np.count_nonzero(diff))))
    return bad


def active_distmod(st: HostState, np_):
    m = st.contacts != np_
    return np.where(m[..., None], st.distmod, 0.0)


def relative_error(a, b, scale=None):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    s = np.maximum(np.abs(b), 1e-300) if scale is None else scale
    return float(np.max(np.abs(a - b) / s)) if a.size else 0.0


def with_model(sb, model, kappa=0.05, V_b=1e-12, db=1e-4):
    """Switch a scene to contact model 1 (with capillary cohesion: kappa,
    liquid bridge volume V_b and the cohesion reach db) or model 3."""
    sb.contactmodel = int(model)
    if model == 1:
        sb.kappa, sb.V_b, sb.db = kappa, V_b, db
    return sb


def nan_aware_mismatches(a: HostState, b: HostState, fields):
    """Like mismatches(), but NaN equals NaN whatever its sign and payload
    (the CPU and the GPU write different NaN bit patterns)."""
    bad = []
    for f in fields:
        A, B = np.asarray(getattr(a, f)), np.asarray(getattr(b, f))
        if f in ("acc", "angacc"):
            A, B = A[:, :3], B[:, :3]
        if A.dtype.kind != "f":
            if not bits_equal(A, B):
                bad.append((f, "int", int(np.count_nonzero(A != B))))
            continue
        na, nb = np.isnan(A), np.isnan(B)
        if not np.array_equal(na, nb):
            bad.append((f, "nan pattern", int(np.count_nonzero(na != nb))))
            continue
        if not bits_equal(np.where(na, 0.0, A), np.where(nb, 0.0, B)):
            bad.append((f, "values", int(np.count_nonzero(np.where(na, 0.0, A) != np.where(nb, 0.0, B)))))
    return bad
