"""Pin the plain-C oracle (oracle/dem_oracle.c) to the reference's own kernel
bodies (oracle/_ref/libref.so) and to the committed golden fixtures."""
import json
from pathlib import Path

import numpy as np
import pytest

import pyoracle
from helpers import (BOND_FIELDS, OUTPUT_FIELDS, STATE_FIELDS, WALL_FIELDS, mismatches,
                     relative_error, run_oracle, with_model)
from sphere_b200 import scenes
from sphere_b200.spherebin import readbin
from sphere_b200.state import config_from_spherebin, state_from_spherebin

GOLDEN = Path(__file__).resolve().parent / "golden"
ALL = STATE_FIELDS + OUTPUT_FIELDS + ("acc", "angacc", "contacts", "delta_t") + WALL_FIELDS

SCENES = {
    "box": lambda: scenes.collision(n=1200, seed=11, periodic=0),
    "periodic_xy": lambda: scenes.collision(n=1200, seed=12, periodic=1),
    "periodic_x_wall": lambda: scenes.collision(n=1000, seed=13, periodic=2, nw=1),
    "box_wall": lambda: scenes.collision(n=1500, seed=14, periodic=0, nw=1),
    "bonded": lambda: scenes.bonded(nx=4, ny=3, nz=3, sigma_b=1e30, tau_b=1e30),
}


def _need_ref(oracle_libs):
    if "ref" not in oracle_libs:
        pytest.skip("reference harness not built (reference checkout absent)")


@pytest.mark.parametrize("name", sorted(SCENES))
def test_restatement_matches_reference_kernels(oracle_libs, name):
    _need_ref(oracle_libs)
    sb = SCENES[name]()
    rc1, a, ra = run_oracle(oracle_libs["orc"], sb, 40, nthreads=4)
    rc2, b, rb = run_oracle(oracle_libs["ref"], sb, 40, nthreads=4)
    assert rc1 == 0 and rc2 == 0
    fields = ALL + (BOND_FIELDS if sb.nb0 else ())
    assert mismatches(a, b, fields) == []
    assert np.array_equal(ra.perm, rb.perm)
    assert np.array_equal(ra.cell_sorted, rb.cell_sorted)
    assert np.array_equal(ra.cell_start, rb.cell_start)
    occupied = ra.cell_start != 0xFFFFFFFF
    assert np.array_equal(ra.cell_end[occupied], rb.cell_end[occupied])
    # the scene exercised what it is meant to: contacts with slip, or bonds
    if sb.nb0:
        assert np.count_nonzero(a.bonds_delta) > 0
    else:
        assert (a.contacts != sb.np).sum() > 100
        assert np.count_nonzero(a.es_dot) > 0


def test_threaded_block_summation_equals_ordered_form(oracle_libs):
    """The reference's summation() run with real 256-thread blocks gives the
    same wall force as the harness's order-equivalent evaluation."""
    _need_ref(oracle_libs)
    lib = oracle_libs["ref"]
    sb = scenes.collision(n=700, seed=21, periodic=0, nw=1)
    lib.orc_set_threaded_summation_max.argtypes = [pyoracle.C.c_uint]
    lib.orc_set_threaded_summation_max(0)
    _, a, _ = run_oracle(lib, sb, 3)
    lib.orc_set_threaded_summation_max(1 << 30)
    try:
        _, b, _ = run_oracle(lib, sb, 3)
    finally:
        lib.orc_set_threaded_summation_max(0)
    assert np.any(a.walls_mvfd[:, 2] != 0.0)
    assert mismatches(a, b, WALL_FIELDS + ("x",)) == []


def _golden_cases():
    idx = GOLDEN / "index.json"
    if not idx.exists():
        return []
    return json.loads(idx.read_text())["cases"]


@pytest.mark.parametrize("case", _golden_cases(), ids=lambda c: c["name"])
def test_oracle_matches_golden_fixtures(oracle_libs, case):
    sb = readbin(GOLDEN / case["input"])
    want = np.load(GOLDEN / case["expected"])
    rc, st, run = run_oracle(oracle_libs["orc"], sb, case["steps"])
    assert rc == 0
    for f in want.files:
        if f == "perm":
            got = run.perm
        elif f == "contacts_active":
            got = st.contacts != sb.np
        elif f == "delta_t_active":
            got = st.delta_t[st.contacts != sb.np]
        else:
            got = getattr(st, f)
        assert np.array_equal(np.asarray(got), want[f]), f


MODEL_SCENES = {
    "box": dict(periodic=0),
    "periodic_xy": dict(periodic=1),
    "periodic_x_wall": dict(periodic=2, nw=1),
}


@pytest.mark.parametrize("name", sorted(MODEL_SCENES))
def test_model1_with_cohesion_matches_reference_kernels(oracle_libs, name):
    """contactLinearViscous + capillaryCohesion_exp (model 1): bit for bit
    when the oracle calls the C library's expf, as the reference's host build
    does."""
    _need_ref(oracle_libs)
    orc = oracle_libs["orc"]
    mk = lambda: with_model(scenes.collision(n=1200, seed=11, **MODEL_SCENES[name]), 1)
    orc.orc_set_libm_float_math(1)
    try:
        rc1, a, ra = run_oracle(orc, mk(), 30, nthreads=4)
    finally:
        orc.orc_set_libm_float_math(0)
    rc2, b, rb = run_oracle(oracle_libs["ref"], mk(), 30, nthreads=4)
    assert rc1 == 0 and rc2 == 0
    assert mismatches(a, b, ALL) == []
    assert np.array_equal(ra.perm, rb.perm)
    # contacts and cohesion both acted; the slots stay empty in model 1
    assert np.count_nonzero(a.p) > 100
    assert (a.contacts == mk().np).all()


def test_model1_nearest_float_exp_stays_close(oracle_libs):
    """With expf evaluated as the float nearest to exp (the CUDA path's
    choice) the oracle leaves the reference's host build only by the last
    bits of a few cohesion forces: within 1e-9 relative after 30 steps."""
    _need_ref(oracle_libs)
    mk = lambda: with_model(scenes.collision(n=1200, seed=11, periodic=1), 1)
    rc1, a, _ = run_oracle(oracle_libs["orc"], mk(), 30, nthreads=4)
    rc2, b, _ = run_oracle(oracle_libs["ref"], mk(), 30, nthreads=4)
    assert rc1 == 0 and rc2 == 0
    assert relative_error(a.x[:, :3], b.x[:, :3], scale=np.abs(b.x[:, :3]).max()) < 1e-12
    vscale = np.abs(b.vel[:, :3]).max()
    assert relative_error(a.vel[:, :3], b.vel[:, :3], scale=vscale) < 1e-9


@pytest.mark.parametrize("name", sorted(MODEL_SCENES))
def test_model3_matches_reference_kernels(oracle_libs, name):
    """contactHertz (model 3) raises the negative overlap to fractional
    powers, so every touching pair gets NaN forces; the oracle reproduces the
    reference's step, NaN bits included."""
    _need_ref(oracle_libs)
    mk = lambda: with_model(scenes.collision(n=1200, seed=11, **MODEL_SCENES[name]), 3)
    rc1, a, _ = run_oracle(oracle_libs["orc"], mk(), 1, nthreads=4)
    rc2, b, _ = run_oracle(oracle_libs["ref"], mk(), 1, nthreads=4)
    assert rc1 == 0 and rc2 == 0
    assert mismatches(a, b, ALL) == []
    touching = (a.contacts != mk().np).any(axis=1)
    assert touching.sum() > 100
    assert np.isnan(a.force[touching, :3]).all()
    assert not np.isnan(a.force[~touching, :3]).any()


def test_packed_column_matches_reference_kernels(oracle_libs):
    """The jammed column: six contacts per sphere, across the periodic faces
    and against the floor and the stress-controlled top wall."""
    _need_ref(oracle_libs)
    sb = scenes.packed(nx=12, ny=12, nz=10)
    rc1, a, ra = run_oracle(oracle_libs["orc"], sb, 40, nthreads=4)
    rc2, b, rb = run_oracle(oracle_libs["ref"], sb, 40, nthreads=4)
    assert rc1 == 0 and rc2 == 0
    assert mismatches(a, b, ALL) == []
    assert np.array_equal(ra.perm, rb.perm)
    assert (a.contacts != sb.np).sum() == 6 * sb.np - 2 * 144
    assert np.count_nonzero(a.delta_t) > 0


def test_packed_column_stays_jammed(oracle_libs):
    """The contact-heavy bench scene holds its six contacts per sphere: over
    600 steps the lattice only vibrates (speeds under 1 cm/s) and no contact
    opens.  With the reference's model-2 normal viscosity on, the same column
    flies apart within a few hundred steps, which is why it is off there."""
    sb = scenes.packed(nx=10, ny=10, nz=10)
    rc, st, _ = run_oracle(oracle_libs["orc"], sb, 600, nthreads=4)
    assert rc == 0
    assert np.abs(st.vel[:, :3]).max() < 1e-2
    # 6 per sphere less one for each sphere of the top and bottom layers
    assert (st.contacts != sb.np).sum() == 6 * sb.np - 2 * 100
    sb.gamma_n = 3.0
    rc, st, _ = run_oracle(oracle_libs["orc"], sb, 600, nthreads=4)
    assert rc != 0 or np.abs(st.vel[:, :3]).max() > 1.0
