"""Parity of the CUDA path (libsphk through its C ABI) with the CPU oracle
and with the golden fixtures made from the reference's own kernels.

The bar is bit-exactness for everything: cell ids, permutation, contact
slots, tangential history, forces, positions and walls.  Scenes are small
enough for the oracle to finish in seconds."""
import json
from pathlib import Path

import numpy as np
import pytest

from helpers import (BOND_FIELDS, OUTPUT_FIELDS, STATE_FIELDS, WALL_FIELDS, active_distmod,
                     mismatches, nan_aware_mismatches, run_oracle, with_model)
from sphere_b200 import scenes
from sphere_b200.spherebin import readbin
from sphere_b200.sphk import SphError, Simulation
from sphere_b200.state import config_from_spherebin, state_from_spherebin

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
ALL = STATE_FIELDS + OUTPUT_FIELDS + ("acc", "angacc", "contacts", "delta_t") + WALL_FIELDS

SCENES = {
    "box": lambda: scenes.collision(n=1500, seed=31, periodic=0),
    "periodic_xy": lambda: scenes.collision(n=1500, seed=32, periodic=1),
    "periodic_x_wall": lambda: scenes.collision(n=1200, seed=33, periodic=2, nw=1),
    "box_wall": lambda: scenes.collision(n=2000, seed=34, periodic=0, nw=1),
    "bonded": lambda: scenes.bonded(nx=4, ny=3, nz=3, sigma_b=1e30, tau_b=1e30),
    # the cluster straddles the periodic x/y boundaries: cell ids saturate
    # and alias while particles cross, which turns the cell-level pruning off
    "periodic_crossing": lambda: _crossing(),
    "polydisperse_small": lambda: _small_polydisperse(),
    # jammed lattice: six contacts per sphere, across the periodic faces too
    "packed": lambda: scenes.packed(nx=12, ny=12, nz=10),
}


def _crossing():
    sb = scenes.collision(n=1500, seed=35, periodic=1, straddle=True, vmax=3.0)
    # every 10th particle sits just inside a periodic face and moves out
    # through it, so positions leave the grid for a step before the wrap
    rng = np.random.default_rng(36)
    sel = np.arange(0, sb.np, 10)
    for j, i in enumerate(sel):
        ax = j % 2
        hi = (j // 2) % 2 == 0
        sb.x[i, ax] = sb.L[ax] - 1e-7 if hi else 1e-7
        sb.vel[i, ax] = (1.0 if hi else -1.0) * rng.uniform(0.5, 2.0)
    return sb


def _small_polydisperse():
    # the bench workload at 20,000 spheres with the wall lowered onto the pack
    sb = scenes.polydisperse(n=20000, seed=5, L=(0.0543, 0.0543, 0.1086), num=(13, 13, 27))
    sb.w_x = sb.w_x - 0.3e-3
    sb.vel = np.random.default_rng(6).uniform(-0.05, 0.05, (sb.np, 3))
    return sb


def run_gpu(sb, chunks, **kw):
    cfg = config_from_spherebin(sb)
    with Simulation(cfg, **kw) as sim:
        sim.upload(state_from_spherebin(sb))
        for n in chunks:
            sim.step(n)
        sim.sync()
        st = sim.download()
        cells = sim.cells()
        stats = sim.stats()
    return st, cells, stats


@pytest.mark.parametrize("name", sorted(SCENES))
@pytest.mark.parametrize("chunks", [(40,), (1, 7, 13, 19)], ids=["one_call", "four_calls"])
def test_gpu_matches_oracle_bit_for_bit(oracle_libs, name, chunks):
    sb = SCENES[name]()
    rc, want, orun = run_oracle(oracle_libs["orc"], sb, sum(chunks))
    assert rc == 0
    got, (cell_sorted, perm, cstart, cend), stats = run_gpu(sb, chunks)
    fields = ALL + (BOND_FIELDS if sb.nb0 else ())
    assert mismatches(got, want, fields) == []
    assert np.array_equal(active_distmod(got, sb.np), active_distmod(want, sb.np))
    assert got.t_current == want.t_current
    # the cell list of the last step: cell ids, permutation, start/end
    assert np.array_equal(perm, orun.perm)
    assert np.array_equal(cell_sorted, orun.cell_sorted)
    assert np.array_equal(cstart, orun.cell_start)
    occ = orun.cell_start != 0xFFFFFFFF
    assert np.array_equal(cend[occ], orun.cell_end[occ])
    assert stats["active_contacts"] == int((want.contacts != sb.np).sum())


@pytest.mark.parametrize("name", ["box", "periodic_crossing", "box_wall", "polydisperse_small"])
@pytest.mark.parametrize("skin", [0.0, 0.6], ids=["sweep_every_step", "wide_skin"])
def test_contact_detection_modes_agree_with_oracle(oracle_libs, name, skin):
    """Verlet lists off (the full 27-cell sweep every step) and with a wide
    skin give the oracle's results bit for bit."""
    sb = SCENES[name]()
    rc, want, _ = run_oracle(oracle_libs["orc"], sb, 30)
    assert rc == 0
    got, _, _ = run_gpu(sb, (30,), verlet_skin=skin)
    assert mismatches(got, want, ALL) == []


@pytest.mark.parametrize("name", ["packed", "polydisperse_small", "box_wall", "periodic_crossing"])
def test_second_block_shapes_agree_with_oracle(oracle_libs, name):
    """The contact search and contact force kernels in their second compiled
    block shapes (SPH_OPT_BLOCK_SHAPES = 1) give the oracle's results bit for
    bit."""
    sb = SCENES[name]()
    rc, want, _ = run_oracle(oracle_libs["orc"], sb, 30)
    assert rc == 0
    got, _, _ = run_gpu(sb, (11, 19), block_shapes=1)
    assert mismatches(got, want, ALL) == []


@pytest.mark.parametrize("span", [2, 4])
@pytest.mark.parametrize("name", ["packed", "polydisperse_small", "box_wall", "periodic_crossing"])
def test_contact_search_spans_agree_with_oracle(oracle_libs, name, span):
    """The contact search making the list decisions of 2 or 4 particles per
    thread and dealing the ones that need a search to the warp's lanes (the
    layout chosen at 1M spheres) gives the oracle's results bit for bit."""
    sb = SCENES[name]()
    rc, want, _ = run_oracle(oracle_libs["orc"], sb, 30)
    assert rc == 0
    got, _, _ = run_gpu(sb, (11, 19), topo_span=span)
    assert mismatches(got, want, ALL) == []


@pytest.mark.parametrize("name", ["box", "periodic_xy"])
def test_verlet_epochs_restart_exactly(oracle_libs, name):
    """300 steps: the displacement bound restarts the list epoch several
    times and particles change cells often; results stay bit-exact."""
    sb = SCENES[name]()
    rc, want, _ = run_oracle(oracle_libs["orc"], sb, 300)
    assert rc == 0
    got, _, _ = run_gpu(sb, (100, 77, 123))
    assert mismatches(got, want, ALL) == []


def _golden_cases():
    idx = GOLDEN / "index.json"
    return json.loads(idx.read_text())["cases"] if idx.exists() else []


@pytest.mark.parametrize("case", _golden_cases(), ids=lambda c: c["name"])
def test_gpu_matches_golden_fixtures(case):
    sb = readbin(GOLDEN / case["input"])
    want = np.load(GOLDEN / case["expected"])
    steps = case["steps"]
    got, (_, perm, _, _), _ = run_gpu(sb, (steps,))
    for f in want.files:
        if f == "perm":
            value = perm
        elif f == "delta_t_active":
            value = got.delta_t[got.contacts != sb.np]
        else:
            value = getattr(got, f)
        assert np.asarray(value).tobytes() == want[f].tobytes(), f


def test_relayout_does_not_change_results(oracle_libs):
    sb = scenes.collision(n=1500, seed=41, periodic=1)
    a, _, _ = run_gpu(sb, (30,))
    b, _, stats = run_gpu(sb, (30,), relayout_every=4)
    assert stats["relayouts"] >= 7
    assert mismatches(a, b, ALL) == []


def test_relayout_keeps_bonds_on_their_particles():
    """Re-sorting storage every 7 steps of a stretched bar leaves its bonds,
    their history and their breaks exactly as a run without relayouts: each
    bond's storage pair follows its particles to their new places."""
    sb = scenes.tension(nx=6, ny=6, nz=6, pull=0.2)
    a, _, _ = run_gpu(sb, (120,))
    b, _, stats = run_gpu(sb, (120,), relayout_every=7)
    assert stats["relayouts"] >= 17
    assert mismatches(a, b, ALL + BOND_FIELDS) == []
    assert int((a.bonds[:, 0] >= sb.np).sum()) > 0


@pytest.mark.parametrize("graph_steps", [1, 3, 16])
def test_graph_batching_does_not_change_results(graph_steps):
    sb = scenes.collision(n=800, seed=42, periodic=0, nw=1)
    a, _, _ = run_gpu(sb, (37,), graph_steps=8)
    b, _, _ = run_gpu(sb, (37,), graph_steps=graph_steps)
    assert mismatches(a, b, ALL) == []


def test_null_step_known_answer():
    """tests/io_tests.py:27-33: with no gravity and no contacts the state after
    the run is identical to the input except for the time fields."""
    sb = readbin(GOLDEN / "io_null_step.bin")
    got, _, _ = run_gpu(sb, (3,))
    st0 = state_from_spherebin(sb)
    for f in ("x", "vel", "angvel", "angpos", "xysum", "es", "ev", "walls_nx", "walls_mvfd"):
        assert np.array_equal(getattr(got, f), getattr(st0, f)), f


def test_nc_overflow_is_reported(oracle_libs):
    """A large sphere overlapped by more than 32 small ones: the reference
    writes past the slot row; here the step reports SPH_ERR_NC_OVERFLOW."""
    from sphere_b200.spherebin import Spherebin
    rng = np.random.default_rng(5)
    n_small = 40
    sb = Spherebin(np_=n_small + 1, nw=0, sid="overflow")
    dirs = rng.normal(size=(n_small, 3))
    dirs /= np.linalg.norm(dirs, axis=1)[:, None]
    center = np.array([0.05, 0.05, 0.05])
    sb.x = np.vstack([center, center + dirs * 0.0108])
    sb.radius = np.concatenate([[0.01], np.full(n_small, 1e-3)])
    sb.origo = np.zeros(3)
    sb.L = np.full(3, 0.1)
    sb.num = np.array([4, 4, 4], dtype=np.uint32)
    sb.k_n = sb.k_t = 1e3
    sb.time_dt = 1e-6
    rc, _, _ = run_oracle(oracle_libs["orc"], sb, 1)
    assert rc & 1
    cfg = config_from_spherebin(sb)
    with Simulation(cfg) as sim:
        sim.upload(state_from_spherebin(sb))
        sim.step(1)
        with pytest.raises(SphError) as e:
            sim.sync()
        assert e.value.code == -2


def test_out_of_grid_is_reported():
    sb = scenes.collision(n=64, seed=6, periodic=0)
    sb.vel[0] = [0.0, 0.0, 500.0]      # leaves the grid within a few steps
    cfg = config_from_spherebin(sb)
    with Simulation(cfg) as sim:
        sim.upload(state_from_spherebin(sb))
        sim.step(200)
        with pytest.raises(SphError) as e:
            sim.sync()
        assert e.value.code == -3


MODEL_SCENES = {
    "box": dict(periodic=0),
    "periodic_xy": dict(periodic=1),
    "periodic_x_wall": dict(periodic=2, nw=1),
    "box_wall": dict(periodic=0, nw=1),
}


@pytest.mark.parametrize("name", sorted(MODEL_SCENES))
@pytest.mark.parametrize("skin", [0.0, 0.1], ids=["sweep_every_step", "verlet"])
def test_model1_with_cohesion_matches_oracle(oracle_libs, name, skin):
    """Contact model 1 (contactLinearViscous, processed during the neighbour
    sweep) with capillary cohesion: bit for bit over 60 steps in two calls,
    with the Verlet lists on and off."""
    mk = lambda: with_model(scenes.collision(n=1500, seed=61, **MODEL_SCENES[name]), 1)
    rc, want, _ = run_oracle(oracle_libs["orc"], mk(), 60)
    assert rc == 0
    got, _, stats = run_gpu(mk(), (23, 37), verlet_skin=skin)
    assert mismatches(got, want, ALL) == []
    assert stats["active_contacts"] == 0          # no slots in model 1
    assert np.count_nonzero(want.p) > 100


def test_model1_cohesion_reaches_beyond_contact(oracle_libs):
    """A pair with a gap below db attracts under model 1: the capillary term
    is found through the neighbour search exactly as the oracle finds it."""
    sb = with_model(scenes.collision(n=2, seed=1, periodic=0, vmax=0.0, wmax=0.0,
                                     g=(0.0, 0.0, 0.0)), 1, kappa=0.05, V_b=1e-12, db=2e-4)
    sb.radius[:] = 1e-3
    sb.x[0] = (0.03, 0.03, 0.03)
    sb.x[1] = (0.03 + 2e-3 + 1e-4, 0.03, 0.03)
    rc, want, _ = run_oracle(oracle_libs["orc"], sb, 3)
    assert rc == 0
    got, _, _ = run_gpu(sb, (3,))
    assert mismatches(got, want, ALL) == []
    assert got.force[0, 0] > 0.0 and got.force[1, 0] < 0.0


@pytest.mark.parametrize("name", sorted(MODEL_SCENES))
def test_model3_reproduces_reference_step(oracle_libs, name):
    """Contact model 3 (contactHertz) gives NaN forces to every touching
    pair, as the reference does; the GPU reproduces the step, with NaN in the
    same places and every other value bit for bit."""
    mk = lambda: with_model(scenes.collision(n=1500, seed=62, **MODEL_SCENES[name]), 3)
    rc, want, _ = run_oracle(oracle_libs["orc"], mk(), 1)
    assert rc == 0
    sb = mk()
    with Simulation(config_from_spherebin(sb)) as sim:
        sim.upload(state_from_spherebin(sb))
        sim.step(1)
        # the NaN positions have left the grid: the step says so
        with pytest.raises(SphError) as e:
            sim.sync()
        assert e.value.code == -3
        got = sim.download()
    assert nan_aware_mismatches(got, want, ALL) == []
    touching = (want.contacts != mk().np).any(axis=1)
    assert touching.sum() > 100 and np.isnan(got.force[touching, :3]).all()


@pytest.mark.parametrize("periodic", [0, 1])
def test_sparse_scene_forms_contacts_exactly(oracle_libs, periodic):
    """A loose, fast scene: most particles are far from everything, so their
    list tests are skipped on the gap bound, while pairs keep closing and
    forming new contacts inside list epochs.  Bit-exact over 300 steps."""
    sb = scenes.collision(n=1500, seed=38 + periodic, periodic=periodic, phi_target=0.12, vmax=2.0)
    rc, want, _ = run_oracle(oracle_libs["orc"], sb, 300)
    assert rc == 0
    got, _, stats = run_gpu(sb, (120, 180))
    assert mismatches(got, want, ALL) == []
    assert stats["active_contacts"] > 0


def test_bonded_tension_breaks_bonds_exactly(oracle_libs):
    """The bonded-tension workload at small size: both ends pulled apart
    (fixvel) at 2 m/s with finite bond strengths, so bonds stretch and break
    (marker nb0, nb0 >= np); bit for bit over 500 steps, bond history and
    breaks included."""
    sb = scenes.bonded(nx=5, ny=3, nz=3, sigma_b=2e3, tau_b=2e3, pull=2.0)
    assert sb.nb0 >= sb.np
    rc, want, _ = run_oracle(oracle_libs["orc"], sb, 500)
    assert rc == 0
    got, _, _ = run_gpu(sb, (200, 300))
    assert mismatches(got, want, ALL + BOND_FIELDS) == []
    broken = int((got.bonds[:, 0] == sb.nb0).sum())
    assert 0 < broken < sb.nb0


def test_stretched_bar_breaks_two_thirds_of_its_bonds_exactly(oracle_libs):
    """The bonded-tension workload's bar (FCC, every lattice neighbour
    bonded) at 5,324 spheres and 29,106 bonds, stretched as a whole so that
    bonds throughout the bar break within the run (about two thirds of them,
    all that lie along the pull); bit for bit over 120 steps in two calls,
    bond history and breaks included."""
    sb = scenes.tension(nx=11, ny=11, nz=11, pull=0.2)
    assert sb.np == 5324 and sb.nb0 > 5 * sb.np
    rc, want, _ = run_oracle(oracle_libs["orc"], sb, 120)
    assert rc == 0
    got, _, _ = run_gpu(sb, (45, 75))
    assert mismatches(got, want, ALL + BOND_FIELDS) == []
    broken = int((got.bonds[:, 0] >= sb.np).sum())
    assert 0.5 * sb.nb0 < broken < sb.nb0


def _ensemble_stats(sb, st):
    m = 4.0 / 3.0 * np.pi * st.x[:, 3] ** 3 * sb.rho
    ke = float(np.sum(0.5 * m * np.sum(st.vel[:, :3] ** 2, axis=1)))
    v_solid = float(np.sum(4.0 / 3.0 * np.pi * st.x[:, 3] ** 3))
    phi = v_solid / float(np.prod(sb.L))
    coordination = float((st.contacts != sb.np).sum()) / sb.np
    return dict(kinetic=ke, packing_fraction=phi, coordination=coordination,
                shear_energy=float(st.es.sum()), viscous_energy=float(st.ev.sum()))


def test_ensemble_statistics_after_ten_thousand_steps(oracle_libs):
    """10^4 steps of a colliding scene: the trajectories stay bit-identical,
    so packing fraction, coordination number and energies agree exactly."""
    sb = scenes.collision(n=600, seed=77, periodic=0)
    rc, want, _ = run_oracle(oracle_libs["orc"], sb, 10_000)
    assert rc == 0
    got, _, _ = run_gpu(sb, (3000, 7000))
    assert mismatches(got, want, ALL) == []
    assert _ensemble_stats(sb, got) == _ensemble_stats(sb, want)
    assert _ensemble_stats(sb, got)["viscous_energy"] > 0.0
