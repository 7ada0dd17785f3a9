"""The hot path at the bench's full sizes (1,000,000 spheres), checked through
properties that hold at any size, since the oracle is too slow to step a
million spheres: the step is deterministic whatever the graph length, the
cell list is a stable sort of the cell ids (src/device.cu:763-765) with
consistent start/end markers (src/sorting.cuh:49-121), and the jammed column
keeps the contact count its lattice fixes."""
import numpy as np
import pytest

from helpers import OUTPUT_FIELDS, STATE_FIELDS, WALL_FIELDS, mismatches
from sphere_b200 import scenes
from sphere_b200.sphk import Simulation
from sphere_b200.state import config_from_spherebin, state_from_spherebin

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def headline():
    """The bench's 1M polydisperse scene with the wall lowered onto the
    pack and seeded velocities, so that walls, cell changes and list
    restarts all happen within a few dozen steps."""
    sb = scenes.polydisperse()
    sb.w_x = sb.w_x - 0.3e-3
    sb.vel = np.random.default_rng(8).uniform(-0.2, 0.2, (sb.np, 3))
    return sb


def test_full_size_graph_length_changes_no_bit(headline):
    cfg = config_from_spherebin(headline)
    st0 = state_from_spherebin(headline)
    outs, stats = [], []
    for gs in (1, 8):
        with Simulation(cfg, graph_steps=gs) as sim:
            sim.upload(st0)
            sim.step(24)
            sim.sync()
            outs.append(sim.download())
            stats.append(sim.stats())
    assert mismatches(outs[0], outs[1], STATE_FIELDS + OUTPUT_FIELDS + WALL_FIELDS) == []
    assert stats[0]["cell_rebuilds"] == stats[1]["cell_rebuilds"] > 0
    assert outs[0].walls_nx[0, 3] != st0.walls_nx[0, 3]   # the wall moved


def test_full_size_cell_list_is_a_stable_sort(headline):
    cfg = config_from_spherebin(headline)
    with Simulation(cfg) as sim:
        sim.upload(state_from_spherebin(headline))
        sim.step(30)
        sim.sync()
        cell, perm, start, end = sim.cells()
    n = cfg.np
    c = cell.astype(np.int64)
    assert np.all(np.diff(c) >= 0)
    assert np.array_equal(np.sort(perm), np.arange(n, dtype=np.uint32))
    # members of a cell in ascending particle index
    same = np.diff(c) == 0
    assert np.all(np.diff(perm.astype(np.int64))[same] > 0)
    # start/end markers of every occupied cell, 0xffffffff for empty ones
    occ = np.unique(c)
    first = np.searchsorted(c, occ, "left")
    last = np.searchsorted(c, occ, "right")
    assert np.array_equal(start[occ], first.astype(np.uint32))
    assert np.array_equal(end[occ], last.astype(np.uint32))
    empty = np.setdiff1d(np.arange(cfg.ncells), occ)
    assert np.all(start[empty] == 0xFFFFFFFF)


def test_full_size_packed_column_keeps_every_contact():
    side = 100
    sb = scenes.packed(nx=side, ny=side, nz=side)
    cfg = config_from_spherebin(sb)
    with Simulation(cfg) as sim:
        sim.upload(state_from_spherebin(sb))
        sim.step(100)
        sim.sync()
        st = sim.download()
        stats = sim.stats()
    # six lattice neighbours each, less the missing one of the top and the
    # bottom layer; the lattice only vibrates
    assert stats["active_contacts"] == 6 * sb.np - 2 * side * side
    assert np.abs(st.vel[:, :3]).max() < 1e-2
