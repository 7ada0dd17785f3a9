"""The batched ensemble context (sph_batch_create): several independent
scenes of different sizes, grids, periodicity, stiffness, friction and time
step, stepped together by one context.  Each scene's result must be the
oracle's for that scene alone, bit for bit."""
import ctypes as C

import numpy as np
import pytest

from helpers import OUTPUT_FIELDS, STATE_FIELDS, mismatches, run_oracle
from sphere_b200 import scenes, sphk
from sphere_b200.sphk import BatchSimulation
from sphere_b200.state import config_from_spherebin, state_from_spherebin

FIELDS = STATE_FIELDS + OUTPUT_FIELDS + ("acc", "angacc", "contacts", "delta_t")


def _mixed():
    return [
        scenes.collision(n=900, seed=81, periodic=0),
        scenes.ensemble_member(0, n_range=(300, 3000)),
        scenes.collision(n=1200, seed=82, periodic=1),
        scenes.ensemble_member(1, n_range=(300, 3000), cell_factor=2.5),
        scenes.collision(n=700, seed=83, periodic=2),
        scenes.ensemble_member(2, n_range=(300, 3000)),
    ]


@pytest.mark.parametrize("patch, msg", [
    (dict(nw=1), b"no dynamic walls"),
    (dict(nb0=3), b"no bonds"),
    (dict(contactmodel=1), b"contact model 2"),
    (dict(np=0), b"np must be positive"),
])
def test_batch_rejects_unsupported_scenes_without_gpu(sphk_lib, patch, msg):
    cfgs = [sphk.make_config(config_from_spherebin(scenes.collision(n=20, seed=s))) for s in (1, 2)]
    for k, v in patch.items():
        setattr(cfgs[1], k, v)
    arr = (sphk.SphConfig * 2)(*cfgs)
    ctx = C.c_void_p()
    assert sphk_lib.sph_batch_create(arr, 2, C.byref(ctx)) == -5
    err = sphk_lib.sph_last_error(ctx)
    assert msg in err and b"scene 1" in err
    assert sphk_lib.sph_destroy(ctx) == 0


def test_pack_and_split_are_inverse():
    sbs = _mixed()[:3]
    states = [state_from_spherebin(sb) for sb in sbs]
    packed = sphk.pack_states(states)
    assert packed.x.shape[0] == sum(sb.np for sb in sbs)
    back = sphk.split_state(packed, [sb.np for sb in sbs])
    for a, b in zip(back, states):
        assert mismatches(a, b, FIELDS) == []


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(), dict(verlet_skin=0.0), dict(relayout_every=5, graph_steps=3),
                                dict(block_shapes=1)],
                         ids=["default", "sweep_every_step", "relayout_graphs", "block_shapes_1"])
def test_batch_matches_each_scene_alone(oracle_libs, kw):
    sbs = _mixed()
    want = []
    for sb in sbs:
        rc, st, _ = run_oracle(oracle_libs["orc"], sb, 40)
        assert rc == 0
        want.append(st)
    with BatchSimulation([config_from_spherebin(sb) for sb in sbs], **kw) as sim:
        sim.upload([state_from_spherebin(sb) for sb in sbs])
        sim.step(17)
        sim.step(23)
        sim.sync()
        got = sim.download_all()
        stats = sim.stats()
    for i, (g, w) in enumerate(zip(got, want)):
        assert mismatches(g, w, FIELDS) == [], f"scene {i}"
    assert stats["active_contacts"] == sum(int((w.contacts != sb.np).sum()) for w, sb in zip(want, sbs))


@pytest.mark.gpu
def test_batch_of_one_equals_single_context():
    sb = scenes.collision(n=1500, seed=84, periodic=1)
    from sphere_b200.sphk import Simulation
    with Simulation(config_from_spherebin(sb)) as sim:
        sim.upload(state_from_spherebin(sb))
        sim.step(30)
        sim.sync()
        a = sim.download()
    with BatchSimulation([config_from_spherebin(sb)]) as sim:
        sim.upload([state_from_spherebin(sb)])
        sim.step(30)
        sim.sync()
        b = sim.download_all()[0]
    assert mismatches(a, b, FIELDS) == []
