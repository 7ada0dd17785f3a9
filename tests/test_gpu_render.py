"""The ray tracer on the GPU (sph_render), pixel for pixel against the
oracle, which is pinned to the reference's own kernels."""
import numpy as np
import pytest

from helpers import run_oracle
from sphere_b200 import scenes
from sphere_b200.sphk import SphError, Simulation
from sphere_b200.state import config_from_spherebin, state_from_spherebin
from test_render import CASES, render_scene

pytestmark = pytest.mark.gpu


def gpu_render(sb, st, method, maxval, cut, w, h, steps=0):
    with Simulation(config_from_spherebin(sb)) as sim:
        sim.upload(st)
        if steps:
            sim.step(steps)
            sim.sync()
        return sim.render(method, maxval, cut, w, h)


@pytest.mark.parametrize("case", CASES, ids=[f"m{c[0]}_{c[3]}x{c[4]}_cut{c[2]}" for c in CASES])
def test_gpu_render_matches_oracle(oracle_libs, case):
    import pyoracle
    method, maxval, cut, w, h = case
    sb, st = render_scene()
    want, _ = pyoracle.render(oracle_libs["orc"], oracle_libs["orc"], st, sb.L, method, maxval,
                              cut, w, h)
    got = gpu_render(sb, st, method, maxval, cut, w, h)
    assert np.array_equal(got[..., :3], want[..., :3])


def test_gpu_render_after_steps_matches_oracle(oracle_libs):
    """The image of the device's state after 30 steps equals the oracle's
    image of its own (bit-identical) state."""
    import pyoracle
    sb = scenes.collision(n=1500, seed=72, periodic=1, straddle=True)
    _, st, _ = run_oracle(oracle_libs["orc"], sb, 30, nthreads=4)
    want, _ = pyoracle.render(oracle_libs["orc"], oracle_libs["orc"], st, sb.L, 2, 0.4, 0.0,
                              160, 160)
    got = gpu_render(sb, state_from_spherebin(sb), 2, 0.4, 0.0, 160, 160, steps=30)
    assert np.array_equal(got[..., :3], want[..., :3])


def test_gpu_render_dense_pack_and_ties(oracle_libs):
    """A dense polydisperse pack (many spheres per pixel) and duplicated
    spheres (equal distances: the lowest index must win)."""
    import pyoracle
    sb = scenes.polydisperse(n=20000, seed=9, L=(0.0543, 0.0543, 0.1086), num=(13, 13, 27))
    st = state_from_spherebin(sb)
    st.x[1::2] = st.x[0::2][: st.x[1::2].shape[0]]   # pairs of identical spheres
    st.vel[:, 3] = 0.0
    st.vel[2::4, 3] = 1.0
    for method in (0, 2):
        want, _ = pyoracle.render(oracle_libs["orc"], oracle_libs["orc"], st, sb.L, method, 0.05,
                                  0.0, 200, 150)
        got = gpu_render(sb, st, method, 0.05, 0.0, 200, 150)
        assert np.array_equal(got[..., :3], want[..., :3]), method


def test_gpu_render_sphere_around_the_eye_plane(oracle_libs):
    """A sphere large enough to reach the plane through the eye parallel to
    the image: its projection is unbounded, so every pixel is tested."""
    import pyoracle
    sb, st = render_scene(seed=73, n=300)
    st.x[5, 3] = 6.0 * float(sb.L[0])
    want, _ = pyoracle.render(oracle_libs["orc"], oracle_libs["orc"], st, sb.L, 0, 1.0, 0.0, 64, 64)
    got = gpu_render(sb, st, 0, 1.0, 0.0, 64, 64)
    assert np.array_equal(got[..., :3], want[..., :3])


def test_gpu_render_rejects_oversized_images():
    sb, st = render_scene(n=100)
    with Simulation(config_from_spherebin(sb)) as sim:
        sim.upload(st)
        with pytest.raises(SphError) as e:
            sim.render(0, 1.0, 0.0, 8192, 4096)
        assert e.value.code == -8
