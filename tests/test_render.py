"""The ray tracer (src/raytracer.cuh, DEM::render) on the CPU: the oracle's
restatement pinned to the reference's own kernels, pixel for pixel."""
import numpy as np
import pytest

from sphere_b200 import scenes
from sphere_b200.state import state_from_spherebin

# (method, maxval, lower cutoff, width, height): square, wide (the
# reference's integer height/width collapses the rows), tall (its row index
# wraps modulo the width), every colour map, and the cutoff filter
CASES = [
    (0, 1.0e3, 0.0, 96, 96),
    (1, 50.0, 0.0, 80, 80),
    (2, 0.5, 0.0, 120, 72),
    (3, 300.0, 0.0, 64, 100),
    (4, 1e-4, 0.0, 72, 72),
    (5, 1.0, 0.0, 72, 72),
    (2, 0.5, 0.25, 96, 96),
]


def render_scene(seed=71, n=700):
    sb = scenes.collision(n=n, seed=seed, periodic=0, vmax=0.5, wmax=300.0)
    st = state_from_spherebin(sb)
    rng = np.random.default_rng(seed)
    st.p[:] = rng.uniform(0.0, 100.0, st.p.shape)
    st.xysum[:, 0] = rng.normal(0.0, 1e-4, sb.np)
    st.angpos[:, :3] = rng.normal(0.0, 0.5, (sb.np, 3))
    st.vel[::13, 3] = 1.0   # some fixed particles: grey, and left out under a cutoff
    return sb, st


@pytest.mark.parametrize("case", CASES, ids=[f"m{c[0]}_{c[3]}x{c[4]}_cut{c[2]}" for c in CASES])
def test_restatement_matches_reference_render_kernels(oracle_libs, case):
    if "ref" not in oracle_libs:
        pytest.skip("reference harness not built (reference checkout absent)")
    import pyoracle
    method, maxval, cut, w, h = case
    sb, st = render_scene()
    a, _ = pyoracle.render(oracle_libs["orc"], oracle_libs["orc"], st, sb.L, method, maxval, cut,
                           w, h, nthreads=4)
    b, _ = pyoracle.render(oracle_libs["ref"], oracle_libs["orc"], st, sb.L, method, maxval, cut,
                           w, h, nthreads=4)
    assert np.array_equal(a[..., :3], b[..., :3])
    hit = (a[..., :3] != 255).any(axis=2)
    assert hit.sum() > 50 and (~hit).sum() > 50   # spheres and background both present
