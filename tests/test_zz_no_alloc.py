"""sph_cell_list_noalloc: the cell list for callers that cannot allocate
device memory (a plugin host that owns the device memory pool, or a loop
that must not pay cudaMalloc's device-wide synchronisation).

The entry point takes device-resident positions and device outputs from the
caller and uses only a fixed scratch array inside the library.  It must give
the same cell list as the allocating path (a context's sph_get_cells for the
same positions), bit for bit, on consecutive calls: the shared scratch keeps
the previous call's contents and each call must clear what it needs."""
import ctypes as C

import numpy as np
import pytest

from sphere_b200 import scenes, sphk
from sphere_b200.sphk import SphError, Simulation
from sphere_b200.state import config_from_spherebin, state_from_spherebin

pytestmark = pytest.mark.gpu


def _noalloc(lib, cfg, x_dev, np_, ncells, torch):
    outs = [torch.full((n,), 7, dtype=torch.int32, device="cuda") for n in (np_, np_, ncells, ncells)]
    conf = sphk.make_config(cfg)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.sph_cell_list_noalloc(C.byref(conf), C.c_void_p(x_dev.data_ptr()),
                                   *(C.c_void_p(o.data_ptr()) for o in outs), C.c_void_p(stream))
    assert rc == 0
    torch.cuda.synchronize()
    return [o.cpu().numpy().view(np.uint32) for o in outs]


def _outside_and_nan():
    # particles past every face of the grid, a crowd in one far bucket, and
    # positions that are not finite: they all share the out-of-grid bucket,
    # members in particle order
    sb = scenes.collision(n=2000, seed=74, periodic=0)
    rng = np.random.default_rng(75)
    sel = rng.choice(sb.np, 400, replace=False)
    for j, i in enumerate(sel):
        ax = j % 3
        sb.x[i, ax] = (sb.L[ax] + 0.01 * (1 + j)) if (j // 3) % 2 == 0 else -0.01 * (1 + j)
    sb.x[sel[:7], 2] = np.nan
    sb.x[sel[7], 0] = np.inf
    return sb


def _one_dense_cell():
    # a coarse grid: most particles in a handful of cells
    sb = scenes.collision(n=3000, seed=76, periodic=0)
    sb.num = np.array([2, 1, 2], dtype=sb.num.dtype)
    return sb


@pytest.mark.parametrize("builder", [
    lambda: scenes.collision(n=3000, seed=71, periodic=1),
    lambda: scenes.collision(n=2500, seed=72, periodic=0, nw=1),
    _outside_and_nan,
    _one_dense_cell,
], ids=["periodic", "box_wall", "outside_and_nan", "dense_cells"])
def test_noalloc_cell_list_matches_context_path(builder):
    torch = pytest.importorskip("torch")
    sb = builder()
    cfg = config_from_spherebin(sb)
    st = state_from_spherebin(sb)
    with Simulation(cfg) as sim:
        try:
            sim.upload(st)
        except SphError as e:
            # the context reports positions outside the grid, and still
            # holds their cell list
            assert sphk.ERRORS[e.code] == "SPH_ERR_OUT_OF_GRID"
        want = sim.cells()
    lib = sphk.load_library()
    x_dev = torch.tensor(st.x, dtype=torch.float64, device="cuda").contiguous()
    dev_before = torch.cuda.current_device()
    first = _noalloc(lib, cfg, x_dev, cfg.np, cfg.ncells, torch)
    second = _noalloc(lib, cfg, x_dev, cfg.np, cfg.ncells, torch)
    assert torch.cuda.current_device() == dev_before
    for got in (first, second):
        for g, w, name in zip(got, want, ("cell_sorted", "perm", "cell_start", "cell_end")):
            assert np.array_equal(g, w), name


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = sphk.load_library()
    sb = scenes.collision(n=100, seed=73)
    conf = sphk.make_config(config_from_spherebin(sb))
    conf.np = sphk_max = 1048576 + 1
    dummy = C.c_void_p(1)
    assert lib.sph_cell_list_noalloc(C.byref(conf), dummy, dummy, dummy, dummy, dummy, None) == -8
    conf.np = 100
    conf.num[0], conf.num[1], conf.num[2] = 1024, 1024, 1
    assert lib.sph_cell_list_noalloc(C.byref(conf), dummy, dummy, dummy, dummy, dummy, None) == -8
    assert sphk_max > 1048576
