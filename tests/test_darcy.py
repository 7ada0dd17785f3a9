"""Darcy flow (src/darcy.cuh, src/darcy.cpp) on the CPU: the oracle's
restatement pinned to the reference's own Darcy kernels, and the host-side
initialisation (sph_darcy_init) against the reference's per-cell loops."""
import math

import numpy as np
import pytest

from helpers import STATE_FIELDS, mismatches
from sphere_b200 import scenes
from sphere_b200.darcy import DarcyState
from sphere_b200.state import config_from_spherebin, state_from_spherebin

DARCY_FIELDS = ("H", "H_new", "V", "dH", "K", "T", "Ss", "W", "phi", "dphi")
NU = 8.9e-4   # water, Pa s

SCENES = {
    "box": lambda: scenes.collision(n=900, seed=41, periodic=0),
    # clusters across the periodic faces: the porosity stencil wraps and
    # shifts positions by +-L
    "periodic_xy": lambda: scenes.collision(n=900, seed=42, periodic=1, straddle=True),
    "periodic_x": lambda: scenes.collision(n=900, seed=43, periodic=2, straddle=True),
    # a dynamic top wall beside the flow (the wall kernel runs in the same step)
    "box_wall": lambda: scenes.collision(n=900, seed=45, periodic=0, nw=1),
    # 1 cm cells: about 2500 particles in the 6 x 6 x 6 cells around a
    # porosity tile, more than its shared-memory stage holds, so the GPU walks
    # them in global memory; the second tile of each axis is partial
    "dense_cells": lambda: _coarse(scenes.collision(n=2500, seed=46, periodic=1), 6),
}


def _coarse(sb, cells):
    sb.num = np.full(3, cells, dtype=np.uint32)
    return sb


def seeded_grid(num, seed):
    """A fluid grid with every node of every field set (ghosts included), so
    that every copy and every read is visible in the results."""
    rng = np.random.default_rng(seed)
    ds = DarcyState.zeros(num)
    n = ds.H.size
    ds.H[:] = rng.uniform(9.0e3, 1.1e4, n)
    ds.H_new[:] = rng.uniform(9.0e3, 1.1e4, n)
    ds.V[:] = rng.normal(0.0, 1e-6, (n, 3))
    ds.dH[:] = rng.normal(0.0, 1.0, (n, 3))
    ds.phi[:] = rng.uniform(0.2, 0.8, n)
    ds.dphi[:] = rng.normal(0.0, 1e-3, n)
    ds.K[:] = rng.uniform(1e-9, 1e-8, n)
    ds.T[:] = rng.uniform(1e-12, 1e-11, (n, 3))
    ds.Ss[:] = rng.uniform(0.5, 1.5, n)
    ds.W[:] = rng.normal(0.0, 1e-3, n)
    return ds


def d_factor_of(sb):
    """src/device.cu:673-678 from the mean radius (summed in particle order)"""
    r_sum = 0.0
    for r in sb.radius:
        r_sum += float(r)
    r_bar2 = r_sum / sb.np * 2.0
    return r_bar2 * r_bar2 / 180.0 * 1.0e-6


def run_darcy_oracle(lib, sb, nsteps, ds, nthreads=4, chunks=None):
    import pyoracle
    cfg = config_from_spherebin(sb)
    st = state_from_spherebin(sb)
    run = pyoracle.OracleRun(lib, cfg, st, darcy=ds, nu=NU, d_factor=d_factor_of(sb))
    rc = 0
    for n in (chunks or (nsteps,)):
        rc |= run.step(n, nthreads)
    return rc, st, ds


def darcy_mismatches(a: DarcyState, b: DarcyState):
    return [f for f in DARCY_FIELDS
            if getattr(a, f).tobytes() != getattr(b, f).tobytes()]


@pytest.mark.parametrize("name", sorted(SCENES))
def test_restatement_matches_reference_darcy_kernels(oracle_libs, name):
    if "ref" not in oracle_libs:
        pytest.skip("reference harness not built (reference checkout absent)")
    sb = SCENES[name]()
    cfg = config_from_spherebin(sb)
    start = seeded_grid(cfg.num, 7)
    rc1, sa, a = run_darcy_oracle(oracle_libs["orc"], sb, 25, start.copy())
    rc2, sb_, b = run_darcy_oracle(oracle_libs["ref"], sb, 25, start.copy())
    assert rc1 == 0 and rc2 == 0
    assert darcy_mismatches(a, b) == []
    # the particles are stepped as without the flow
    assert mismatches(sa, sb_, STATE_FIELDS) == []
    # both ran the flow: every cell's conductivity was recomputed from its
    # porosity, the pressure moved, and the ghost nodes were written
    for f in ("K", "phi", "H", "V", "dH"):
        changed = np.any(a.interior(f) != start.interior(f), axis=tuple(range(1, a.interior(f).ndim)))
        assert changed.all() if f in ("K", "phi") else changed.any(), f
    assert np.all(a.interior("phi") >= 0.1) and np.all(a.interior("phi") <= 0.9)
    assert (a.interior("phi") < 0.9).any() and np.count_nonzero(a.interior("dphi")) > 0
    nx, ny, nz = cfg.num
    ghost = a.node(nx, 1, 1)
    assert a.K[ghost] == a.K[a.node(0, 1, 1)]


def test_darcy_block_leaves_particles_unchanged(oracle_libs):
    """The flow is one-way: the particles' state after a run with it is
    bit for bit the state after the same run without it."""
    import pyoracle
    from helpers import run_oracle
    sb = SCENES["periodic_xy"]()
    _, with_flow, _ = run_darcy_oracle(oracle_libs["orc"], sb, 20, seeded_grid(sb.num, 3))
    _, without, _ = run_oracle(oracle_libs["orc"], sb, 20, nthreads=4)
    assert mismatches(with_flow, without, STATE_FIELDS) == []
    assert pyoracle.OrcScene  # the binding exposes the Darcy fields


def test_split_runs_equal_one_run(oracle_libs):
    """The pressure buffers' swap and the first-step rule carry across calls."""
    sb = SCENES["box"]()
    _, _, a = run_darcy_oracle(oracle_libs["orc"], sb, 21, seeded_grid(sb.num, 5))
    _, _, b = run_darcy_oracle(oracle_libs["orc"], sb, 21, seeded_grid(sb.num, 5),
                               chunks=(1, 6, 14))
    assert darcy_mismatches(a, b) == []


def test_first_step_leaves_porosity_change_zero(oracle_libs):
    sb = SCENES["box"]()
    _, _, a = run_darcy_oracle(oracle_libs["orc"], sb, 1, seeded_grid(sb.num, 9))
    assert np.all(a.interior("dphi") == 0.0)
    _, _, b = run_darcy_oracle(oracle_libs["orc"], sb, 2, seeded_grid(sb.num, 9))
    assert np.count_nonzero(b.interior("dphi")) > 0


# ---- host-side initialisation ------------------------------------------------

def init_reference_loops(cfg, nu, x, ds):
    """DEM::initDarcy (src/darcy.cpp:760-798) as the reference loops it: for
    every cell, every particle in index order (cellPorosity,
    src/darcy.cpp:600-627).  Small cases only."""
    nx, ny, nz = (int(v) for v in cfg.num)
    dx, dy, dz = cfg.L[0] / nx, cfg.L[1] / ny, cfg.L[2] / nz
    ds.Ss[:] = 1.0
    ds.W[:] = 0.0
    r_sum = 0.0
    for i in range(cfg.np):
        r_sum += float(x[i, 3])
    r_bar2 = r_sum / float(cfg.np) * 2.0 * 1.0e-6
    d_factor = r_bar2 * r_bar2 / 180.0
    vol = [4.0 / 3.0 * math.pi * float(r) * float(r) * float(r) for r in x[:, 3]]
    for ix in range(nx):
        for iy in range(ny):
            for iz in range(nz):
                lo = (ix * dx, iy * dy, iz * dz)
                hi = ((ix + 1) * dx, (iy + 1) * dy, (iz + 1) * dz)
                cv = dx * dy * dz
                void = cv
                inside = np.nonzero((x[:, 0] >= lo[0]) & (x[:, 1] >= lo[1]) & (x[:, 2] >= lo[2]) &
                                    (x[:, 0] < hi[0]) & (x[:, 1] < hi[1]) & (x[:, 2] < hi[2]))[0]
                for i in inside:
                    void -= vol[i]
                phi = min(0.99, max(0.01, void / cv))
                k = int(ds.node(ix, iy, iz))
                ds.phi[k] = phi
                kk = phi * phi * phi / ((1.0 - phi) * (1.0 - phi)) * d_factor
                K = kk * 1000.0 * -cfg.g[2] / nu
                ds.K[k] = K
                ds.T[k] = (K * dx, K * dy, K * dz)
                ds.dphi[k] = 0.0
    return ds


@pytest.mark.parametrize("name", ["box", "periodic_xy"])
def test_host_init_matches_reference_loops(sphk_lib, name):
    from sphere_b200.sphk import darcy_init
    sb = SCENES[name]()
    cfg = config_from_spherebin(sb)
    x = state_from_spherebin(sb).x
    # a few particles exactly on cell boundaries and outside the grid
    x = x.copy()
    dx = cfg.L[0] / cfg.num[0]
    x[0, 0] = 3 * dx
    x[1, 1] = 0.0
    x[2, 2] = -1e-4
    x[3, 0] = cfg.L[0]
    a = DarcyState.zeros(cfg.num)
    b = DarcyState.zeros(cfg.num)
    value = darcy_init(cfg, NU, x, a)
    init_reference_loops(cfg, NU, x, b)
    assert darcy_mismatches(a, b) == []
    assert 0.0 < value <= 0.5


def test_host_init_reports_an_unstable_step(sphk_lib):
    from sphere_b200.sphk import SphError, darcy_init
    sb = SCENES["box"]()
    cfg = config_from_spherebin(sb)
    cfg.dt = 1.0e6   # far beyond the explicit scheme's limit
    with pytest.raises(SphError) as e:
        darcy_init(cfg, NU, state_from_spherebin(sb).x, DarcyState.zeros(cfg.num))
    assert e.value.code == -9


def test_host_init_rejects_nonpositive_viscosity(sphk_lib):
    from sphere_b200.sphk import SphError, darcy_init
    sb = SCENES["box"]()
    cfg = config_from_spherebin(sb)
    with pytest.raises(SphError) as e:
        darcy_init(cfg, 0.0, state_from_spherebin(sb).x, DarcyState.zeros(cfg.num))
    assert e.value.code == -5


# ---- file format and the DEM class ---------------------------------------------

def darcy_scene(tmp_path=None, sid="darcy", nu=NU, n=500, seed=44, steps=23):
    """A settling scene with a fluid section: uniform pressure, zero velocity,
    porosity and conductivity to be set up by DEM::initDarcy."""
    sb = scenes.collision(n=n, seed=seed, periodic=1, vmax=0.3)
    sb.sid = sid
    sb.nu = nu
    sb.time_current = 0.0
    sb.time_total = steps * sb.time_dt
    sb.time_file_dt = 5.0 * sb.time_dt
    sb.time_step_count = 0
    ds = DarcyState.zeros(sb.num)
    shape = tuple(int(v) for v in sb.num)
    ds.set_cells(H=np.full(shape, 1.0e4), phi=np.full(shape, 0.5), K=np.full(shape, 1e-9))
    ds.to_spherebin(sb)
    path = None
    if tmp_path is not None:
        (tmp_path / "output").mkdir(exist_ok=True)
        path = sb.writebin(path=tmp_path / f"{sid}.bin", verbose=False)
    return sb, path


def test_fluid_section_round_trips_in_the_reference_layout():
    from sphere_b200.spherebin import Spherebin
    sb, _ = darcy_scene()
    rng = np.random.default_rng(3)
    shape = tuple(int(v) for v in sb.num)
    sb.f_v = rng.normal(size=shape + (3,))
    sb.f_rho, sb.f_phi, sb.f_K = (rng.normal(size=shape) for _ in range(3))
    raw = sb.to_bytes()
    back = Spherebin.from_bytes(raw)
    for f in ("f_v", "f_rho", "f_phi", "f_K"):
        assert np.array_equal(getattr(back, f), getattr(sb, f)), f
    # python/sphere.py:516-527: per cell, z outermost, V[3], H, phi, K
    want = []
    for z in range(shape[2]):
        for y in range(shape[1]):
            for x in range(shape[0]):
                want += list(sb.f_v[x, y, z]) + [sb.f_rho[x, y, z], sb.f_phi[x, y, z],
                                                  sb.f_K[x, y, z]]
    tail = np.frombuffer(raw[-8 * len(want):], np.float64)
    assert np.array_equal(tail, np.array(want))
    assert back == sb


@pytest.fixture(scope="module")
def darcy_driver(sphk_lib, tmp_path_factory):
    """tests/darcy_driver.cpp linked with the DEM class and libsphk."""
    import subprocess
    from pathlib import Path
    from sphere_b200 import build
    root = Path(__file__).resolve().parent.parent
    host = root / "sphere_b200" / "csrc" / "host"
    out = tmp_path_factory.mktemp("driver") / "darcy_driver"
    cmd = ["g++", "-O2", "-std=c++17", "-I", str(root / "include"), "-I", str(host),
           str(host / "sphere.cpp"), str(host / "file_io.cpp"),
           str(Path(__file__).resolve().parent / "darcy_driver.cpp"), "-o", str(out),
           "-L", str(build.LIB.parent), "-lsphk", f"-Wl,-rpath,{build.LIB.parent}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


def test_dem_class_refuses_an_unstable_darcy_step(darcy_driver, tmp_path):
    import subprocess
    sb, _ = darcy_scene()
    sb.time_dt = 1.0e6
    sb.time_total = 2.0e6
    path = sb.writebin(path=tmp_path / "unstable.bin", verbose=False)
    r = subprocess.run([str(darcy_driver), str(path), "0"], cwd=tmp_path, capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 1 and "explicit Darcy solution will be unstable" in r.stderr


def test_dem_class_sets_up_darcy_flow_without_a_device(darcy_driver, tmp_path):
    import subprocess
    _, path = darcy_scene(tmp_path)
    r = subprocess.run([str(darcy_driver), str(path), "0"], cwd=tmp_path, capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stderr
