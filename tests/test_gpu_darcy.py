"""Darcy flow on the GPU (sph_darcy_*), bit for bit against the oracle."""
import numpy as np
import pytest

from helpers import STATE_FIELDS, mismatches
from sphere_b200.darcy import DarcyState
from sphere_b200.sphk import SphError, Simulation, darcy_init
from sphere_b200.state import config_from_spherebin, state_from_spherebin
from test_darcy import (NU, SCENES, darcy_driver, darcy_mismatches, run_darcy_oracle,  # noqa: F401
                         seeded_grid)

pytestmark = pytest.mark.gpu


def run_gpu_darcy(sb, ds, chunks, profile=False, graph_steps=None):
    cfg = config_from_spherebin(sb)
    with Simulation(cfg, graph_steps=graph_steps) as sim:
        sim.upload(state_from_spherebin(sb))
        sim.darcy_upload(ds, NU)
        if profile:
            sim.set_profile(True)
        for n in chunks:
            sim.step(n)
        sim.sync()
        st = sim.download()
        out = sim.darcy_download()
        prof = sim.profile() if profile else None
    return st, out, prof


@pytest.mark.parametrize("name", sorted(SCENES))
@pytest.mark.parametrize("chunks", [(25,), (1, 7, 17)], ids=["one_call", "three_calls"])
def test_gpu_darcy_matches_oracle(oracle_libs, name, chunks):
    sb = SCENES[name]()
    start = seeded_grid(sb.num, 7)
    _, so, o = run_darcy_oracle(oracle_libs["orc"], sb, sum(chunks), start.copy())
    sg, g, _ = run_gpu_darcy(sb, start.copy(), chunks)
    assert darcy_mismatches(g, o) == []
    assert mismatches(sg, so, STATE_FIELDS) == []


@pytest.mark.parametrize("graph_steps", [1, 3, 8])
def test_gpu_darcy_graph_batching_and_profile_mode_agree(oracle_libs, graph_steps):
    """Graph lengths of both parities and the one-by-one profile launches
    keep the pressure buffers' roles."""
    sb = SCENES["periodic_xy"]()
    start = seeded_grid(sb.num, 11)
    _, _, o = run_darcy_oracle(oracle_libs["orc"], sb, 19, start.copy())
    _, g, _ = run_gpu_darcy(sb, start.copy(), (5, 14), graph_steps=graph_steps)
    assert darcy_mismatches(g, o) == []
    _, p, prof = run_gpu_darcy(sb, start.copy(), (19,), profile=True)
    assert darcy_mismatches(p, o) == []
    assert prof["darcy"] > 0.0 and prof["steps"] == 19


def test_gpu_darcy_from_host_initialisation(oracle_libs):
    """The reference's start: the file's cells (here zero velocity and a
    uniform pressure), then DEM::initDarcy on the host, then the flow."""
    sb = SCENES["box"]()
    cfg = config_from_spherebin(sb)
    ds = DarcyState.zeros(cfg.num)
    ds.set_cells(H=np.full(tuple(int(v) for v in cfg.num), 1.0e4))
    darcy_init(cfg, NU, state_from_spherebin(sb).x, ds)
    _, _, o = run_darcy_oracle(oracle_libs["orc"], sb, 30, ds.copy())
    _, g, _ = run_gpu_darcy(sb, ds.copy(), (30,))
    assert darcy_mismatches(g, o) == []
    assert np.count_nonzero(g.interior("V")) > 0


def test_gpu_darcy_is_refused_in_differentiable_mode():
    sb = SCENES["box"]()
    cfg = config_from_spherebin(sb)
    with Simulation(cfg) as sim:
        sim.upload(state_from_spherebin(sb))
        sim.diff_begin(checkpoint_every=10)
        with pytest.raises(SphError):
            sim.darcy_upload(seeded_grid(sb.num, 1), NU)


class _DarcyOracleStepper:
    """The oracle with the Darcy block, for sphere_b200.driver.run."""

    def __init__(self, lib, sb, ds):
        import pyoracle
        from test_darcy import d_factor_of
        self.sb, self.ds = sb, ds
        self.st = state_from_spherebin(sb)
        self.run = pyoracle.OracleRun(lib, config_from_spherebin(sb), self.st, darcy=ds, nu=NU,
                                      d_factor=d_factor_of(sb))

    def __call__(self, n):
        assert self.run.step(n, 0) == 0

    def snapshot(self):
        from sphere_b200.state import to_spherebin
        out = to_spherebin(self.sb, self.st)
        self.ds.to_spherebin(out)
        return out


def _darcy_text(ds, name):
    nx, ny, nz = ds.num
    cells = ds.cells(name)
    out = []
    for z in range(nz):
        for y in range(ny):
            out.append("".join("%f\t" % cells[x, y, z] for x in range(nx)) + "\n")
        out.append("\n")
    return "".join(out)


def test_dem_class_runs_the_darcy_flow(oracle_libs, darcy_driver, tmp_path):
    """DEM(..., darcyflow = 1): every output file (particles and fluid
    section) and the closing d_phi.txt / d_K.txt, byte for byte against the
    same schedule through the oracle."""
    import subprocess
    from sphere_b200 import driver
    from sphere_b200.spherebin import readbin
    from test_darcy import darcy_scene
    _, path = darcy_scene(tmp_path)
    r = subprocess.run([str(darcy_driver), str(path), "1"], cwd=tmp_path, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    # the reference writes output00000 after DEM::initDarcy
    sb0 = readbin(path)
    ds = DarcyState.from_spherebin(sb0)
    darcy_init(config_from_spherebin(sb0), NU, state_from_spherebin(sb0).x, ds)
    ds.to_spherebin(sb0)
    stepper = _DarcyOracleStepper(oracle_libs["orc"], sb0, ds)
    want_dir = tmp_path / "want"
    driver.run(sb0, stepper, outdir=want_dir)
    want = sorted(p.name for p in want_dir.iterdir())
    got = sorted(p.name for p in (tmp_path / "output").iterdir())
    assert got == want and len(got) >= 5
    for name in want:
        assert (tmp_path / "output" / name).read_bytes() == (want_dir / name).read_bytes(), name
    assert (tmp_path / "d_phi.txt").read_text() == _darcy_text(stepper.ds, "phi")
    assert (tmp_path / "d_K.txt").read_text() == _darcy_text(stepper.ds, "K")
    last = readbin(want_dir / [n for n in want if n.endswith(".bin")][-1])
    assert np.count_nonzero(last.f_v) > 0
