"""The ``sphere`` executable and the ``DEM`` class (src/main.cpp:27-182,
src/sphere.cpp:16-341, src/device.cu:576-1299) built over the C ABI.

CPU tests cover the command line and the pre-flight checks, which end before
any device work.  The GPU test runs a scene through the executable and checks
every output file and status.dat byte for byte against the same schedule
driven through the oracle."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from sphere_b200 import build, driver, scenes
from sphere_b200.spherebin import readbin
from sphere_b200.state import config_from_spherebin, state_from_spherebin, to_spherebin


@pytest.fixture(scope="module")
def cli():
    return build.build_cli()


def _run(cli, args, cwd):
    return subprocess.run([str(cli)] + [str(a) for a in args], cwd=cwd, capture_output=True,
                          text=True, timeout=600)


def _scene(tmp_path, sid="cli", **kw):
    sb = scenes.collision(n=kw.pop("n", 400), seed=kw.pop("seed", 51), **kw)
    sb.sid = sid
    sb.time_current = 0.0
    sb.time_total = 23.0 * sb.time_dt
    sb.time_file_dt = 5.0 * sb.time_dt
    sb.time_step_count = 0
    (tmp_path / "output").mkdir(exist_ok=True)
    return sb, sb.writebin(path=tmp_path / f"{sid}.bin", verbose=False)


def test_help_and_version(cli, tmp_path):
    r = _run(cli, ["--help"], tmp_path)
    assert r.returncode == 0 and "--dry" in r.stdout
    r = _run(cli, ["-V"], tmp_path)
    assert r.returncode == 0 and "ABI version" in r.stdout


def test_missing_input_file_argument(cli, tmp_path):
    r = _run(cli, [], tmp_path)
    assert r.returncode == 1 and "missing input binary file" in r.stderr


def test_unreadable_input_file(cli, tmp_path):
    r = _run(cli, ["-q", tmp_path / "nothere.bin"], tmp_path)
    assert r.returncode == 1 and "Could not read input binary file" in r.stderr


def test_render_flags_need_an_input_file(cli, tmp_path):
    r = _run(cli, ["--render"], tmp_path)
    assert r.returncode == 1 and "missing input binary file" in r.stderr
    r = _run(cli, ["--method", "colour", "--render"], tmp_path)
    assert r.returncode == 1 and "Visualization method not understood" in r.stderr


def test_dry_run_reports_parameters(cli, tmp_path):
    sb, path = _scene(tmp_path, nw=1)
    r = _run(cli, ["--dry", path], tmp_path)
    assert r.returncode == 0, r.stderr
    assert f"np = {sb.np}" in r.stdout
    assert "Linear-elastic-visco-frictional" in r.stdout
    assert "Number of dynamic walls: 1" in r.stdout
    assert not any((tmp_path / "output").iterdir())


def test_particle_outside_grid_is_rejected(cli, tmp_path):
    sb, _ = _scene(tmp_path)
    sb.x[3, 0] = sb.L[0] * 1.5
    path = sb.writebin(path=tmp_path / "bad.bin", verbose=False)
    r = _run(cli, ["-q", path], tmp_path)
    assert r.returncode == 1 and "outside of the computational grid" in r.stderr


def test_nonpositive_stiffness_is_rejected(cli, tmp_path):
    sb, _ = _scene(tmp_path)
    sb.k_n = 0.0
    path = sb.writebin(path=tmp_path / "bad.bin", verbose=False)
    r = _run(cli, ["-q", path], tmp_path)
    assert r.returncode == 1 and "k_n" in r.stderr


def test_dont_check_skips_the_checks(cli, tmp_path):
    sb, _ = _scene(tmp_path)
    sb.k_n = 0.0
    path = sb.writebin(path=tmp_path / "bad.bin", verbose=False)
    r = _run(cli, ["-q", "-dc", "-n", path], tmp_path)
    assert r.returncode == 0


def test_schedule_matches_a_literal_restatement():
    """driver.schedule against the reference loop written out step by step
    (src/device.cu:731,1109-1110,1123,1187), float file clock included."""
    for cur, tot, dt, fdt in [(0.0, 23e-6, 1e-6, 5e-6), (0.0, 1e-3, 3.3e-7, 1e-4),
                              (2e-6, 2e-6, 1e-6, 1e-6), (0.0, 1e-5, 1e-6, 0.0)]:
        t, ftc, step, outs = cur, np.float32(0.0), 0, []
        while t <= tot:
            step += 1
            t += dt
            ftc = np.float32(float(ftc) + dt)
            if float(ftc) >= fdt:
                outs.append(step)
                ftc = np.float32(0.0)
        got_outs, got_total, _ = driver.schedule(cur, tot, dt, fdt)
        assert got_outs == outs and got_total == step


class _OracleStepper:
    def __init__(self, lib, sb):
        import pyoracle
        self.sb = sb
        self.st = state_from_spherebin(sb)
        self.run = pyoracle.OracleRun(lib, config_from_spherebin(sb), self.st)

    def __call__(self, n):
        assert self.run.step(n, 0) == 0

    def snapshot(self):
        return to_spherebin(self.sb, self.st)


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(periodic=1), dict(periodic=0, nw=1)],
                         ids=["periodic", "wall"])
def test_cli_run_writes_the_oracles_files(cli, oracle_libs, tmp_path, kw):
    sb, path = _scene(tmp_path, **kw)
    r = _run(cli, ["-q", path], tmp_path)
    assert r.returncode == 0, r.stderr
    want_dir = tmp_path / "want"
    driver.run(readbin(path), _OracleStepper(oracle_libs["orc"], readbin(path)), outdir=want_dir)
    got = sorted(p.name for p in (tmp_path / "output").iterdir())
    want = sorted(p.name for p in want_dir.iterdir())
    assert got == want and len(got) >= 5
    assert (tmp_path / "output" / "cli.output00000.bin").read_bytes() == path.read_bytes()
    for name in want:
        assert (tmp_path / "output" / name).read_bytes() == (want_dir / name).read_bytes(), name


@pytest.mark.gpu
@pytest.mark.parametrize("flags,method,maxval,cut", [
    (["--render"], 0, 0.0, 0.0),
    (["--method", "vel", "0.4", "-l", "0.1", "--render"], 2, 0.4, 0.1),
], ids=["normal", "vel_cutoff"])
def test_cli_render_writes_the_oracles_image(cli, oracle_libs, tmp_path, flags, method, maxval,
                                             cut):
    """sphere [-m ...] --render <file>: img_out/<sid>.ppm, 800 x 800 P6, byte
    for byte against the oracle's image of the file's state."""
    import pyoracle
    sb, path = _scene(tmp_path, sid="rt", n=900, seed=53)
    (tmp_path / "img_out").mkdir()
    r = _run(cli, ["-q"] + flags + [path.name], tmp_path)
    assert r.returncode == 0, r.stderr
    st = state_from_spherebin(readbin(path))
    img, _ = pyoracle.render(oracle_libs["orc"], oracle_libs["orc"], st, sb.L, method, maxval, cut,
                             800, 800)
    want = b"P6 800 800 255\n" + np.ascontiguousarray(img[..., :3]).tobytes()
    assert (tmp_path / "img_out" / "rt.ppm").read_bytes() == want
