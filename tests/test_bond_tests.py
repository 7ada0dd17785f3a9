"""Restatement of the reference's two-particle bond test (tests/bond_tests.py:
15-91): two spheres of radius 0.5 joined by one bond, at a gap of 0.2 radii
and touching, with no damping.

- Stability: at rest, the state stays at rest and the total energy (kinetic +
  rotational + bond potential) stays zero.
- Normal expansion: particle 1 moves away along x at 1e-4 m/s; energy is
  conserved to 1e-5 (compareFloats, tests/pytestutils.py:21) and both
  particles end with positive x velocity, zero y/z velocity and no spin.

The runs follow the reference workflow: write the input file, run the
schedule of DEM::startTime, read the last output file.  On the CPU the oracle
steps the schedule; on the GPU the `sphere` executable runs it, and its last
output must equal the oracle's byte for byte."""
import subprocess

import numpy as np
import pytest

from sphere_b200 import build, driver
from sphere_b200.spherebin import Spherebin, readbin
from sphere_b200.state import config_from_spherebin, state_from_spherebin, to_spherebin

RADIUS = 0.5


def bond_scene(gap, case):
    sb = Spherebin(np_=2, sid=f"bondtest_{case}_{int(gap * 10)}")
    sb.x[0, :] = (10.0, 10.0, 10.0)
    sb.x[1, :] = (10.0 + 2.0 * RADIUS + gap, 10.0, 10.0)
    sb.radius = np.ones(sb.np) * RADIUS
    sb.initGridAndWorldsize(margin=10, periodic=1, contactmodel=2, g=np.array([0.0, 0.0, 0.0]))
    sb.bond(0, 1)
    sb.defaultParams(gamma_n=0.0, gamma_t=0.0)
    sb.zeroKinematics()
    sb.initTemporal(total=0.2, file_dt=0.01)
    if case == "expansion":
        sb.vel[1, 0] = 1e-4
    return sb


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


def total_energy(sb):
    return sb.energy("kin") + sb.energy("rot") + sb.energy("bondpot")


def check_case(case, sb0, last):
    z2_3 = np.zeros((2, 3))
    if case == "stability":
        assert abs(0.0 - total_energy(last)) < 1e-5
        assert np.array_equal(last.vel, z2_3)
        assert np.array_equal(last.angvel, z2_3)
    else:
        e0 = sb0.energy("kin") + sb0.energy("rot")
        assert abs(e0 - total_energy(last)) < 1e-5
        assert last.vel[0, 0] > 0.0 and last.vel[1, 0] > 0.0
        assert np.array_equal(last.vel[:, 1:2], np.zeros((2, 1)))
        assert np.array_equal(last.angvel, z2_3)


CASES = [(gap, case) for gap in (0.2, 0.0) for case in ("stability", "expansion")]


@pytest.mark.parametrize("gap, case", CASES)
def test_bond_oracle(oracle_libs, gap, case, tmp_path):
    sb = bond_scene(gap, case)
    last, outs, total = driver.run(sb, _OracleStepper(oracle_libs["orc"], bond_scene(gap, case)),
                                   outdir=tmp_path / "output")
    assert len(outs) >= 19 and total > 2000
    check_case(case, sb, last)


@pytest.mark.gpu
@pytest.mark.parametrize("gap, case", CASES)
def test_bond_cli(oracle_libs, gap, case, tmp_path):
    """Spherebin.run() on the built executable, then readlast()."""
    build.build_cli()
    sb = bond_scene(gap, case)
    (tmp_path / "input").mkdir()
    (tmp_path / "output").mkdir()
    sb.writebin(folder=tmp_path / "input", verbose=False)
    assert sb.run(verbose=False, root=tmp_path) == 0
    last = Spherebin(sid=sb.sid)
    last.readlast(verbose=False, root=tmp_path)
    check_case(case, sb, last)
    want, _, _ = driver.run(sb, _OracleStepper(oracle_libs["orc"], bond_scene(gap, case)),
                            outdir=tmp_path / "want")
    assert last.to_bytes() == want.to_bytes()


def test_run_dry_through_spherebin(tmp_path):
    """Spherebin.run(dry=True) reaches the executable and returns its status."""
    build.build_cli()
    sb = bond_scene(0.2, "stability")
    (tmp_path / "input").mkdir()
    sb.writebin(folder=tmp_path / "input", verbose=False)
    assert sb.run(verbose=False, dry=True, root=tmp_path, hideinputfile=True) == 0
    r = subprocess.run([str(build.CLI), "-n", f"input/{sb.sid}.bin"], cwd=tmp_path,
                       capture_output=True, text=True)
    assert "No. of particle bonds: 1" in r.stdout
    assert readbin(tmp_path / "input" / f"{sb.sid}.bin") == sb
