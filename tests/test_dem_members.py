"""The DEM class's analysis members and Darcy array printers
(src/sphere.cpp:487-602, src/darcy.cpp:483-528,801-824) on the host state,
against the reference's algorithms written out with numpy: minPos/maxPos
from 0, findOverlaps over every pair i < j in (i, j) order with its
arithmetic, and the printers' text layout."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from sphere_b200.spherebin import Spherebin

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def driver(sphk_lib, tmp_path_factory):
    from sphere_b200 import build
    host = ROOT / "sphere_b200" / "csrc" / "host"
    out = tmp_path_factory.mktemp("members") / "dem_members_driver"
    cmd = ["g++", "-O2", "-std=c++17", "-I", str(ROOT / "include"), "-I", str(host),
           str(host / "sphere.cpp"), str(host / "file_io.cpp"),
           str(Path(__file__).resolve().parent / "dem_members_driver.cpp"), "-o", str(out),
           "-L", str(build.LIB.parent), "-lsphk", f"-Wl,-rpath,{build.LIB.parent}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


def scene(n=600, seed=5):
    """Random spheres in a small box, so that many overlap; one coincident
    pair, one particle with a NaN coordinate, one with negative coordinates
    and one of radius zero."""
    rng = np.random.default_rng(seed)
    sb = Spherebin(np_=n, nw=0, sid="members")
    sb.x = rng.uniform(0.0, 0.02, size=(n, 3))
    sb.radius = rng.uniform(0.5e-3, 1.5e-3, n)
    sb.x[7] = sb.x[3]
    sb.x[11, 1] = np.nan
    sb.x[20] = (-0.003, -0.001, -0.002)
    sb.radius[30] = 0.0
    sb.origo = np.zeros(3)
    sb.L = np.array([0.02, 0.02, 0.02])
    sb.num = np.array([6, 5, 4], dtype=np.uint32)
    return sb


def expected_overlaps(x, r):
    n = len(r)
    out = []
    for i in range(n - 1):
        d = x[i + 1:] - x[i]
        ln = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
        delta = ln - (r[i] + r[i + 1:])
        for k in np.nonzero(delta < 0.0)[0]:
            out.append((i, i + 1 + int(k), float(delta[k])))
    return out


def darcy_text(arr, num, vec=False):
    nx, ny, nz = (int(v) for v in num)
    lines = []
    for z in range(nz):
        for y in range(ny):
            row = ""
            for xx in range(nx):
                k = (xx + 1) + (nx + 2) * (y + 1) + (nx + 2) * (ny + 2) * (z + 1)
                row += ("%f,%f,%f\t" % tuple(arr[k]) if vec else "%f\t" % arr[k])
            lines.append(row + "\n")
        lines.append("\n")
    return "".join(lines)


def test_analysis_members_and_darcy_printers(driver, tmp_path):
    sb = scene()
    path = sb.writebin(path=tmp_path / "members.bin", verbose=False)
    nodes = int(np.prod(sb.num.astype(np.int64) + 2))
    r = subprocess.run([str(driver), str(path), str(tmp_path), str(nodes)], cwd=tmp_path,
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr

    x, rad = sb.x.astype(np.float64), sb.radius.astype(np.float64)
    lo = [0.0, 0.0, 0.0]
    hi = [0.0, 0.0, 0.0]
    for i in range(sb.np):
        for d in range(3):
            v = x[i, d]
            lo[d] = v if v < lo[d] else lo[d]
            hi[d] = v if v > hi[d] else hi[d]
    got = (tmp_path / "minmax.txt").read_text().split()
    assert [float(v) for v in got] == lo + hi
    assert lo[0] == -0.003 and np.isfinite(hi[1])

    want = expected_overlaps(x, rad)
    rows = (tmp_path / "overlaps.txt").read_text().splitlines()
    assert len(rows) == len(want) and len(want) > 100
    for row, (i, j, d) in zip(rows, want):
        a, b, dd = row.split()
        assert (int(a), int(b)) == (i, j)
        assert float(dd) == d            # %.17g round-trips a double exactly
    assert any(i == 3 and j == 7 for i, j, _ in want)
    assert not any(11 in (i, j) for i, j, _ in want)

    k = np.arange(nodes, dtype=np.uint64)
    s = ((k * np.uint64(2654435761)) % np.uint64(1000003)).astype(np.float64) / 1000.0 - 500.0
    v = np.stack([s, -0.5 * s, 0.25 * k.astype(np.float64)], axis=1)
    assert (tmp_path / "scalar.txt").read_text() == darcy_text(s, sb.num)
    assert (tmp_path / "vector.txt").read_text() == darcy_text(v, sb.num, vec=True)
    assert r.stdout == "\nscalar field:\n" + darcy_text(s, sb.num)
