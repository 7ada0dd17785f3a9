"""The reference binary state format (src/file_io.cpp:29-490,
python/sphere.py:254-529): byte-exact round trips and input validation."""
import numpy as np
import pytest

from sphere_b200 import scenes
from sphere_b200.spherebin import Spherebin, readbin


def _expected_size(sb):
    n, nw, nb0 = sb.np, sb.nw, sb.nb0
    return (4 + 4 + 4 * 8 + 4 + 3 * 8 * 2 + 3 * 4 + 4 + n * (4 + 2 + 4 + 3 * 4 + 5) * 8
            + (3 + 14) * 8 + 4 + 3 * 8 + 4 + nw * 4 + nw * 8 * 8 + 3 * 8 + 4 + 2 * 8
            + nb0 * 8 + nb0 * 8 * 8 + 8)


@pytest.mark.parametrize("builder", [
    lambda: scenes.collision(n=300, seed=3, nw=1),
    lambda: scenes.settling(nx=5, ny=4, nz=3),
    lambda: scenes.bonded(nx=3, ny=2, nz=2),
])
def test_roundtrip_is_byte_exact(builder, tmp_path):
    sb = builder()
    raw = sb.to_bytes()
    assert len(raw) == _expected_size(sb)
    path = sb.writebin(path=tmp_path / "a.bin", verbose=False)
    back = readbin(path)
    assert back.to_bytes() == raw
    assert back == sb
    np.testing.assert_array_equal(back.x, sb.x)
    np.testing.assert_array_equal(back.bonds, sb.bonds)


def test_python_io_restates_reference_io_test(tmp_path):
    # tests/io_tests.py:8-21: build a scene, write, read back, compare
    orig = Spherebin(np_=100, nw=1, sid="test-initgrid")
    rng = np.random.default_rng(0)
    orig.generateRadii(rng=rng)
    orig.defaultParams()
    orig.initRandomGridPos(g=np.zeros(3), rng=rng)
    orig.initTemporal(current=0.0, total=0.0)
    orig.time_total = 2.0 * orig.time_dt
    orig.time_file_dt = orig.time_dt
    orig.writebin(folder=tmp_path, verbose=False)
    py = Spherebin()
    py.readbin(tmp_path / "test-initgrid.bin", verbose=False)
    assert py == orig


def test_truncated_file_is_rejected():
    raw = scenes.collision(n=50, seed=1).to_bytes()
    with pytest.raises(ValueError, match="truncated"):
        Spherebin.from_bytes(raw[:-9])


def test_too_many_walls_is_rejected():
    sb = scenes.collision(n=20, seed=1)
    raw = bytearray(sb.to_bytes())
    # nw sits after the 14 + 3 parameter doubles, g and contactmodel
    n = sb.np
    off = 4 + 4 + 32 + 4 + 48 + 12 + 4 + n * 27 * 8 + 24 + 14 * 8 + 4 + 24
    assert int.from_bytes(raw[off:off + 4], "little") == sb.nw
    raw[off:off + 4] = (7).to_bytes(4, "little")
    with pytest.raises(ValueError, match="MAXWALLS"):
        Spherebin.from_bytes(bytes(raw))


def test_wrong_dimensionality_is_rejected():
    raw = bytearray(scenes.collision(n=10, seed=1).to_bytes())
    raw[0:4] = (2).to_bytes(4, "little")
    with pytest.raises(ValueError, match="dimensionality"):
        Spherebin.from_bytes(bytes(raw))
