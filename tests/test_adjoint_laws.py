"""The reverse (adjoint) passes of the differentiable contact laws
(sphere_b200/csrc/diff_law.h) against central differences of their forward
passes, on the host: for random output adjoints b and every input u,
sum(b * (f(u + h) - f(u - h)) / 2h) must equal the reverse pass's adjoint
of u, in both friction branches (sticking and sliding)."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
HERE = Path(__file__).resolve().parent


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    out = tmp_path_factory.mktemp("difflaw") / "libdifflaw_check.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared",
                    "-I", str(ROOT / "sphere_b200" / "csrc"), str(HERE / "difflaw_check.cpp"),
                    "-o", str(out)], check=True)
    lib = C.CDLL(str(out))
    dp = C.POINTER(C.c_double)
    for name, n in (("pair_fwd_c", 3), ("pair_rev_c", 5), ("wall_fwd_c", 3), ("wall_rev_c", 4)):
        getattr(lib, name).argtypes = [dp] * n
        getattr(lib, name).restype = None
    return lib


def _p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))


def pair_fwd(lib, law, x):
    out = np.zeros(9)
    lib.pair_fwd_c(_p(law), _p(x), out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def _pair_case(rng, slip):
    ra, rb = rng.uniform(0.9e-3, 1.1e-3, 2)
    overlap = rng.uniform(1e-6, 2e-5)
    d = rng.normal(size=3)
    d /= np.linalg.norm(d)
    xab = d * (ra + rb - overlap)
    va, vb = rng.normal(scale=0.05, size=(2, 3))
    wa, wb = rng.normal(scale=20.0, size=(2, 3))
    d0u = rng.normal(scale=2e-6, size=3)
    law = np.array([1e5, 8e4, 0.5, 0.1, 0.05 if slip else 5.0, 0.0, 1e-6])
    x = np.concatenate([xab, [ra, rb], va, vb, wa, wb, d0u])
    return law, x


# input slots of the 20-double vector that the reverse returns adjoints for
IN_SLOTS = list(range(0, 3)) + list(range(5, 20))


@pytest.mark.parametrize("slip", [False, True], ids=["sticking", "sliding"])
@pytest.mark.parametrize("seed", range(4))
def test_pair_reverse_matches_central_differences(lib, slip, seed):
    rng = np.random.default_rng(100 + seed)
    law, x = _pair_case(rng, slip)
    bars = rng.normal(size=9) * np.r_[np.ones(6), np.full(3, 1e5)]
    inbar = np.zeros(18)
    lawbar = np.zeros(4)
    lib.pair_rev_c(_p(law), _p(x), _p(bars), inbar.ctypes.data_as(C.POINTER(C.c_double)),
                   lawbar.ctypes.data_as(C.POINTER(C.c_double)))
    # confirm the branch: sliding means |f_t| reached mu |f_n|
    fd = []
    for k in IN_SLOTS:
        h = 1e-6 * max(abs(x[k]), 1e-9 if k < 3 else (1e-3 if k < 11 else 1e-2))
        if k >= 17:
            h = 1e-6 * max(abs(x[k]), 1e-7)
        xp, xm = x.copy(), x.copy()
        xp[k] += h
        xm[k] -= h
        fd.append(bars @ (pair_fwd(lib, law, xp) - pair_fwd(lib, law, xm)) / (2 * h))
    fd = np.array(fd)
    scale = np.abs(fd).max()
    assert np.abs(inbar - fd).max() <= 1e-5 * scale, np.c_[inbar, fd]
    for j, k in enumerate((0, 1, 2, 4)):   # kn kt gn mu
        h = 1e-6 * law[k]
        lp, lm = law.copy(), law.copy()
        lp[k] += h
        lm[k] -= h
        g = bars @ (pair_fwd(lib, lp, x) - pair_fwd(lib, lm, x)) / (2 * h)
        assert abs(lawbar[j] - g) <= 1e-5 * max(abs(g), 1e-12 * scale) + 1e-9 * abs(g) + 1e-30, (j, lawbar[j], g)


@pytest.mark.parametrize("case", ["sticking", "sliding", "normal_only"])
def test_wall_reverse_matches_central_differences(lib, case):
    rng = np.random.default_rng({"sticking": 1, "sliding": 2, "normal_only": 3}[case])
    ra = 1e-3
    va = rng.normal(scale=0.05, size=3)
    wa = rng.normal(scale=20.0, size=3)
    if case == "normal_only":
        va[:] = 0.0
        wa[:] = 0.0
    w = np.array([1e5, 0.5, 0.05 if case == "sticking" else 50.0, 0.5, 0.5])
    q = np.concatenate([[ra], va, wa, [0.0, 0.0, 1.0], [-1e-5], [0.0]])
    bars = rng.normal(size=6)
    out = np.zeros(8)
    lib.wall_rev_c(_p(w), _p(q), _p(bars), out.ctypes.data_as(C.POINTER(C.c_double)))

    def f(qq, ww=w):
        o = np.zeros(6)
        lib.wall_fwd_c(_p(ww), _p(qq), o.ctypes.data_as(C.POINTER(C.c_double)))
        return o

    fd = []
    for k in list(range(1, 7)) + [10]:
        h = 1e-6 * max(abs(q[k]), 1e-3 if k < 4 else (1e-2 if k < 7 else 1e-7))
        qp, qm = q.copy(), q.copy()
        qp[k] += h
        qm[k] -= h
        fd.append(bars @ (f(qp) - f(qm)) / (2 * h))
    got = out[:7]
    fd = np.array(fd)
    assert np.abs(got - fd).max() <= 1e-5 * np.abs(fd).max(), np.c_[got, fd]
    h = 1e-6 * w[0]
    wp, wm = w.copy(), w.copy()
    wp[0] += h
    wm[0] -= h
    g = bars @ (f(q, wp) - f(q, wm)) / (2 * h)
    assert abs(out[7] - g) <= 1e-5 * abs(g)
