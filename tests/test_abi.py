"""The C ABI of libsphk (include/sphk.h): the library loads, exports every
declared entry point and rejects bad configurations before touching a GPU."""
import ctypes as C
import subprocess

import numpy as np
import pytest

from sphere_b200 import scenes, sphk
from sphere_b200.state import config_from_spherebin


def test_library_exports_every_declared_symbol(sphk_lib):
    names = sphk.exported_symbols()
    assert len(names) >= 14
    dyn = subprocess.run(["nm", "-D", "--defined-only", str(sphk.LIB_PATH)],
                         capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in dyn.splitlines() if ln.strip()}
    missing = [n for n in names if n not in exported]
    assert missing == []
    for n in names:
        assert getattr(sphk_lib, n) is not None


def test_version(sphk_lib):
    assert sphk_lib.sph_version() == 3


@pytest.mark.parametrize("patch, msg", [
    (dict(np=0), b"np must be positive"),
    (dict(nw=7), b"MAXWALLS"),
    (dict(contactmodel=0), b"contact model"),
    (dict(contactmodel=4), b"contact model"),
    (dict(dt=0.0), b"dt must be positive"),
])
def test_bad_config_rejected_without_gpu(sphk_lib, patch, msg):
    cfg = sphk.make_config(config_from_spherebin(scenes.collision(n=20, seed=1)))
    for k, v in patch.items():
        setattr(cfg, k, v)
    ctx = C.c_void_p()
    rc = sphk_lib.sph_create(C.byref(cfg), C.byref(ctx))
    assert rc == -5
    assert msg in sphk_lib.sph_last_error(ctx)
    assert sphk_lib.sph_destroy(ctx) == 0


def test_null_arguments(sphk_lib):
    assert sphk_lib.sph_create(None, None) == -5
    assert sphk_lib.sph_destroy(None) == 0
