"""Test configuration: the ``gpu`` marker and shared fixtures.

Tests marked ``gpu`` need a CUDA device and the built libsphk; everything
else runs on the CPU (oracle pinning, binary format, the C-ABI surface,
multi-process host logic).
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and the built libsphk")


@pytest.fixture(scope="session")
def oracle_libs():
    import pyoracle
    if not pyoracle.LIB_ORC.exists() or (not pyoracle.LIB_REF.exists() and pyoracle.REF_SRC.exists()):
        pyoracle.build(ref=True)
    libs = {"orc": pyoracle.load("orc")}
    if pyoracle.LIB_REF.exists():
        libs["ref"] = pyoracle.load("ref")
    return libs


@pytest.fixture(scope="session")
def sphk_lib():
    from sphere_b200 import build, sphk
    build.build_lib()
    return sphk.load_library()
