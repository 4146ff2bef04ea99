import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "cuda-stereo-matching_b200")
ORACLE = os.path.join(REPO, "oracle")
for p in (PKG, ORACLE, REPO):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def _ensure_built():
    import build as pkg_build  # cuda-stereo-matching_b200/build.py
    import build_oracle

    if not os.path.exists(pkg_build.OUT):
        pkg_build.build()
    build_oracle.build_oracle()
    build_oracle.build_ref()


_ensure_built()

EMU_SRC = os.path.join(REPO, "tests", "native", "delaunay_emu.cpp")
EMU_LIB = os.path.join(REPO, "tests", "native", "libdelemu.so")


@pytest.fixture(scope="session")
def emu_lib():
    import ctypes

    if not os.path.exists(EMU_LIB) or os.path.getmtime(EMU_LIB) < max(
            os.path.getmtime(EMU_SRC), os.path.getmtime(os.path.join(PKG, "csrc", "delaunay_core.h"))):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", EMU_SRC, "-o", EMU_LIB], check=True)
    return ctypes.CDLL(EMU_LIB)


def gpu_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
