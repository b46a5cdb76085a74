"""Shared fixtures.  `-m gpu` tests call the CUDA library through its C ABI; the rest run on CPU."""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "ecmc-qcb_b200")
ORACLE_DIR = os.path.join(ROOT, "oracle")


def load_package():
    """Imports ecmc-qcb_b200/ (a directory name that is not a Python identifier) as `ecmc_qcb_b200`."""
    if "ecmc_qcb_b200" in sys.modules:
        return sys.modules["ecmc_qcb_b200"]
    spec = importlib.util.spec_from_file_location("ecmc_qcb_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ecmc_qcb_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    if ORACLE_DIR not in sys.path:
        sys.path.insert(0, ORACLE_DIR)
    import oracle  # noqa: E402

    oracle.build()
    return oracle


def load_reference():
    """The reference's own hot-path code (oracle/_ref/libqcb_ref.so), or None when it is not built."""
    if ORACLE_DIR not in sys.path:
        sys.path.insert(0, ORACLE_DIR)
    import ref  # noqa: E402

    return ref if (ref.available() or ref.build()) else None


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); calls libqcb.so")
    config.addinivalue_line("markers", "slow: long CPU test")


@pytest.fixture(scope="session")
def qcb():
    return load_package()


@pytest.fixture(scope="session")
def orc():
    return load_oracle()


@pytest.fixture(scope="session")
def refc():
    r = load_reference()
    if r is None:
        pytest.skip("oracle/_ref/libqcb_ref.so is not built (make -C oracle ref needs the reference tree)")
    return r


@pytest.fixture(scope="session")
def gpu(qcb):
    import ctypes

    try:
        rt = ctypes.CDLL("libcudart.so.12")
        n = ctypes.c_int(0)
        if rt.cudaGetDeviceCount(ctypes.byref(n)) != 0 or n.value == 0:
            raise RuntimeError("no device")
    except OSError:
        pass
    qcb.load_library()
    return qcb


def rel_err(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
