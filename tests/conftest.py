"""Shared test set-up.

CPU tests (-m "not gpu") check the oracle against the reference's own
outputs and the C-ABI library's exports.  GPU tests (-m gpu) compare the
CUDA path with the oracle.  The oracle is built from its sources on first
use (gcc); the CUDA library is built by koral_b200.build (nvcc, sm_100a).
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU")


def _ensure_oracle():
    from oracle.koral_oracle import ORACLE_LIB
    src = [os.path.join(ROOT, "oracle", f) for f in ("koral_oracle.c", "koral_oracle.h")]
    if not os.path.exists(ORACLE_LIB) or any(os.path.getmtime(s) > os.path.getmtime(ORACLE_LIB) for s in src):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])


@pytest.fixture(scope="session")
def oracle():
    _ensure_oracle()
    import oracle.koral_oracle as ko
    return ko


@pytest.fixture(scope="session")
def kgpu():
    from koral_b200 import build
    build.build()
    import koral_b200
    return koral_b200


def ref_lib_available(name):
    from oracle.koral_oracle import REF_DIR
    return os.path.exists(os.path.join(REF_DIR, name))
