"""Shared test setup: import paths, the gpu marker and checker fixtures.

CPU tests (-m "not gpu") check the oracle against the golden fixtures made by
the reference, the host build of the library's portable code against the
oracle, and the C ABI surface. GPU tests (-m gpu) run the CUDA library through
its C ABI and compare with the oracle and the fixtures.
"""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PACKAGE = ROOT / 'custom-ray-tracing-shader_b200'
ORACLE = ROOT / 'oracle'
GOLDEN = Path(__file__).resolve().parent / 'golden'
for p in (PACKAGE, ORACLE, GOLDEN):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA GPU (B200); runs the CUDA library through its C ABI')


def _make(target_dir, *targets):
    subprocess.run(['make', '-C', str(target_dir), *targets], check=True, stdout=subprocess.DEVNULL)


@pytest.fixture(scope='session')
def oracle():
    from oracle_api import Oracle, ORACLE_LIB
    if not ORACLE_LIB.exists():
        _make(ORACLE, 'oracle')
    return Oracle()


@pytest.fixture(scope='session')
def reference():
    from oracle_api import Reference, REFERENCE_LIB
    if not REFERENCE_LIB.exists():
        pytest.skip('reference harness not built (reference sources absent on this machine)')
    return Reference()


@pytest.fixture(scope='session')
def lib():
    """The CUDA library. Missing library is an error, not a skip."""
    from native_api import load_library, LIBRARY
    if not LIBRARY.exists():
        _make(PACKAGE)
    return load_library()


@pytest.fixture
def session(lib):
    from native_api import Session
    s = Session(lib)
    yield s
    s.close()


def golden(name):
    return np.load(GOLDEN / name, allow_pickle=False)


def sha256(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
