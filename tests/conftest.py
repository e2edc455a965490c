"""Shared test setup.

* ``gpu`` marks tests that need an sm_100 GPU; they call the product only
  through the C ABI (libnbr.so via n-body-ring-solver_b200/nbr.py).
* The CPU checkers live in oracle/ (test infrastructure): the plain-C
  restatement (liboracle.so) and, where it was built, the reference's own CPU
  solver compiled from its sources (oracle/_ref).
"""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "n-body-ring-solver_b200")
ORACLE_DIR = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
# The reference checkout, where present (this container only; GPU tests never
# read it): $NBR_REFERENCE_DIR, else the directory "reference" beside the repo.
REFERENCE_CPU = os.path.join(os.path.abspath(os.environ.get("NBR_REFERENCE_DIR")
                                             or os.path.join(ROOT, os.pardir, "reference")), "CPU")
for p in (PKG, ORACLE_DIR):
    if p not in sys.path:
        sys.path.insert(0, p)
# Autotune results of a test run go to a scratch file, not next to libnbr.so.
os.environ.setdefault("NBR_TUNE_CACHE",
                      os.path.join(tempfile.mkdtemp(prefix="nbr_tune_"), "nbr_tune_cache.json"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU; calls the CUDA path")


def _ensure_built():
    if not os.path.exists(os.path.join(ORACLE_DIR, "liboracle.so")):
        subprocess.run(["make", "-C", ORACLE_DIR, "oracle"], check=True, capture_output=True)
    if not os.path.exists(os.path.join(PKG, "libnbr.so")):
        subprocess.run(["make", "-C", PKG, "libnbr.so"], check=True, capture_output=True)


@pytest.fixture(scope="session")
def oracle():
    _ensure_built()
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle import Reference, reference_available
    if not reference_available():
        pytest.skip("reference CPU solver not built here (needs the reference sources)")
    return Reference()


@pytest.fixture(scope="session")
def nbr():
    _ensure_built()
    import nbr as mod
    mod.load()
    return mod


@pytest.fixture(scope="session")
def ctx(nbr):
    c = nbr.Context(0)
    yield c
    c.close()


def golden(name):
    path = os.path.join(GOLDEN, name)
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def rel_err(a, b):
    """Per-particle |a - b| / |b| for (3, n) arrays."""
    num = np.linalg.norm(np.asarray(a) - np.asarray(b), axis=0)
    den = np.linalg.norm(np.asarray(b), axis=0)
    return num / np.where(den > 0, den, 1.0)


def state_copy(s):
    return {k: np.array(v, dtype=np.float64, copy=True) for k, v in s.items()}
