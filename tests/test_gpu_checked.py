"""The bounds-checked build (libnbr_checked.so): every kernel index is tested
against its array's allocated length before the access.  A battery of calls
at edge sizes must run without a single out-of-range index and give the same
results as the normal build; and the checker must trip when the host
under-reports a length (a test hook; the real access stays in bounds)."""
import json
import os
import subprocess
import sys

import pytest

from conftest import PKG, ROOT

pytestmark = pytest.mark.gpu
CHECKED = os.path.join(PKG, "libnbr_checked.so")
SCRIPT = os.path.join(ROOT, "tests", "checked", "run_checked.py")


def _run(lib, extra_env=None):
    env = dict(os.environ)
    if lib:
        env["NBR_LIB_PATH"] = lib
    env.update(extra_env or {})
    p = subprocess.run([sys.executable, SCRIPT], capture_output=True, text=True, env=env, timeout=900)
    return p


@pytest.fixture(scope="module")
def checked_lib():
    if not os.path.exists(CHECKED):
        subprocess.run(["make", "-C", PKG, "checked"], check=True, capture_output=True)
    return CHECKED


def test_checked_build_finds_no_out_of_range_index(checked_lib):
    p = _run(checked_lib)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-4000:]
    got = json.loads(p.stdout.strip().splitlines()[-1])
    assert got["calls"] > 150
    q = _run(None)  # the normal build on the same calls
    assert q.returncode == 0, q.stderr[-4000:]
    want = json.loads(q.stdout.strip().splitlines()[-1])
    assert got["calls"] == want["calls"]
    for k, v in want["results"].items():
        assert abs(got["results"][k] - v) <= 1e-12 * max(1.0, abs(v)), k


def test_checked_build_reports_an_under_reported_length(checked_lib, nbr):
    code = ("import sys, os; sys.path.insert(0, %r); import nbr\n"
            "c = nbr.Context(0); c.upload(nbr.plummer(1000, 1))\n"
            "try:\n    c.forces(nbr.FP64, eps2=1e-6)\nexcept nbr.NbrError as e:\n"
            "    print('status', e.status); sys.exit(0)\n"
            "print('no error'); sys.exit(1)\n") % PKG
    env = dict(os.environ, NBR_LIB_PATH=checked_lib, NBR_TEST_SHRINK_BOUNDS="1")
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=300)
    assert p.returncode == 0 and "status 9" in p.stdout, p.stdout + p.stderr
