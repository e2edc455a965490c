"""The no-allocation force entry point (nbr_forces_noalloc), called through the
C ABI with caller-owned device buffers, must give what the ordinary entry
point nbr_forces gives.

Some callers cannot let a library allocate device memory (their memory pool
owns every allocation, or they run under a fixed device-memory budget, or a
cudaMalloc's synchronisation is too costly in their loop); this entry point
keeps all of its scratch in a static device array instead.  Two calls in a
row, with different sizes, check that the shared scratch is cleared and
reused correctly.  This file is collected last on purpose.
"""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64, FP32C = 0, 1
# Tolerances of the other parity tests: FP64 per particle; FP32C median and
# worst particle (the two entry points may run different FP32C kernels, e.g.
# the Newton-3 one behind nbr_forces, so they agree to FP32C accuracy).
TOL = {FP64: (1e-12, 1e-12), FP32C: (1e-6, 1e-4)}


def _entry(nbr):
    lib = nbr.load()
    f = lib.nbr_forces_noalloc
    f.argtypes = [C.c_int, C.c_size_t] + [C.c_void_p] * 4 + [C.c_double, C.c_double] + \
                 [C.c_void_p] * 3 + [C.c_void_p]
    f.restype = C.c_int
    return lib, f


def _rel(a, b):
    num = np.linalg.norm(a - b, axis=0)
    den = np.linalg.norm(b, axis=0)
    return num / np.where(den > 0, den, 1.0)


def _call(lib, f, prec, s, eps2, G=1.0):
    """One nbr_forces_noalloc call on device copies of s; returns (rc, a)."""
    import torch
    n = len(s["x"])
    dev = {k: torch.from_numpy(np.ascontiguousarray(s[k])).cuda() for k in ("x", "y", "z", "m")}
    out = torch.full((3, n), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    rc = f(prec, n, dev["x"].data_ptr(), dev["y"].data_ptr(), dev["z"].data_ptr(),
           dev["m"].data_ptr(), G, eps2, out[0].data_ptr(), out[1].data_ptr(),
           out[2].data_ptr(), C.c_void_p(stream))
    return rc, out.cpu().numpy()


def _check_oracle(oracle, s, a, prec, eps2, idx=None):
    if idx is None:
        ref = oracle.accel(s["x"], s["y"], s["z"], s["m"], eps2=eps2, extended=True)
        got = a
    else:
        ref = oracle.accel_subset(s["x"], s["y"], s["z"], s["m"], idx, eps2=eps2)
        got = a[:, idx]
    e = _rel(got, ref)
    med, worst = TOL[prec]
    assert np.median(e) <= med and e.max() <= worst, (len(s["x"]), np.median(e), e.max())


@pytest.mark.parametrize("prec", [FP64, FP32C])
def test_noalloc_matches_nbr_forces_two_calls(nbr, oracle, prec):
    lib, f = _entry(nbr)
    eps2 = 1e-6
    with nbr.Context(0) as ctx:
        for n, seed in ((20000, 31), (12345, 32)):
            s = nbr.plummer(n, seed)
            ctx.upload(s)
            want = ctx.forces(prec, G=1.0, eps2=eps2)
            rc, got = _call(lib, f, prec, s, eps2)
            assert rc == 0, lib.nbr_last_error_string(None)
            assert np.all(np.isfinite(got))
            e = _rel(got, want)
            med, worst = TOL[prec]
            assert np.median(e) <= med and e.max() <= worst, (n, np.median(e), e.max())
            _check_oracle(oracle, s, got, prec, eps2, idx=np.arange(0, n, 37))


@pytest.mark.parametrize("prec", [FP64, FP32C])
def test_noalloc_edge_sizes_against_the_oracle(nbr, oracle, prec):
    """Tiny systems (a single tile, the split clamped to one, mostly padding)
    and the largest accepted one (every split region and the last scratch
    offsets in use), in one sequence so that each call follows a larger or a
    smaller one on the shared scratch."""
    lib, f = _entry(nbr)
    eps2 = 1e-4
    for n in (1, 33, 129, 32768, 2, 1025):
        s = nbr.plummer(n, 40 + n)
        rc, got = _call(lib, f, prec, s, eps2)
        assert rc == 0, lib.nbr_last_error_string(None)
        if n == 1:
            assert np.all(got == 0.0)
            continue
        idx = np.arange(0, n, 61) if n > 4096 else None
        _check_oracle(oracle, s, got, prec, eps2, idx)


def test_noalloc_bounded_wait_expires_cleanly(nbr, oracle):
    """A source tile whose copy is never issued (test hook) makes the bounded
    wait run out: NBR_ERR_TIMEOUT, no fault, and the next call is correct."""
    lib, f = _entry(nbr)
    s = nbr.plummer(20000, 33)
    os.environ["NBR_WAIT_LIMIT_MS"] = "100"
    os.environ["NBR_TEST_SKIP_TILE"] = "1"
    try:
        rc, _ = _call(lib, f, FP64, s, 1e-6)
        assert rc == 4, lib.nbr_last_error_string(None)
    finally:
        del os.environ["NBR_TEST_SKIP_TILE"]
        del os.environ["NBR_WAIT_LIMIT_MS"]
    rc, got = _call(lib, f, FP64, s, 1e-6)
    assert rc == 0, lib.nbr_last_error_string(None)
    _check_oracle(oracle, s, got, FP64, 1e-6, idx=np.arange(0, 20000, 41))


def test_noalloc_rejects_sizes_above_the_limit(nbr):
    lib, f = _entry(nbr)
    n = 32769
    rc = f(FP64, n, 1, 1, 1, 1, 1.0, 0.0, 1, 1, 1, None)  # rejected before any pointer is used
    assert rc == 1
    assert b"no-allocation limit" in lib.nbr_last_error_string(None)
