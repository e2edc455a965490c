"""The autotuner: times kernel configurations on the uploaded work and caches
the fastest per (precision, size bucket) in a JSON file ($NBR_TUNE_CACHE, set
to a scratch file by conftest.py); results stay within the usual tolerances
whatever configuration wins."""
import json
import os

import numpy as np
import pytest

from conftest import rel_err
from test_gpu_batch import make_batch, system

pytestmark = pytest.mark.gpu
FP64, FP32C = 0, 1


def _cache():
    with open(os.environ["NBR_TUNE_CACHE"]) as f:
        return json.load(f)


def test_single_system_autotune(ctx, nbr, oracle):
    n, eps2 = 16384, 1e-6
    s = nbr.plummer(n, 8)
    ctx.upload(s)
    ctx.autotune(FP32C, eps2)
    cache = _cache()
    key = "fp32c:i14:j7"  # 2^14 receivers, 2^7 source tiles
    assert key in cache
    ni, warps, split = cache[key]
    # 4, 8: the large kernels; 1: small-N warp splitting; 3: Newton-3 (8 warps)
    assert ni in (1, 3, 4, 8) and warps in (2, 4, 8) and split >= 1
    a = ctx.forces(FP32C, eps2=eps2)
    idx = np.arange(0, n, 97)
    ref = oracle.accel_subset(s["x"], s["y"], s["z"], s["m"], idx, eps2=eps2)
    assert np.median(rel_err(a[:, idx], ref)) <= 1e-6


@pytest.mark.parametrize("prec", [FP64, FP32C])
def test_batch_autotune(ctx, nbr, oracle, prec):
    sizes = [40, 130, 300, 513, 1000, 2000, 3000]
    off, st = make_batch(nbr, sizes, seed=12)
    ctx.batch_upload(off, st)
    eps2 = 1e-6
    ctx.batch_autotune(prec, eps2)
    name = "fp32c" if prec == FP32C else "fp64"
    key = f"batch:{name}:s2:n11"  # 7 systems (2^2 <= 7 < 2^3), largest 3000 (2^11)
    cache = _cache()
    assert key in cache
    ni, warps, per_sm = cache[key]
    assert ni in (4, 8) and per_sm >= 1
    a = ctx.batch_forces(prec, eps2=eps2)
    for s in range(len(sizes)):
        sub = system(st, off, s)
        ref = oracle.accel(sub["x"], sub["y"], sub["z"], sub["m"], eps2=eps2, extended=True)
        e = rel_err(a[:, off[s]:off[s + 1]], ref)
        assert (e.max() <= 1e-12) if prec == FP64 else (np.median(e) <= 1e-6)
    # a new upload of a batch in the same bucket picks the cached configuration
    ctx.batch_upload(off, st)
    b = ctx.batch_forces(prec, eps2=eps2)
    np.testing.assert_array_equal(a, b)
