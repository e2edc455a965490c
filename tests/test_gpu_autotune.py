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
    ni, warps, split, tile, unroll = cache[key]
    # 4, 8: the large kernels; 1: small-N warp splitting; 3: Newton-3 (8 or
    # 16 warps); tile / unroll: the large kernel's j-tile and unroll depth,
    # swept when its default configuration wins (0: the defaults)
    assert ni in (1, 3, 4, 8) and warps in (2, 4, 8, 16) and split >= 1
    if (ni, warps) == (8, 2):
        assert tile in (64, 128, 256) and unroll in (2, 4, 8)
    else:
        assert tile == 0 and unroll == 0
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
    ni, warps, per_sm = cache[key][:3]
    assert ni in (3, 4, 8) and per_sm >= 1
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


@pytest.mark.parametrize("prec", [FP64, FP32C])
def test_large_kernel_tilings_agree(ctx, nbr, oracle, prec):
    """Every built (j-tile, unroll) of the large kernel's default
    configuration gives the usual accuracy.  A larger system uploaded first
    leaves stale FP32C records past the smaller system's last tile (33 tiles:
    a 256-source stage spans one past the end), which the kernel must skip."""
    ni, warps = (8, 2) if prec == FP32C else (4, 4)
    ctx.upload(nbr.plummer(8192, 1))
    ctx.forces(prec, eps2=1e-6)
    s = nbr.plummer(4097, 2)
    ctx.upload(s)
    ref = oracle.accel(s["x"], s["y"], s["z"], s["m"], eps2=1e-6, extended=True)
    ctx.set_force_config(prec, ni, warps, 0)
    try:
        for tile in (64, 128, 256):
            for unroll in (2, 4, 8):
                ctx.set_force_tiling(prec, tile, unroll)
                assert ctx.get_force_tiling(prec, 1e-6) == (tile, unroll)
                for split in (1, 5):
                    ctx.set_force_config(prec, ni, warps, split)
                    ctx.set_force_tiling(prec, tile, unroll)
                    e = rel_err(ctx.forces(prec, eps2=1e-6), ref)
                    if prec == FP64:
                        assert e.max() <= 1e-12, (tile, unroll, split, e.max())
                    else:
                        assert np.median(e) <= 1e-6 and e.max() <= 1e-4, (tile, unroll, split)
        with pytest.raises(nbr.NbrError):
            ctx.set_force_tiling(prec, 96, 4)
    finally:
        ctx.set_force_config(prec, 0)
