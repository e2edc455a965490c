"""The persistent small-system run (nbr_persist.cu): every step of nbr_run for
an FP64 system of at most 4096 particles in one cooperative launch, with one
bounded grid barrier per force evaluation.

It must reproduce the launch-per-evaluation path (forced with the small-N
kernel) to FP64 summation order, and the oracle's trajectories, for every
scheme; keep first-same-as-last across calls; and report a barrier that never
completes as NBR_ERR_TIMEOUT without faulting (a test hook keeps one CTA from
arriving, the wait limit is short).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64 = 0
KDK, DKD, EULER = 0, 1, 2
PERSIST = 2  # ForceConfig ni of the persistent run; warps = lane groups


def _run(ctx, s, cfg, scheme, order, dt, steps, eps2, calls=1):
    ctx.set_force_config(FP64, *cfg)
    try:
        ctx.upload(s)
        st = None
        for _ in range(calls):
            st = ctx.run(FP64, scheme, order, dt, steps, eps2=eps2)
        return ctx.download(), st
    finally:
        ctx.set_force_config(FP64, 0)


def _maxdiff(a, b):
    return max(np.abs(a[k] - b[k]).max() / max(1.0, np.abs(b[k]).max()) for k in
               ("x", "y", "z", "vx", "vy", "vz"))


@pytest.mark.parametrize("n", [2, 3, 127, 1000, 2048, 4096])
@pytest.mark.parametrize("groups", [4, 8, 16])
@pytest.mark.parametrize("warps", [8, 16])
def test_persistent_matches_launch_per_step(ctx, nbr, n, groups, warps):
    s = nbr.plummer(n, 60 + n)
    for scheme, order, eps2 in ((KDK, 2, 1e-6), (DKD, 4, 1e-6), (EULER, 2, 1e-6), (KDK, 2, 0.0)):
        got, st = _run(ctx, s, (PERSIST, groups, warps), scheme, order, 1e-3, 7, eps2, calls=2)
        assert st["kernels"] == 1, st
        want, _ = _run(ctx, s, (1, 8, 0), scheme, order, 1e-3, 7, eps2, calls=2)
        assert _maxdiff(got, want) <= 1e-12, (scheme, order, eps2, _maxdiff(got, want))


@pytest.mark.parametrize("n", [3, 1000, 2048, 4096])
@pytest.mark.parametrize("groups", [8, 16])
def test_persistent_eight_receivers_per_lane(ctx, nbr, n, groups):
    """The layout with 8 receivers per lane (nbr_set_force_tiling tile = 8)."""
    s = nbr.plummer(n, 90 + n)
    for scheme, eps2 in ((KDK, 1e-6), (EULER, 0.0)):
        ctx.set_force_config(FP64, PERSIST, groups, 16)
        ctx.set_force_tiling(FP64, 8, 0)
        try:
            ctx.upload(s)
            st = ctx.run(FP64, scheme, 2, 1e-3, 7, eps2=eps2)
            got = ctx.download()
        finally:
            ctx.set_force_config(FP64, 0)
        assert st["kernels"] == 1
        want, _ = _run(ctx, s, (1, 8, 0), scheme, 2, 1e-3, 7, eps2)
        assert _maxdiff(got, want) <= 1e-12, (scheme, eps2, _maxdiff(got, want))


def test_persistent_is_the_default_for_small_fp64_systems(ctx, nbr, oracle):
    """Plummer N = 2048, eps = 1e-3, KDK dt = 1e-3, 100 steps (the small-system
    workload) through the default path: one launch, the oracle's trajectory."""
    s = nbr.plummer(2048, 0)
    ctx.upload(s)
    st = ctx.run(FP64, KDK, 2, 1e-3, 100, eps2=1e-6)
    assert st["kernels"] == 1 and st["force_evals"] == 101
    got = ctx.download()
    want = oracle.kdk(s, 1e-3, 100, eps2=1e-6)
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.abs(got[k] - want[k]).max() <= 1e-10, k


def test_persistent_keeps_first_same_as_last(ctx, nbr, oracle):
    """Two KDK calls of 5 steps equal one call of 10: the second call reuses
    the accelerations the first one left (5 evaluations, not 6)."""
    s = nbr.plummer(1500, 3)
    ctx.upload(s)
    ctx.run(FP64, KDK, 2, 1e-3, 5, eps2=1e-6)
    st = ctx.run(FP64, KDK, 2, 1e-3, 5, eps2=1e-6)
    assert st["force_evals"] == 5
    got = ctx.download()
    want = oracle.kdk(s, 1e-3, 10, eps2=1e-6)
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.abs(got[k] - want[k]).max() <= 1e-11, k


def test_persistent_grid_barrier_expires_cleanly(nbr, oracle):
    s = nbr.plummer(2048, 9)
    with nbr.Context(0) as c:
        c.upload(s)
        os.environ["NBR_WAIT_LIMIT_MS"] = "100"
        os.environ["NBR_TEST_SKIP_TILE"] = "0"
        try:
            with pytest.raises(nbr.NbrError) as ei:
                c.run(FP64, KDK, 2, 1e-3, 4, eps2=1e-6)
            assert ei.value.status == 4
        finally:
            del os.environ["NBR_TEST_SKIP_TILE"]
            del os.environ["NBR_WAIT_LIMIT_MS"]
        c.upload(s)
        c.run(FP64, KDK, 2, 1e-3, 4, eps2=1e-6)
        got = c.download()
    want = oracle.kdk(s, 1e-3, 4, eps2=1e-6)
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.abs(got[k] - want[k]).max() <= 1e-11, k


FP32C = 1


@pytest.mark.parametrize("n", [2, 127, 1000, 2048, 4096])
@pytest.mark.parametrize("groups", [4, 8, 16])
def test_persistent_fp32c(ctx, nbr, oracle, n, groups):
    """The FP32C form of the persistent run (forced with ni = 2): the oracle's
    KDK and Euler trajectories within the FP32C tolerance of the other
    FP32C trajectory tests, one launch per run, and the FP32C accelerations
    it leaves against the FP64 ones."""
    s = nbr.plummer(n, 70 + n)
    for scheme, eps2 in ((KDK, 1e-6), (EULER, 1e-6), (KDK, 0.0)):
        ctx.set_force_config(FP32C, PERSIST, groups, 0)
        try:
            ctx.upload(s)
            st = ctx.run(FP32C, scheme, 2, 1e-3, 5, eps2=eps2)
            got = ctx.download()
        finally:
            ctx.set_force_config(FP32C, 0)
        assert st["kernels"] == 1 and st["force_evals"] == (6 if scheme == KDK else 5)
        want = oracle.kdk(s, 1e-3, 5, eps2=eps2) if scheme == KDK else oracle.euler(s, 1e-3, 5, eps2=eps2)
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.abs(got[k] - want[k]).max() <= 1e-6, (scheme, eps2, k)


def test_persistent_fp32c_far_from_the_origin(ctx, nbr, oracle):
    """Its records are relative to the system's FP64 mean position, so a
    system shifted far from the coordinate origin keeps FP32 resolution."""
    s = nbr.plummer(2048, 5)
    for k, d in (("x", 1.0e3), ("y", -2.0e3), ("z", 5.0e2)):
        s[k] = s[k] + d
    ctx.set_force_config(FP32C, PERSIST, 8, 0)
    try:
        ctx.upload(s)
        ctx.run(FP32C, KDK, 2, 1e-3, 5, eps2=1e-6)
        got = ctx.download()
    finally:
        ctx.set_force_config(FP32C, 0)
    want = oracle.kdk(s, 1e-3, 5, eps2=1e-6)
    for k in ("vx", "vy", "vz"):
        assert np.abs(got[k] - want[k]).max() <= 1e-6, k
    for k in ("x", "y", "z"):
        assert np.abs(got[k] - want[k]).max() <= 1e-6 * (1.0 + np.abs(want[k]).max()), k
