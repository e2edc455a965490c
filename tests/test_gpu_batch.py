"""Batched independent systems (nbr_batch_*) against the oracle, system by system.

Tolerances as for single systems: FP64 <= 1e-12 per particle, FP32C median
<= 1e-6; trajectories (KDK, 20 steps) within 1e-10 of the oracle's.
"""
import os

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

FP64, FP32C = 0, 1
KEYS6 = ("x", "y", "z", "vx", "vy", "vz")
# every receiver-tile shape: tiny systems, exact tiles, ragged last tiles
SIZES = [1, 2, 3, 16, 17, 31, 33, 64, 65, 100, 127, 128, 129, 200, 255, 256, 257, 700, 1500]


def make_batch(nbr, sizes, seed=5):
    off = np.zeros(len(sizes) + 1, dtype=np.int64)
    off[1:] = np.cumsum(sizes)
    st = {k: np.zeros(int(off[-1])) for k in nbr.KEYS}
    for s, n in enumerate(sizes):
        sub = nbr.plummer(int(n), nbr.system_seed(seed, s))
        for k in nbr.KEYS:
            st[k][off[s]:off[s + 1]] = sub[k]
    return off, st


def system(st, off, s):
    return {k: st[k][off[s]:off[s + 1]] for k in st}


# work lists: one-tile items, two-tile items, Newton-3 row blocks
WORK = [(FP64, 0), (FP64, 1), (FP64, 2), (FP32C, 0), (FP32C, 1), (FP32C, 2)]
WORK_IDS = ["fp64-one-tile", "fp64-two-tile", "fp64-newton3", "fp32c-one-tile", "fp32c-two-tile",
            "fp32c-newton3"]


@pytest.mark.parametrize("prec,wide", WORK, ids=WORK_IDS)
def test_batch_forces_match_oracle(ctx, nbr, oracle, prec, wide):
    off, st = make_batch(nbr, SIZES)
    ctx.batch_upload(off, st)
    ctx.batch_set_config(prec, wide, 0)
    eps2 = 1e-6
    a = ctx.batch_forces(prec, eps2=eps2)
    errs = []
    for s, n in enumerate(SIZES):
        sub = system(st, off, s)
        ref = oracle.accel(sub["x"], sub["y"], sub["z"], sub["m"], eps2=eps2, extended=True)
        got = a[:, off[s]:off[s + 1]]
        if n == 1:
            assert np.all(got == 0.0)
            continue
        e = rel_err(got, ref)
        errs.append(e)
        if prec == FP64:
            assert e.max() <= 1e-12, (n, e.max())
    if prec == FP32C:
        allerr = np.concatenate(errs)
        assert np.median(allerr) <= 1e-6 and allerr.max() <= 1e-4


@pytest.mark.parametrize("eps2", [1e-6, 0.0])
def test_batch_newton3_row_blocks(ctx, nbr, oracle, eps2):
    """The Newton-3 work list on systems of 3 to 17 tiles (odd and even tile
    counts, ragged last tiles) beside small systems that keep two-tile items:
    every particle against the oracle, the run repeated bit for bit (the
    reactions are summed in a fixed order), and equal to the two-tile list
    to FP32C accuracy."""
    sizes = [5, 129, 257, 300, 384, 385, 640, 1000, 2049, 2100]
    off, st = make_batch(nbr, sizes, seed=21)
    ctx.batch_upload(off, st)
    ctx.batch_set_config(FP32C, 2, 0)
    a = ctx.batch_forces(FP32C, eps2=eps2)
    b = ctx.batch_forces(FP32C, eps2=eps2)
    np.testing.assert_array_equal(a, b)
    errs = []
    for s, n in enumerate(sizes):
        sub = system(st, off, s)
        ref = oracle.accel(sub["x"], sub["y"], sub["z"], sub["m"], eps2=eps2, extended=True)
        e = rel_err(a[:, off[s]:off[s + 1]], ref)
        assert np.median(e) <= 1e-6, (n, np.median(e))
        errs.append(e)
    assert np.concatenate(errs).max() <= 1e-4
    ctx.batch_set_config(FP32C, 1, 0)
    w = ctx.batch_forces(FP32C, eps2=eps2)
    assert rel_err(a, w).max() <= 1e-4


@pytest.mark.parametrize("eps2", [1e-6, 0.0])
def test_batch_newton3_row_blocks_fp64(ctx, nbr, oracle, eps2):
    """The FP64 Newton-3 work list (one-tile row blocks for systems of two
    tiles or more, one-tile items for the rest): every particle within 1e-12
    of the oracle, the run repeated bit for bit, and within 1e-13 of the
    one-tile list (only the summation order differs)."""
    sizes = [5, 128, 129, 200, 256, 300, 385, 640, 1000, 2049]
    off, st = make_batch(nbr, sizes, seed=23)
    ctx.batch_upload(off, st)
    ctx.batch_set_config(FP64, 2, 0)
    a = ctx.batch_forces(FP64, eps2=eps2)
    b = ctx.batch_forces(FP64, eps2=eps2)
    np.testing.assert_array_equal(a, b)
    for s, n in enumerate(sizes):
        sub = system(st, off, s)
        ref = oracle.accel(sub["x"], sub["y"], sub["z"], sub["m"], eps2=eps2, extended=True)
        e = rel_err(a[:, off[s]:off[s + 1]], ref)
        assert e.max() <= 1e-12, (n, e.max())
    ctx.batch_set_config(FP64, 0, 0)
    w = ctx.batch_forces(FP64, eps2=eps2)
    assert rel_err(a, w).max() <= 1e-13


def test_batch_set_config_rejects_bad_values(ctx, nbr):
    off, st = make_batch(nbr, [300, 400])
    ctx.batch_upload(off, st)
    for wide, per in ((3, 0), (-2, 0), (1, -1)):
        with pytest.raises(nbr.NbrError):
            ctx.batch_set_config(FP64, wide, per)


def test_batch_systems_do_not_interact(ctx, nbr):
    """Two copies of one system at the same place: each feels only itself."""
    s1 = nbr.plummer(300, 1)
    off = np.array([0, 300, 600])
    st = {k: np.concatenate([s1[k], s1[k]]) for k in nbr.KEYS}
    ctx.batch_upload(off, st)
    a = ctx.batch_forces(FP64, eps2=1e-6)
    np.testing.assert_array_equal(a[:, :300], a[:, 300:])
    ctx.upload(s1)
    single = ctx.forces(FP64, eps2=1e-6)
    assert rel_err(a[:, :300], single).max() <= 1e-13


@pytest.mark.parametrize("prec,wide", WORK, ids=WORK_IDS)
def test_batch_kdk_matches_oracle(ctx, nbr, oracle, prec, wide):
    sizes = [64, 130, 513, 1000]
    off, st = make_batch(nbr, sizes, seed=9)
    ctx.batch_upload(off, st)
    ctx.batch_set_config(prec, wide, 1 if wide else 0)
    eps2 = 1e-6
    stats = ctx.batch_run(prec, dt=1e-3, steps=20, eps2=eps2)
    assert stats["force_evals"] == 21
    assert stats["pairs"] == 21 * sum(n * (n - 1) for n in sizes)
    got = ctx.batch_download()
    for s in range(len(sizes)):
        want = oracle.kdk(system(st, off, s), 1e-3, 20, eps2=eps2)
        for k in KEYS6:
            d = np.abs(got[k][off[s]:off[s + 1]] - want[k]).max()
            assert d <= (1e-10 if prec == FP64 else 1e-6), (s, k, d)


def test_batch_first_same_as_last(ctx, nbr):
    off, st = make_batch(nbr, [100, 300], seed=4)
    ctx.batch_upload(off, st)
    ctx.batch_run(FP64, dt=1e-3, steps=10, eps2=1e-6)
    one = ctx.batch_download()
    ctx.batch_upload(off, st)
    a = ctx.batch_run(FP64, dt=1e-3, steps=5, eps2=1e-6)
    b = ctx.batch_run(FP64, dt=1e-3, steps=5, eps2=1e-6)
    assert a["force_evals"] == 6 and b["force_evals"] == 5
    two = ctx.batch_download()
    for k in KEYS6:
        assert np.abs(two[k] - one[k]).max() <= 1e-13


def test_batch_diagnostics(ctx, nbr, oracle):
    sizes = [1, 50, 400, 1200]
    off, st = make_batch(nbr, sizes, seed=12)
    ctx.batch_upload(off, st)
    d = ctx.batch_diagnostics(eps2=1e-6)
    for s in range(len(sizes)):
        e = oracle.energy(system(st, off, s), eps2=1e-6)
        assert abs(d[s]["T"] - e["T"]) <= 1e-12 * max(abs(e["T"]), 1e-300)
        assert abs(d[s]["U"] - e["U"]) <= 1e-12 * max(abs(e["U"]), 1e-300) + 1e-300
        np.testing.assert_allclose(d[s]["P"], e["P"], atol=1e-14)
        assert abs(d[s]["M"] - e["M"]) <= 1e-14


@pytest.mark.parametrize("wide", [1, 2], ids=["two-tile", "newton3"])
def test_batch_full_workload(ctx, nbr, oracle, wide):
    """The 4096-system log-uniform workload: two FP32C steps; sampled systems
    checked against the oracle; pair count as the workload defines it."""
    off, st = nbr.batch_plummer(4096, 3)
    ctx.batch_upload(off, st)
    ctx.batch_set_config(FP32C, wide, 0)
    eps2 = 1e-6
    a = ctx.batch_forces(FP32C, eps2=eps2)
    rng = np.random.default_rng(1)
    for s in rng.choice(4096, 6, replace=False):
        sub = system(st, off, s)
        ref = oracle.accel(sub["x"], sub["y"], sub["z"], sub["m"], eps2=eps2, extended=True)
        assert np.median(rel_err(a[:, off[s]:off[s + 1]], ref)) <= 1e-6
    sizes = np.diff(off)
    stats = ctx.batch_run(FP32C, dt=1e-3, steps=2, eps2=eps2)
    assert stats["pairs"] == 2 * float((sizes * (sizes - 1)).sum())


@pytest.mark.parametrize("prec,wide", [(FP32C, 1), (FP32C, 2), (FP64, 2)],
                         ids=["fp32c-two-tile", "fp32c-newton3", "fp64-newton3"])
def test_batch_bounded_wait_expires_cleanly(nbr, prec, wide):
    """Tile 2 of every item never arrives (a test hook; for a Newton-3 row
    block, a later column tile): the wait gives up, the call reports
    NBR_ERR_TIMEOUT and the context keeps working."""
    off, st = make_batch(nbr, [700, 900], seed=2)
    with nbr.Context(0) as c:
        c.batch_upload(off, st)
        c.batch_set_config(prec, wide, 0)
        os.environ["NBR_WAIT_LIMIT_MS"] = "100"
        os.environ["NBR_TEST_SKIP_TILE"] = "2"
        try:
            with pytest.raises(nbr.NbrError) as ei:
                c.batch_forces(prec, eps2=1e-6)
            assert ei.value.status == 4
        finally:
            del os.environ["NBR_TEST_SKIP_TILE"]
            del os.environ["NBR_WAIT_LIMIT_MS"]
        a = c.batch_forces(FP64, eps2=1e-6)
        assert np.all(np.isfinite(a))


def test_batch_rejects_bad_input(ctx, nbr):
    off, st = make_batch(nbr, [10, 20])
    with pytest.raises(nbr.NbrError):
        ctx.batch_upload(np.array([0, 10, 10, 30]), st)  # empty system
    bad = {k: v.copy() for k, v in st.items()}
    bad["m"][3] = np.inf
    with pytest.raises(nbr.NbrError) as ei:
        ctx.batch_upload(off, bad)
    assert ei.value.status == 7
