"""nbr_step_range / nbr_state_pointers / nbr_state_changed on one GPU.

The i-partition is emulated with several contexts on the same GPU, one per
rank, exchanging owned slices by device copies between steps (each launch
finishes before the next begins: no kernel waits on another).  With the same
kernel configuration forced everywhere, the per-receiver summation order is
the same as in one whole-system run, so the emulated ranks must reproduce
nbr_run bit for bit.  The process-group exchange itself is covered on CPU by
test_shard.py.
"""
import numpy as np
import pytest
import torch

import nbr_shard

pytestmark = pytest.mark.gpu

CFG = {0: (4, 4, 4), 1: (8, 2, 4)}  # precision -> (ni, warps, split) on every context


def _contexts(nbr, k, s, precision):
    out = []
    for _ in range(k):
        c = nbr.Context(0)
        c.set_force_config(precision, *CFG[precision])
        c.upload(s)
        out.append(c)
    return out


def _exchange(ctxs, n):
    """Every context receives every other context's owned position slice."""
    world = len(ctxs)
    for c in ctxs:
        c.synchronize()
    st = [c.state_tensors() for c in ctxs]
    for r in range(world):
        i0, _, owned = nbr_shard.shard_bounds(n, world, r)
        for q in range(world):
            if q != r and owned:
                for k in ("x", "y", "z"):
                    st[q][k][i0:i0 + owned].copy_(st[r][k][i0:i0 + owned])
    torch.cuda.synchronize()
    for c in ctxs:
        c.state_changed()


def _gather_velocities(ctxs, n):
    world = len(ctxs)
    st = [c.state_tensors() for c in ctxs]
    for r in range(world):
        i0, _, owned = nbr_shard.shard_bounds(n, world, r)
        for k in ("vx", "vy", "vz"):
            st[0][k][i0:i0 + owned].copy_(st[r][k][i0:i0 + owned])
    torch.cuda.synchronize()
    ctxs[0].state_changed()


def _emulated_run(nbr, s, precision, scheme, dt, steps, world, eps2):
    n = len(s["x"])
    ctxs = _contexts(nbr, world, s, precision)
    if scheme == nbr.KDK:
        sched = [(0.5 * dt, dt)] + [(dt, dt)] * (steps - 1) + [(0.5 * dt, 0.0)]
    else:
        sched = [(dt, dt)] * steps
    for kick, drift in sched:
        for r, c in enumerate(ctxs):
            i0, _, owned = nbr_shard.shard_bounds(n, world, r)
            if owned:
                c.step_range(precision, scheme, i0, owned, kick, drift, 1.0, eps2)
        _exchange(ctxs, n)
    _gather_velocities(ctxs, n)
    out = ctxs[0].download()
    for c in ctxs:
        c.synchronize()
        c.close()
    return out


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32c"])
@pytest.mark.parametrize("scheme", [0, 2], ids=["kdk", "euler"])
@pytest.mark.parametrize("n,world", [(8192, 2), (5000, 3)])
def test_emulated_ranks_match_whole_run(nbr, oracle, precision, scheme, n, world):
    """Bit for bit against one whole-system run, and directly against the
    oracle's trajectory (KDK or Euler in FP64, every ordered pair in index
    order): FP64 within 1e-11, FP32C within 1e-6 (absolute, positions and
    velocities of order 1)."""
    s = nbr.plummer(n, 5)
    eps2, dt, steps = 1e-6, 1e-3, 3
    whole = nbr.Context(0)
    whole.set_force_config(precision, *CFG[precision])
    whole.upload(s)
    whole.run(precision, scheme, 2, dt, steps, eps2=eps2)
    ref = whole.download()
    whole.close()
    got = _emulated_run(nbr, s, precision, scheme, dt, steps, world, eps2)
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    want = (oracle.kdk(s, dt, steps, eps2=eps2) if scheme == nbr.KDK
            else oracle.euler(s, dt, steps, eps2=eps2))
    tol = 1e-11 if precision == nbr.FP64 else 1e-6
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.abs(got[k] - want[k]).max() <= tol, k


def test_step_range_matches_oracle_forces(nbr, oracle):
    """The owned slice's accelerations (FP64) against the oracle's, through
    a step with kick 1 and drift 0 from zero velocities: v = a."""
    n = 3000
    s = nbr.plummer(n, 6)
    s["vx"][:] = 0.0; s["vy"][:] = 0.0; s["vz"][:] = 0.0
    c = nbr.Context(0)
    c.upload(s)
    c.step_range(nbr.FP64, nbr.KDK, 1024, 1500, 1.0, 0.0, 1.0, 1e-4)
    c.synchronize()
    st = c.state_tensors()
    v = np.stack([st[k][:n].cpu().numpy() for k in ("vx", "vy", "vz")])
    c.close()
    a = oracle.accel(s["x"], s["y"], s["z"], s["m"], 1.0, 1e-4)
    sl = slice(1024, 2524)
    np.testing.assert_allclose(v[:, sl], a[:, sl], rtol=1e-12, atol=1e-12 * np.abs(a).max())
    assert not v[:, :1024].any() and not v[:, 2524:].any()


def test_step_range_argument_errors(nbr):
    s = nbr.plummer(1000, 1)
    c = nbr.Context(0)
    c.upload(s)
    for args in ((100, 10), (0, 0), (1024, 5)):
        with pytest.raises(nbr.NbrError) as e:
            c.step_range(nbr.FP64, nbr.KDK, args[0], args[1], 1.0, 1.0)
        assert e.value.status == 1
    with pytest.raises(nbr.NbrError):
        c.step_range(7, nbr.KDK, 0, 128, 1.0, 1.0)
    ptrs, ln = c.state_pointers()
    assert ln >= 1024 + 1024 and all(p for p in ptrs.values())
    c.close()


def _slices(ctx, prec, eps2, V, ld):
    out = torch.zeros((V, 3, ld), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()  # the zero fill runs on torch's stream, the slices on the context's
    for v in range(V):
        ctx.n3_slice_accel(prec, eps2, v, V, out[v])
    ctx.synchronize()
    return out


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "fp32c"])
@pytest.mark.parametrize("n", [300, 5000, 20000])
def test_newton3_slices_sum_to_the_forces(nbr, oracle, prec, n):
    """The Newton-3 slices of the multi-GPU partition: for any slice count
    their sum is every particle's acceleration (each pair once), against the
    oracle; slices beyond the number of row groups are empty (all zeros)."""
    s = nbr.plummer(n, 7)
    eps2 = 1e-6
    ref = oracle.accel(s["x"], s["y"], s["z"], s["m"], eps2=eps2, extended=True)
    ld = -(-n // 1024) * 1024
    with nbr.Context(0) as c:
        c.upload(s)
        for V in (1, 3, 8, 40):
            P = _slices(c, prec, eps2, V, ld).cpu().numpy()
            # a range of slices in one call (one pair launch) gives the same bits
            if V >= 3:
                Q = torch.zeros((V - 1, 3, ld), dtype=torch.float64, device="cuda")
                torch.cuda.synchronize()
                c.n3_slice_accel(prec, eps2, 1, V, Q, slice_end=V)
                c.synchronize()
                np.testing.assert_array_equal(Q.cpu().numpy(), P[1:])
            a = P[0].copy()
            for v in range(1, V):
                a += P[v]
            e = np.linalg.norm(a[:, :n] - ref, axis=0) / np.linalg.norm(ref, axis=0)
            if prec == 0:
                assert e.max() <= 1e-12, (V, e.max())
            else:
                assert np.median(e) <= 1e-6 and e.max() <= 1e-4, (V, np.median(e), e.max())
            # entries n .. past the last 256-particle block are the zero-mass
            # padding particles' own accelerations; past that block nothing is written
            nb = -(-n // 256)
            assert not P[:, :, nb * 256:].any()
            groups = -(-nb // 8)  # row groups of 8 blocks: at most that many non-empty slices
            assert sum(bool(P[v].any()) for v in range(V)) <= min(V, groups)


def _n3_emulated(nbr, s, prec, scheme, dt, steps, world, eps2, V=8):
    """Newton-3 across `world` emulated ranks on one GPU: each context
    computes its slices for every particle, the owned columns are exchanged
    by device copies (the all-to-all), each rank adds them in slice order for
    its receivers (nbr_step_range_sum), then positions are exchanged."""
    n = len(s["x"])
    ctxs = [nbr.Context(0) for _ in range(world)]
    for c in ctxs:
        c.upload(s)
    ld = max(-(-n // 1024) * 1024, world * nbr_shard.shard_bounds(n, world, 0)[1])
    if scheme == nbr.KDK:
        sched = [(0.5 * dt, dt)] + [(dt, dt)] * (steps - 1) + [(0.5 * dt, 0.0)]
    else:
        sched = [(dt, dt)] * steps
    for kick, drift in sched:
        P = torch.zeros((V, 3, ld), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        for r, c in enumerate(ctxs):
            v0, v1 = nbr_shard.slice_range(V, world, r)
            for v in range(v0, v1):
                c.n3_slice_accel(prec, eps2, v, V, P[v])
            c.synchronize()
        for r, c in enumerate(ctxs):
            i0, cnt, owned = nbr_shard.shard_bounds(n, world, r)
            if owned:
                src = P[:, :, i0:i0 + cnt].contiguous()
                torch.cuda.synchronize()
                c.step_range_sum(prec, scheme, i0, owned, kick, drift, 1.0, src)
        _exchange(ctxs, n)
    _gather_velocities(ctxs, n)
    out = ctxs[0].download()
    for c in ctxs:
        c.synchronize()
        c.close()
    return out


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "fp32c"])
@pytest.mark.parametrize("scheme", [0, 2], ids=["kdk", "euler"])
def test_newton3_emulated_ranks(nbr, oracle, prec, scheme):
    """1, 2 and 3 emulated ranks give the same bits (the sum order depends
    only on the slice count), and the oracle's trajectory."""
    n, eps2, dt, steps = 6000, 1e-6, 1e-3, 3
    s = nbr.plummer(n, 8)
    one = _n3_emulated(nbr, s, prec, scheme, dt, steps, 1, eps2)
    for world in (2, 3):
        got = _n3_emulated(nbr, s, prec, scheme, dt, steps, world, eps2)
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            np.testing.assert_array_equal(got[k], one[k], err_msg=k)
    want = oracle.kdk(s, dt, steps, eps2=eps2) if scheme == nbr.KDK else oracle.euler(s, dt, steps, eps2=eps2)
    tol = 1e-11 if prec == 0 else 1e-6
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.abs(one[k] - want[k]).max() <= tol, k


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "fp32c"])
def test_banded_newton3_evaluation(nbr, oracle, prec):
    """The banded whole-system Newton-3 evaluation (slices accumulated in
    order in an FP64 buffer, then the epilogue), forced by a test hook on a
    system small enough for the oracle: forces and a KDK run."""
    import os
    n, eps2 = 20000, 1e-6
    s = nbr.plummer(n, 12)
    os.environ["NBR_TEST_N3_SLICES"] = "5"
    try:
        with nbr.Context(0) as c:
            c.set_force_config(prec, 3, 8, 0)
            c.upload(s)
            a = c.forces(prec, eps2=eps2)
            c.upload(s)
            c.run(prec, 0, 2, 1e-3, 3, eps2=eps2)
            got = c.download()
    finally:
        del os.environ["NBR_TEST_N3_SLICES"]
    idx = np.arange(0, n, 53)
    ref = oracle.accel_subset(s["x"], s["y"], s["z"], s["m"], idx, eps2=eps2)
    e = np.linalg.norm(a[:, idx] - ref, axis=0) / np.linalg.norm(ref, axis=0)
    assert (e.max() <= 1e-12) if prec == 0 else (np.median(e) <= 1e-6 and e.max() <= 1e-4)
    want = oracle.kdk(s, 1e-3, 3, eps2=eps2)
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.abs(got[k] - want[k]).max() <= (1e-11 if prec == 0 else 1e-6), k


def test_banded_newton3_at_two_million(nbr, oracle):
    """N = 2^21: past the single-launch scratch limit, the default Newton-3
    evaluation runs in slices of bounded scratch; sampled receivers against
    the extended-precision oracle (FP64 to 1e-12, FP32C median 1e-6) and
    Newton's third law over all particles."""
    n, eps2 = 1 << 21, 1e-6
    s = nbr.plummer(n, 2)
    with nbr.Context(0) as c:
        c.upload(s)
        assert c.get_force_config(0, eps2)[0] == 3 and c.get_force_config(1, eps2)[0] == 3
        a64 = c.forces(0, eps2=eps2)
        a32 = c.forces(1, eps2=eps2)
    idx = np.random.default_rng(1).choice(n, 128, replace=False)
    ref = oracle.accel_subset(s["x"], s["y"], s["z"], s["m"], idx, eps2=eps2)
    e64 = np.linalg.norm(a64[:, idx] - ref, axis=0) / np.linalg.norm(ref, axis=0)
    e32 = np.linalg.norm(a32[:, idx] - ref, axis=0) / np.linalg.norm(ref, axis=0)
    assert e64.max() <= 1e-12, e64.max()
    assert np.median(e32) <= 1e-6, np.median(e32)
    for a in (a64, a32):
        net = np.abs((a * s["m"]).sum(axis=1)).max()
        assert net <= 1e-6 * (np.linalg.norm(a, axis=0) * s["m"]).sum()
