"""Host logic of the multi-GPU i-partition (nbr_shard.py), on CPU.

Ranks are gloo processes.  Each drives a stand-in context whose arithmetic
is the oracle's (CPU) and whose state layout is the library's: double
buffered positions of n_pad + 1024 entries, a receiver-range step that
writes only its range of the other buffer.  What is checked is the
partition and the exchange: any world size must give bit-for-bit the
single-rank trajectory, which itself follows the oracle's KDK / Euler.
The GPU side of nbr_step_range is checked in test_gpu_shard.py.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import nbr_shard


class OracleRangeContext:
    """The calls nbr_shard.ShardedSystem makes on a context, computed by the
    oracle on CPU tensors with the library's buffer conventions."""

    def __init__(self):
        from oracle import Oracle
        self.orc = Oracle()
        self.stream = 0

    def upload(self, s):
        n = len(s["x"])
        self.n = n
        ln = -(-n // 1024) * 1024 + 1024
        self.pos = [[np.zeros(ln) for _ in range(3)] for _ in range(2)]
        self.vel = [np.zeros(ln) for _ in range(3)]
        self.m = np.zeros(ln)
        for d, k in enumerate("xyz"):
            self.pos[0][d][:n] = s[k]
            self.vel[d][:n] = s["v" + k]
        self.m[:n] = s["m"]
        self.cur = 0

    def step_range(self, precision, scheme, i0, count, kick, drift, G=1.0, eps2=0.0):
        n, a, b = self.n, self.cur, 1 - self.cur
        x, y, z = (p[:n] for p in self.pos[a])
        acc = self.orc.accel(x.copy(), y.copy(), z.copy(), self.m[:n].copy(), G, eps2)
        r = slice(i0, i0 + count)
        for d in range(3):
            v_old = self.vel[d][r].copy()
            self.vel[d][r] += kick * acc[d][r]
            v_drift = v_old if scheme == 2 else self.vel[d][r]
            self.pos[b][d][r] = self.pos[a][d][r] + drift * v_drift
        self.cur = b

    def n3_slice_accel(self, precision, eps2, v0, V, dst, slice_end=None):
        """Stand-in slices [v0, slice_end): the accelerations from the sources
        of index block v of V (a different partition of the pairs than the
        library's, with the same property: the V slices together hold each
        pair once)."""
        n = self.n
        v1 = v0 + 1 if slice_end is None else slice_end
        out = dst.view(v1 - v0, 3, -1)
        for v in range(v0, v1):
            lo, hi = n * v // V, n * (v + 1) // V
            m = np.zeros(n)
            m[lo:hi] = self.m[lo:hi]
            x, y, z = (p[:n].copy() for p in self.pos[self.cur])
            a = self.orc.accel(x, y, z, m, 1.0, eps2)
            out[v - v0].zero_()
            out[v - v0, :, :n] = torch.from_numpy(a)

    def step_range_sum(self, precision, scheme, i0, count, kick, drift, G, src):
        n, a, b = self.n, self.cur, 1 - self.cur
        cnt = min(count, n - i0)
        acc = np.zeros((3, cnt))
        for v in range(src.shape[0]):  # slice order
            acc += src[v, :, :cnt].numpy()
        acc *= G
        r = slice(i0, i0 + cnt)
        for d in range(3):
            v_old = self.vel[d][r].copy()
            self.vel[d][r] += kick * acc[d]
            v_drift = v_old if scheme == 2 else self.vel[d][r]
            self.pos[b][d][r] = self.pos[a][d][r] + drift * v_drift
        self.cur = b

    def state_tensors(self):
        p = self.pos[self.cur]
        return {"x": torch.from_numpy(p[0]), "y": torch.from_numpy(p[1]), "z": torch.from_numpy(p[2]),
                "vx": torch.from_numpy(self.vel[0]), "vy": torch.from_numpy(self.vel[1]),
                "vz": torch.from_numpy(self.vel[2])}

    def state_changed(self):
        pass

    def download(self):
        n, p = self.n, self.pos[self.cur]
        return {"x": p[0][:n].copy(), "y": p[1][:n].copy(), "z": p[2][:n].copy(),
                "vx": self.vel[0][:n].copy(), "vy": self.vel[1][:n].copy(), "vz": self.vel[2][:n].copy()}


def _system(n, seed):
    rng = np.random.default_rng(seed)
    s = {k: rng.standard_normal(n) for k in ("x", "y", "z")}
    s.update({k: 0.1 * rng.standard_normal(n) for k in ("vx", "vy", "vz")})
    s["m"] = rng.uniform(0.5, 1.5, n) / n
    return s


def _worker(rank, world, port, outdir, n, scheme, steps, method="range"):
    os.environ["OMP_NUM_THREADS"] = "1"
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            init_method=f"tcp://127.0.0.1:{port}")
    try:
        ctx = OracleRangeContext()
        sh = nbr_shard.ShardedSystem(ctx, method=method, slices=8)
        sh.upload(_system(n, 11))
        evals = sh.run(0, scheme, 1e-3, steps, G=1.0, eps2=1e-4)
        out = sh.download()
        np.savez(os.path.join(outdir, f"w{world}_r{rank}.npz"), evals=evals,
                 collectives=sh.collectives, owned=sh.owned, **out)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(world, tmp_path, n, scheme, steps, method="range"):
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path), n, scheme, steps, method),
                       nprocs=world, join=True, start_method="spawn")
    return [dict(np.load(tmp_path / f"w{world}_r{r}.npz")) for r in range(world)]


@pytest.mark.parametrize("n,world", [(1000, 3), (1000, 8), (200, 4), (4096, 2), (128, 1)])
def test_shard_bounds_partition(n, world):
    owned_total = 0
    ln = -(-n // 1024) * 1024 + 1024  # the library's allocated length
    prev_end = 0
    for r in range(world):
        i0, count, owned = nbr_shard.shard_bounds(n, world, r)
        assert count % 128 == 0 and i0 == r * count
        if owned:
            assert i0 == prev_end
            prev_end = i0 + owned
        owned_total += owned
        assert world * count <= ln  # the in-place exchange stays inside the arrays
    assert owned_total == n and prev_end == n


def test_shard_bounds_rejects_bad_args():
    with pytest.raises(ValueError):
        nbr_shard.shard_bounds(0, 2, 0)
    with pytest.raises(ValueError):
        nbr_shard.shard_bounds(10, 2, 2)


@pytest.mark.parametrize("scheme", [0, 2], ids=["kdk", "euler"])
def test_sharded_run_matches_single_rank(tmp_path, oracle, scheme):
    n, steps = 1000, 3
    one = _run(1, tmp_path, n, scheme, steps)[0]
    s0 = _system(n, 11)
    ref = oracle.kdk(s0, 1e-3, steps, 1.0, 1e-4) if scheme == 0 else oracle.euler(s0, 1e-3, steps, 1.0, 1e-4)
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_allclose(one[k], ref[k], rtol=1e-12, atol=1e-14)
    for world in (2, 3):
        outs = _run(world, tmp_path, n, scheme, steps)
        assert sum(int(o["owned"]) for o in outs) == n
        for o in outs:
            assert int(o["evals"]) == (steps + 1 if scheme == 0 else steps)
            # one position exchange per evaluation, one velocity gather at the end
            assert int(o["collectives"]) == int(o["evals"]) + 1
            for k in ("x", "y", "z", "vx", "vy", "vz"):
                np.testing.assert_array_equal(o[k], one[k])


def test_ranks_without_receivers_still_exchange(tmp_path):
    n = 200  # four ranks of 128: ranks 2 and 3 own nothing
    one = _run(1, tmp_path, n, 0, 2)[0]
    outs = _run(4, tmp_path, n, 0, 2)
    assert [int(o["owned"]) for o in outs] == [128, 72, 0, 0]
    for o in outs:
        for k in ("x", "vx", "vz"):
            np.testing.assert_array_equal(o[k], one[k])


@pytest.mark.parametrize("scheme", [0, 2], ids=["kdk", "euler"])
def test_newton3_partition_matches_single_rank_and_oracle(tmp_path, oracle, scheme):
    """Newton-3 across ranks: 8 slices spread over 1, 2, 3 or 4 ranks, the
    partials exchanged by an all-to-all and added in slice order.  Every world
    size gives the single rank's bits, which follow the oracle's trajectory."""
    n, steps = 1000, 3
    one = _run(1, tmp_path, n, scheme, steps, "newton3")[0]
    s0 = _system(n, 11)
    ref = oracle.kdk(s0, 1e-3, steps, 1.0, 1e-4) if scheme == 0 else oracle.euler(s0, 1e-3, steps, 1.0, 1e-4)
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_allclose(one[k], ref[k], rtol=1e-12, atol=1e-14)
    for world in (2, 3, 4):
        outs = _run(world, tmp_path, n, scheme, steps, "newton3")
        assert sum(int(o["owned"]) for o in outs) == n
        for o in outs:
            # per evaluation: the slice all-to-all and the position all-gather
            assert int(o["collectives"]) == 2 * int(o["evals"]) + 1
            for k in ("x", "y", "z", "vx", "vy", "vz"):
                np.testing.assert_array_equal(o[k], one[k])


def test_slice_range_covers_the_slices():
    for V in (1, 5, 8, 16):
        for W in range(1, V + 1):
            got = [nbr_shard.slice_range(V, W, r) for r in range(W)]
            assert got[0][0] == 0 and got[-1][1] == V
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            assert all(v1 > v0 for v0, v1 in got)
