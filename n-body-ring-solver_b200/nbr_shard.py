"""One system split over several GPUs by receivers (the i-partition).

Each process drives one GPU through its own libnbr context.  Every context
holds the whole system; rank r owns the receivers [r * count, (r + 1) * count)
with count = n / world rounded up to a multiple of 128.  A step evaluates the
owned receivers against all n sources and updates them (nbr_step_range), then
one all-gather over the process group gives every rank the new positions of
all particles.  This is hybrid_full_solver (CPU/hybrid_solver.cpp:226-336) on
GPUs: MPI_Bcast of masses and positions (:249-254), the owned slice's forces
against all N (:288), its update (:290-299) and MPI_Allgather of the
positions (:310), here an NCCL all-gather over NVLink on the context's stream.

The exchange is the only collective, once per force evaluation, 24 bytes per
particle.  Velocities stay with their owner until gather_velocities().

method="newton3" evaluates each unordered pair once across the ranks, as
hybrid_ring_solver does by sending partial forces around the ring with the
positions (CPU/hybrid_solver.cpp:52-107): the block-pair triangle is cut
into `slices` slices of equal pair work (nbr_n3_slice_accel), rank r
computes slices [r V / W, (r + 1) V / W) for every particle, an all-to-all
hands each rank every slice's partials of its own receivers, and the rank
adds them in slice order and updates its receivers (nbr_step_range_sum);
then the position all-gather.  The sum order depends only on V, so any
world size W <= V gives the same bits.  Per step and rank: V/W slice
launches, (V/W) x 24 B x n out and about 24 B x n in, plus the all-gather.

The context object only needs upload / step_range (n3_slice_accel /
step_range_sum for newton3) / state_tensors / state_changed / download and a
`stream` attribute (nbr.Context provides them), so the host logic here is
independent of where the arithmetic runs.
"""
from __future__ import annotations

from typing import Dict, Tuple

import numpy as np
import torch
import torch.distributed as dist

TILE = 128


def shard_bounds(n: int, world: int, rank: int) -> Tuple[int, int, int]:
    """(i0, count, owned) of rank: i0 = rank * count, count = the equal,
    128-aligned shard length used by the exchange, owned = the real receivers
    of this rank (count clipped to n; 0 when the rank owns none)."""
    if n <= 0 or world <= 0 or not 0 <= rank < world:
        raise ValueError("need n > 0 and 0 <= rank < world")
    count = -(-n // world)
    count = -(-count // TILE) * TILE
    i0 = rank * count
    owned = max(0, min(count, n - i0))
    return i0, count, owned


def slice_range(slices: int, world: int, rank: int) -> Tuple[int, int]:
    """Slices [v0, v1) of the Newton-3 partition computed by rank (ranks in
    order hold consecutive slices, so receiving in rank order is slice order)."""
    return rank * slices // world, (rank + 1) * slices // world


class ShardedSystem:
    """A system integrated by `world` processes, one context each.

    ctx: this rank's context; group: the torch.distributed process group
    (default: the world).  The context's stream orders everything: the
    exchange runs on it (torch.cuda.ExternalStream) for device tensors."""

    def __init__(self, ctx, group=None, method: str = "range", slices: int = 8):
        self.ctx = ctx
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.n = 0
        self.collectives = 0
        if method not in ("range", "newton3"):
            raise ValueError("method is 'range' or 'newton3'")
        if method == "newton3" and slices < self.world:
            raise ValueError("newton3 needs at least one slice per rank")
        self.method = method
        self.slices = slices

    # ---------------------------------------------------------------- state --
    def upload(self, system: Dict[str, np.ndarray]):
        """Every rank uploads the same whole system (the reference broadcasts
        masses and positions from rank 0, CPU/hybrid_solver.cpp:249-262); the
        caller passes identical arrays on all ranks."""
        self.ctx.upload(system)
        self.n = len(system["x"])
        self.i0, self.count, self.owned = shard_bounds(self.n, self.world, self.rank)
        if self.method == "newton3":
            V, W, c = self.slices, self.world, self.count
            dev = self.ctx.state_tensors()["x"].device
            n_pad = -(-self.n // 1024) * 1024
            ld = max(n_pad, W * c)
            self.v0, self.v1 = slice_range(V, W, self.rank)
            # this rank's slices for every particle; every slice for own receivers
            self._mine = torch.zeros((self.v1 - self.v0, 3, ld), dtype=torch.float64, device=dev)
            self._recv = torch.zeros((V, 3, c), dtype=torch.float64, device=dev)
            if dev.type == "cuda":
                torch.cuda.synchronize(dev)  # zero fills done before the context's stream uses them

    def _stream_ctx(self, t: torch.Tensor):
        if t.is_cuda:
            return torch.cuda.stream(torch.cuda.ExternalStream(self.ctx.stream, device=t.device))
        return _Null()

    def _all_gather(self, arrays):
        """All-gathers the owned slices [i0, i0 + count) of each array in
        place (one all-gather per array, no staging copies): after it, every
        rank's arrays hold every rank's slice."""
        c, w, r = self.count, self.world, self.rank
        t0 = arrays[0]
        if w * c > t0.numel():
            raise RuntimeError(f"shards of {c} x {w} exceed the arrays' {t0.numel()} entries")
        with self._stream_ctx(t0):
            for a in arrays:
                # in place: this rank's shard is already where the gather puts it
                dist.all_gather_into_tensor(a[:w * c], a[r * c:(r + 1) * c], group=self.group)
        self.collectives += 1

    def exchange_positions(self):
        st = self.ctx.state_tensors()
        self._all_gather([st["x"], st["y"], st["z"]])
        self.ctx.state_changed()

    def gather_velocities(self):
        st = self.ctx.state_tensors()
        self._all_gather([st["vx"], st["vy"], st["vz"]])
        self.ctx.state_changed()

    # ------------------------------------------------------------- stepping --
    def step(self, precision: int, scheme: int, kick: float, drift: float, G: float = 1.0,
             eps2: float = 0.0):
        """One force evaluation of the owned receivers with the fused update,
        then the position exchange.  A rank that owns no receivers only takes
        part in the exchange, which overwrites all n positions of its current
        buffer."""
        if self.method == "newton3":
            self._step_newton3(precision, scheme, kick, drift, G, eps2)
        elif self.owned > 0:
            self.ctx.step_range(precision, scheme, self.i0, self.owned, kick, drift, G, eps2)
        self.exchange_positions()

    def _step_newton3(self, precision, scheme, kick, drift, G, eps2):
        V, W, c = self.slices, self.world, self.count
        nv = self.v1 - self.v0
        with self._stream_ctx(self._mine):
            self.ctx.n3_slice_accel(precision, eps2, self.v0, V, self._mine, slice_end=self.v1)
            # columns of every rank's receivers: [W][nv][3][c] out, [V][3][c] in
            send = self._mine[:, :, :W * c].reshape(nv, 3, W, c).permute(2, 0, 1, 3).contiguous()
            out_splits = [(slice_range(V, W, q)[1] - slice_range(V, W, q)[0]) * 3 * c
                          for q in range(W)]
            dist.all_to_all_single(self._recv.view(-1), send.view(-1), out_splits,
                                   [nv * 3 * c] * W, group=self.group)
            if self.owned > 0:
                self.ctx.step_range_sum(precision, scheme, self.i0, self.owned, kick, drift, G,
                                        self._recv)
        self.collectives += 1

    def run(self, precision: int, scheme: int, dt: float, steps: int, G: float = 1.0,
            eps2: float = 0.0) -> int:
        """Advances `steps` steps; returns the force evaluations made.
        scheme KDK (the module's nbr.KDK = 0): steps + 1 evaluations with the
        half kicks of neighbouring steps merged; scheme EULER (2): explicit
        Euler as hybrid_full_solver (x += v dt, v += a dt), one per step."""
        if steps <= 0:
            return 0
        if scheme == 2:
            for _ in range(steps):
                self.step(precision, 2, dt, dt, G, eps2)
            return steps
        if scheme != 0:
            raise ValueError("the i-partition runs KDK (0) or Euler (2)")
        self.step(precision, 0, 0.5 * dt, dt, G, eps2)
        for _ in range(steps - 1):
            self.step(precision, 0, dt, dt, G, eps2)
        self.step(precision, 0, 0.5 * dt, 0.0, G, eps2)
        return steps + 1

    def download(self) -> Dict[str, np.ndarray]:
        """The whole state on every rank (velocities gathered first)."""
        self.gather_velocities()
        return self.ctx.download()


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False
