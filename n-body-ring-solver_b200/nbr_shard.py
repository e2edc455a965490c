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

The context object only needs upload / step_range / state_tensors /
state_changed / download and a `stream` attribute (nbr.Context provides
them), so the host logic here is independent of where the arithmetic runs.
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


class ShardedSystem:
    """A system integrated by `world` processes, one context each.

    ctx: this rank's context; group: the torch.distributed process group
    (default: the world).  The context's stream orders everything: the
    exchange runs on it (torch.cuda.ExternalStream) for device tensors."""

    def __init__(self, ctx, group=None):
        self.ctx = ctx
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.n = 0
        self.collectives = 0

    # ---------------------------------------------------------------- state --
    def upload(self, system: Dict[str, np.ndarray]):
        """Every rank uploads the same whole system (the reference broadcasts
        masses and positions from rank 0, CPU/hybrid_solver.cpp:249-262); the
        caller passes identical arrays on all ranks."""
        self.ctx.upload(system)
        self.n = len(system["x"])
        self.i0, self.count, self.owned = shard_bounds(self.n, self.world, self.rank)

    def _stream_ctx(self, t: torch.Tensor):
        if t.is_cuda:
            return torch.cuda.stream(torch.cuda.ExternalStream(self.ctx.stream, device=t.device))
        return _Null()

    def _all_gather(self, arrays):
        """All-gathers the owned slices [i0, i0 + count) of each array in
        place: after it, every rank's arrays hold every rank's slice."""
        c, w, r = self.count, self.world, self.rank
        t0 = arrays[0]
        if w * c > t0.numel():
            raise RuntimeError(f"shards of {c} x {w} exceed the arrays' {t0.numel()} entries")
        with self._stream_ctx(t0):
            mine = torch.stack([a[r * c:(r + 1) * c] for a in arrays])          # [k, c]
            kk = mine.shape[0]
            out = torch.empty((w * kk, c), dtype=mine.dtype, device=mine.device)
            dist.all_gather_into_tensor(out, mine, group=self.group)           # [w * k, c]
            out = out.view(w, kk, c)
            for k, a in enumerate(arrays):
                a[:w * c].view(w, c).copy_(out[:, k, :])
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
        if self.owned > 0:
            self.ctx.step_range(precision, scheme, self.i0, self.owned, kick, drift, G, eps2)
        self.exchange_positions()

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
