"""Multi-GPU plumbing for a path whose units (image pairs) are independent:
replicas with no collective on the data path.

- pair_indices: the pairs one rank registers when every rank runs its own
  fixed share (weak scaling, one process per GPU).
- max_over_ranks: the job's time is the slowest rank's device time.
- LeastLoadedDispatcher: host-side placement of served requests over the
  GPUs of one node, by the device-memory footprint each GPU has admitted
  and not yet released (an admission budget per GPU).
"""
from __future__ import annotations

from dataclasses import dataclass, field


def pair_indices(pairs_per_rank: int, rank: int) -> range:
    """Global indices of the pairs rank `rank` registers (seeds follow them)."""
    if pairs_per_rank < 0 or rank < 0:
        raise ValueError("pairs_per_rank and rank must be nonnegative")
    return range(rank * pairs_per_rank, (rank + 1) * pairs_per_rank)


def max_over_ranks(values, device=None) -> list[float]:
    """Element-wise maximum of `values` over all ranks of the default process
    group (the values themselves with no group)."""
    import torch
    import torch.distributed as dist
    vals = [float(v) for v in values]
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return vals
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


@dataclass
class LeastLoadedDispatcher:
    """Places each request on the GPU with the most free admission budget
    (ties: the lowest index). A request beyond that GPU's free budget still
    goes there and waits in that GPU's own admission queue; one larger than
    every budget is refused (ValueError)."""

    budgets: list[int]
    used: list[int] = field(default_factory=list)
    placed: dict = field(default_factory=dict)  # tag -> (gpu, bytes)

    def __post_init__(self):
        if not self.budgets or any(b <= 0 for b in self.budgets):
            raise ValueError("every GPU needs a positive budget")
        self.used = [0] * len(self.budgets)

    def place(self, tag, nbytes: int) -> int:
        if tag in self.placed:
            raise ValueError(f"request {tag!r} is already placed")
        fits = [g for g, b in enumerate(self.budgets) if nbytes <= b]
        if not fits:
            raise ValueError("request larger than every GPU's budget")
        best = max(fits, key=lambda g: (self.budgets[g] - self.used[g], -g))
        self.used[best] += nbytes
        self.placed[tag] = (best, nbytes)
        return best

    def release(self, tag) -> int:
        gpu, nbytes = self.placed.pop(tag)
        self.used[gpu] -= nbytes
        return gpu
