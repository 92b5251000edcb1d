"""k-point sharding across GPUs (one process per GPU).

k-points are independent setups (lapw1.F:50-67); the reference farms them
to separate lapw1 processes by k-chunks (lapw1para:246-256, 421-447).  Here
each rank of a torch.distributed job takes a balanced share of the k-points:
longest processing time first on the cost model N_k^2 (the setup is
quadratic in the basis size), no collective on the data path.  After the
local work, one gather brings the per-k results to every rank, together with
each rank's failure (if any), so a failed k-point is reported everywhere
instead of leaving the other ranks waiting.

The batch state records which k-points finished, so an interrupted batch
restarts at the first unfinished one (the reference has no restart inside
a lapw1 run; a failed k-chunk is rerun whole).
"""
from __future__ import annotations

import json
import os
import traceback
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence


def assign_kpoints(sizes: Sequence[int], world: int) -> List[List[int]]:
    """Indices of the k-points each rank sets up: greedy longest-first onto
    the least loaded rank, cost N_k^2; each rank's list is returned in
    ascending k order.  Every k-point goes to exactly one rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]) ** 2, i))
    load = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += int(sizes[i]) ** 2
    return [sorted(x) for x in out]


@dataclass
class BatchState:
    """Completed k indices of a batch, optionally persisted as JSON."""

    path: Optional[str] = None
    done: Dict[int, object] = field(default_factory=dict)

    @classmethod
    def load(cls, path: Optional[str]) -> "BatchState":
        st = cls(path=path)
        if path and os.path.exists(path):
            with open(path) as f:
                st.done = {int(k): v for k, v in json.load(f).items()}
        return st

    def mark(self, k: int, result) -> None:
        self.done[int(k)] = result
        if self.path:
            tmp = self.path + ".tmp"
            with open(tmp, "w") as f:
                json.dump({str(a): b for a, b in self.done.items()}, f)
            os.replace(tmp, self.path)

    def todo(self, ks: Sequence[int]) -> List[int]:
        return [k for k in ks if int(k) not in self.done]


class KShardError(RuntimeError):
    pass


def run_sharded(sizes: Sequence[int], worker: Callable[[int], object], rank: int = 0, world: int = 1,
                group=None, state: Optional[BatchState] = None) -> Dict[int, object]:
    """Run `worker(k)` for this rank's share of the k-points and gather all
    results on every rank.  `worker` returns a JSON-serialisable result
    (eigenvalues, timings, force contributions, ...).  If any rank fails,
    every rank raises KShardError naming the failed k-point after the
    gather; ranks never wait on a rank that died inside `worker`."""
    mine = assign_kpoints(sizes, world)[rank]
    state = state or BatchState()
    local: Dict[int, object] = {}
    err = None
    for k in mine:
        if k in state.done:
            local[k] = state.done[k]
            continue
        try:
            res = worker(k)
        except Exception as e:  # the failure is reported through the gather
            err = (rank, k, f"{type(e).__name__}: {e}", traceback.format_exc(limit=3))
            break
        local[k] = res
        state.mark(k, res)
    if world > 1:
        import torch.distributed as dist
        gathered: List[object] = [None] * world
        dist.all_gather_object(gathered, (local, err), group=group)
    else:
        gathered = [(local, err)]
    errors = [g[1] for g in gathered if g[1] is not None]
    if errors:
        r, k, msg, _ = errors[0]
        raise KShardError(f"k-point {k} failed on rank {r}: {msg}")
    out: Dict[int, object] = {}
    for loc, _ in gathered:
        out.update(loc)
    return dict(sorted(out.items()))


def allreduce_forces(local, group=None):
    """Band-energy gradients summed over the k-points of every rank.

    `local` is this rank's sum over its own k-points of w_k dE_k/dPOS (a
    float64 tensor [NDF, 3]; the k weights w_k of the BZ integration applied
    by the caller).  One all-reduce of 3 NDF doubles (NCCL between GPUs,
    gloo on CPU) gives every rank the total; with one rank it is returned
    unchanged.  This is the only collective of a force run: the setups and
    the per-k adjoints share nothing."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return local
    out = local.clone()
    dist.all_reduce(out, op=dist.ReduceOp.SUM, group=group)
    return out
