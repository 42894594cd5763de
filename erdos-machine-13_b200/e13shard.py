"""Splitting a search workload over ranks (one process per GPU) and combining
the results.

A delete-mode workload is a list of independent jobs, one per deleted state X
(src/e13search.c:463-466 runs them one after another).  Two splits:
  * by job: rank r of N takes every N-th job starting at r (share());
  * by subtree: every rank takes shard r of N of every job (the library's
    e13_search_shard / e13_serve_submit_shard), which balances jobs of very
    different sizes; the expansion before the deal counts in shard 0 only.
Either way the ranks run with no communication and meet once at the end: one
sum of the integer counters (leaves, survivors, steps, deaths per stage), per
job (sum_counts) or in total (reduce_totals), one maximum of the per-rank
times (the job takes as long as its slowest rank) and one gather of the
survivor lines, which are sorted because survivor order is unspecified
(src/e13search.c:185).

`dist` is `torch.distributed` with an initialised process group: NCCL for
device tensors on the GPUs, gloo for CPU tensors.
"""
from __future__ import annotations


def share(items, rank: int, world: int) -> list:
    """This rank's jobs: items[rank], items[rank + world], ..."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return [x for i, x in enumerate(items) if i % world == rank]


def reduce_totals(dist, sums: dict, maxes: dict, device="cpu") -> tuple[dict, dict]:
    """Sums over ranks of the integer counters in `sums` and maxima of the
    numbers in `maxes`.  Every rank passes the same keys and gets the same
    result."""
    import torch

    ks, km = sorted(sums), sorted(maxes)
    s = torch.tensor([int(sums[k]) for k in ks], dtype=torch.int64, device=device)
    m = torch.tensor([float(maxes[k]) for k in km], dtype=torch.float64, device=device)
    if ks:
        dist.all_reduce(s, op=dist.ReduceOp.SUM)
    if km:
        dist.all_reduce(m, op=dist.ReduceOp.MAX)
    return ({k: int(v) for k, v in zip(ks, s.tolist())}, {k: float(v) for k, v in zip(km, m.tolist())})


def gather_lines(dist, lines: list[str]) -> list[str]:
    """Survivor lines of all ranks, sorted (the same list on every rank)."""
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, list(lines))
    return sorted(l for p in parts for l in p)


def sum_counts(dist, per_job: dict, device="cpu") -> dict:
    """Per-job counts {key: {leaves, survivors, steps, hist[10]}} summed over
    ranks; every rank passes the same keys in any order and gets the sums."""
    import torch

    keys = sorted(per_job)
    flat = []
    for k in keys:
        c = per_job[k]
        flat += [int(c["leaves"]), int(c["survivors"]), int(c["steps"])] + [int(h) for h in c["hist"]]
    t = torch.tensor(flat, dtype=torch.int64, device=device)
    if flat:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    v = t.tolist()
    out = {}
    for i, k in enumerate(keys):
        r = v[13 * i: 13 * i + 13]
        out[k] = {"leaves": r[0], "survivors": r[1], "steps": r[2], "hist": r[3:13]}
    return out
