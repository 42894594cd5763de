"""The multi-rank path on CPU: gloo ranks split the FMAX = 2 local-edit search
by deleted state X, each runs its share on the oracle, and the combined
totals and survivor lines must equal the reference's whole-run log."""
import datetime
import os
import socket

import pytest
import torch.multiprocessing as mp

from gpu_common import golden_lines

HERE = os.path.dirname(os.path.abspath(__file__))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, entry, q):
    import time

    import torch.distributed as dist

    import e13shard as S
    import oracle_lib as O

    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}",
                            timeout=datetime.timedelta(seconds=120))
    try:
        base = O.load_machine(entry["machine"])
        sums = {"leaves": 0, "survivors": 0, "steps": 0}
        sums.update({f"hist{j}": 0 for j in range(10)})
        lines = []
        t0 = time.perf_counter()
        mine = S.share(entry["X"], rank, world)
        for X in mine:
            r, job = O.setup(base, X, fmax=entry["fmax"])
            c, recs = O.search(job, nthreads=2)
            for k in ("leaves", "survivors", "steps"):
                sums[k] += c[k]
            for j in range(10):
                sums[f"hist{j}"] += c["hist"][j]
            lines += [O.survivor_line(X, rec, job.nq) for rec in recs]
        tot, mx = S.reduce_totals(dist, sums, {"wall": time.perf_counter() - t0, "jobs": len(mine)})
        q.put((rank, mine, tot, mx, S.gather_lines(dist, lines)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_f2_equals_whole_run(searches, world):
    entry = searches["local_edits_f2"]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, entry, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort()
    # every X on exactly one rank
    xs = sorted(x for _, mine, _, _, _ in got for x in mine)
    assert xs == entry["X"]
    want = {"leaves": sum(e["leaves"] for e in entry["expect"]),
            "survivors": sum(e["survivors"] for e in entry["expect"]),
            "steps": sum(e["steps"] for e in entry["expect"])}
    want.update({f"hist{j}": sum(e["hist"][j] for e in entry["expect"]) for j in range(10)})
    gold = golden_lines(entry)
    for rank, mine, tot, mx, lines in got:
        assert tot == want
        assert mx["jobs"] == max(len(m) for _, m, _, _, _ in got)
        assert lines == gold


def _rank_main_subtrees(rank, world, port, entry, q):
    """Every rank searches shard `rank` of `world` of every job (the oracle's
    subtree split: the serial walk's own leaves count in shard 0 only), then
    the ranks sum the per-job counts and gather the survivor lines."""
    import torch.distributed as dist

    import e13shard as S
    import oracle_lib as O

    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}",
                            timeout=datetime.timedelta(seconds=120))
    try:
        base = O.load_machine(entry["machine"])
        per, lines, shard0 = {}, [], {}
        for X in entry["X"]:
            r, job = O.setup(base, X, fmax=entry["fmax"])
            c, recs = O.search(job, nthreads=2, shard=rank, nshards=world)
            per[X] = c
            lines += [O.survivor_line(X, rec, job.nq) for rec in recs]
        q.put((rank, per, S.sum_counts(dist, per), S.gather_lines(dist, lines)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_subtree_sharded_f2_equals_whole_run(searches, world):
    """The split the sharded bench uses: every rank takes its share of every
    job; the per-job sums over ranks equal the reference's per-X log lines and
    the gathered survivor lines its survivor file.  Each rank's share is a
    proper part: no rank alone has a whole job's leaves."""
    entry = searches["local_edits_f2"]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main_subtrees, args=(r, world, port, entry, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    gold = golden_lines(entry)
    exp = {e["X"]: e for e in entry["expect"]}
    for rank, per, summed, lines in got:
        assert lines == gold
        for X, e in exp.items():
            assert summed[X] == {k: e[k] for k in ("leaves", "survivors", "steps", "hist")}, (rank, X)
    big = max(exp, key=lambda X: exp[X]["leaves"])
    assert all(per[big]["leaves"] < exp[big]["leaves"] for _, per, _, _ in got)


def test_share_rejects_bad_rank():
    import e13shard as S

    assert S.share(list(range(14)), 1, 4) == [1, 5, 9, 13]
    with pytest.raises(ValueError):
        S.share([1, 2], 2, 2)
