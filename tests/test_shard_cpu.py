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


def test_share_rejects_bad_rank():
    import e13shard as S

    assert S.share(list(range(14)), 1, 4) == [1, 5, 9, 13]
    with pytest.raises(ValueError):
        S.share([1, 2], 2, 2)
