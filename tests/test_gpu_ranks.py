"""The multi-rank path of bench.py --gpus N through the product: every rank
holds a serve session of the persistent kernel and submits its subtree share
of every job (e13_serve_submit_shard); e13shard sums the per-job counts and
gathers the survivor lines.  The ranks here are two processes on the one GPU
of this machine, joined by gloo: their kernels never wait on one another (each
rank searches its own shares and the ranks meet only on the host, at the end),
so sharing a GPU changes their timing, not their results.  The combined
counts of the FMAX = 3 local-edit search must equal the reference's log for
every deleted state, and the gathered lines its survivor file."""
import datetime
import os
import socket

import pytest
import torch.multiprocessing as mp

from gpu_common import golden_lines

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, entry, q):
    import sys

    sys.path.insert(0, HERE)
    sys.path.insert(0, os.path.join(os.path.dirname(HERE), "erdos-machine-13_b200"))
    import torch.distributed as dist

    import e13b200 as E
    import e13shard as S

    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}",
                            timeout=datetime.timedelta(seconds=300))
    try:
        base = E.load_machine(os.path.join(HERE, "golden", "machines", entry["machine"]))
        jobs = []
        for X in entry["X"]:
            r, job = E.setup(base, X, fmax=entry["fmax"])
            if r == 0:
                jobs.append((X, job))
        with E.Context(0) as ctx:
            with E.Server(ctx, E.tuning(epoch_us=20000)) as srv:
                got = srv.run_all([j for _, j in jobs], shard=rank, nshards=world)
            per, lines, status = {}, [], 0
            for i, (X, job) in enumerate(jobs):
                res, surv = got[i]
                status |= res.status
                per[X] = res.counts.as_dict()
                lines += [E.survivor_line(job, s) for s in surv]
        tot = S.sum_counts(dist, per)
        allines = S.gather_lines(dist, lines)
        q.put((rank, status, {X: per[X]["leaves"] for X in per}, tot, allines))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_ranks_share_every_job(searches, world):
    entry = searches["local_edits_f3"]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, entry, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res.sort()
    exp = {e["X"]: e for e in entry["expect"]}
    for rank, status, own, tot, lines in res:
        assert status == 0
        assert sum(own.values()) > 0  # every rank searched a share
        for X, c in tot.items():
            e = exp[X]
            assert (c["leaves"], c["survivors"], c["hist"]) == (e["leaves"], e["survivors"], e["hist"]), X
            if e["steps"] is not None:
                assert c["steps"] == e["steps"], X
        assert lines == golden_lines(entry)
    # the ranks split the work: neither did all of it
    for rank, _, own, _, _ in res:
        assert sum(own.values()) < sum(e["leaves"] for e in entry["expect"])
