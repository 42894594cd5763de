"""The serving loop: many searches interleaved in one persistent kernel.
Every job's counts and survivors in the mix must equal the reference's
(golden) and those of the same job searched alone."""
import random

import pytest

import e13b200 as E
import oracle_lib as O
from gpu_common import check_entry, ctx, golden_lines, make_job

pytestmark = pytest.mark.gpu


def _small_mix(searches):
    """(entry, X) pairs of golden searches that finish quickly."""
    out = []
    for X in range(14):
        out.append((searches["local_edits_f2"], X))
    for name in ("doubling_X0", "doubling_X1", "doubling_X2", "split_test_free", "counters_f2_base_01",
                 "counters_f2_base_13", "counters_f2_base_44"):
        e = searches[name]
        out.append((e, e["X"] if not isinstance(e["X"], list) else e["X"][0]))
    out.append((searches["split_test"], 14))
    return out


def _expect(e, X):
    xs = e["X"] if isinstance(e["X"], list) else [e["X"]]
    return e["expect"][xs.index(X)]


def test_mix_equals_golden_and_alone(searches):
    mix = _small_mix(searches)  # 22 jobs: more than the 16 slots, so some wait for a slot
    jobs = [make_job(e, X) for e, X in mix]
    with E.Server(ctx()) as srv:
        got = srv.run_all(jobs)
    assert sorted(got) == list(range(len(jobs)))
    for i, (e, X) in enumerate(mix):
        res, surv = got[i]
        assert res.status == 0
        check_entry(dict(e, expect=[_expect(e, X)]), [res.counts.as_dict()])
        alone, alone_surv = ctx().search(jobs[i])
        assert res.counts.as_dict() == alone.as_dict()
        lines = sorted(E.survivor_line(jobs[i], s) for s in surv)
        assert lines == sorted(E.survivor_line(jobs[i], s) for s in alone_surv)


def test_staggered_arrivals(searches):
    """Jobs arrive while others run (seeded arrival times); results unchanged."""
    mix = _small_mix(searches)[:12] + [(searches["local_edits_f3"], X) for X in (4, 9, 12)]
    jobs = [make_job(e, X) for e, X in mix]
    rng = random.Random(7)
    t, arrivals = 0.0, []
    for _ in jobs:
        t += rng.expovariate(50.0)  # about 20 ms apart
        arrivals.append(t)
    with E.Server(ctx()) as srv:
        got = srv.run_all(jobs, arrivals)
    for i, (e, X) in enumerate(mix):
        res, surv = got[i]
        check_entry(dict(e, expect=[_expect(e, X)]), [res.counts.as_dict()])
        assert res.t_start >= res.t_submit and res.t_done >= res.t_start


def test_big_and_small_jobs_interleave(searches):
    """A large job (division V4, 8.3e8 leaves) next to small ones: all exact."""
    mix = [(searches["division_v4"], 9)] + _small_mix(searches)[:8] + [(searches["counter_sym"], 13)]
    jobs = [make_job(e, X) for e, X in mix]
    with E.Server(ctx()) as srv:
        got = srv.run_all(jobs)
    for i, (e, X) in enumerate(mix):
        res, surv = got[i]
        check_entry(dict(e, expect=[_expect(e, X)]), [res.counts.as_dict()])
    res, surv = got[len(mix) - 1]
    assert sorted(E.survivor_line(jobs[-1], s) for s in surv) == golden_lines(searches["counter_sym"])


def _swap_mix(searches):
    return [(searches["local_edits_f3"], X) for X in range(14)] + [(searches["counter_sym"], 13)]


def _check_mix(searches, mix, jobs, got):
    for i, (e, X) in enumerate(mix):
        res, surv = got[i]
        assert res.status == 0, (X, res.status)
        check_entry(dict(e, expect=[_expect(e, X)]), [res.counts.as_dict()])
    res, surv = got[len(mix) - 1]
    assert sorted(E.survivor_line(jobs[-1], s) for s in surv) == golden_lines(searches["counter_sym"])


def test_preempted_jobs_resume_exactly(searches):
    """Jobs preempted between steps (e13_serve_preempt: frontier nodes and
    counters to host memory, back to the head of the queue) resume where they
    stopped: every job's counts and survivors equal the reference's."""
    mix = _swap_mix(searches)
    jobs = [make_job(e, X) for e, X in mix]
    with E.Server(ctx(), E.tuning(epoch_us=2000)) as srv:
        for i, job in enumerate(jobs):
            srv.submit(job, i)
        got, steps = {}, 0
        while srv.pending():
            for r in srv.step():
                got[r.id] = (r, srv.survivors(r.id))
            steps += 1
            left = [i for i in range(len(jobs)) if i not in got]
            if steps % 3 == 0 and left:  # preempt the lowest-numbered unfinished job (a no-op while it is queued)
                srv.preempt(left[0])
        swaps = srv.swapped_out()
    assert swaps > 0
    _check_mix(searches, mix, jobs, got)


def test_swap_out_when_the_frontier_runs_out_of_room(searches):
    """A frontier with room for one epoch's outputs and 20,000 nodes more: the
    14 FMAX = 2 jobs fit in it (a frontier node leads to at least one leaf of
    its own, and none of them has 20,000 leaves), the FMAX = 3 job X = 11
    (1.4e7 leaves, over 10^5 machines live at once on a full GPU) does not.  After an epoch the session swaps out the job with the most live
    nodes, so the large job goes to host memory while the small ones finish
    (each equal to the reference's log); alone, it still does not fit and ends
    with E13_ERR_OVERFLOW, the session going on."""
    mix = [(searches["local_edits_f2"], X) for X in range(14)] + [(searches["local_edits_f3"], 11)]
    jobs = [make_job(e, X) for e, X in mix]
    out_nodes = 2 * (148 * 768 // 32) * (32 + 256) + 65536  # one epoch's output room at the default shape
    tune = E.tuning(epoch_us=2000, stack_nodes=out_nodes + 20000)
    with E.Server(ctx(), tune, reserve_nodes=64) as srv:
        got = srv.run_all(jobs)
        swaps = srv.swapped_out()
    assert swaps > 0
    for i, (e, X) in enumerate(mix[:-1]):
        res, surv = got[i]
        assert res.status == 0, (X, res.status)
        check_entry(dict(e, expect=[_expect(e, X)]), [res.counts.as_dict()])
    assert got[len(mix) - 1][0].status == -6  # E13_ERR_OVERFLOW


def test_admission_reserves_by_estimate(searches):
    """With estimate-based reservations many small jobs run at once next to a
    large one; with a fixed reservation of the whole capacity they run one at
    a time.  Results are the same either way."""
    mix = [(searches["local_edits_f2"], X) for X in range(14)]
    jobs = [make_job(e, X) for e, X in mix]
    tune = E.tuning(stack_nodes=8 << 20)
    with E.Server(ctx(), tune) as srv:
        got = srv.run_all(jobs)
        _, ep_est = srv.stats()
    with E.Server(ctx(), tune, reserve_nodes=8 << 20) as srv:
        got_fixed = srv.run_all(jobs)
        _, ep_fixed = srv.stats()
    assert ep_est < ep_fixed
    for i, (e, X) in enumerate(mix):
        assert got[i][0].counts.as_dict() == got_fixed[i][0].counts.as_dict()
        check_entry(dict(e, expect=[_expect(e, X)]), [got[i][0].counts.as_dict()])


@pytest.mark.parametrize("nshards", [2, 3])
def test_serve_shards_add_up(searches, nshards):
    """e13_serve_submit_shard: the shards of each job, run as separate jobs of
    one session, add up to the reference's counts, and their survivors together
    are the job's."""
    cases = [(searches["local_edits_f3"], 11), (searches["counter_sym"], 13), (searches["local_edits_f2"], 8)]
    with E.Server(ctx()) as srv:
        for k, (e, X) in enumerate(cases):
            job = make_job(e, X)
            for sh in range(nshards):
                srv.submit_shard(job, 100 * k + sh, sh, nshards)
        out = {}
        while srv.pending():
            for r in srv.step():
                out[r.id] = (r, srv.survivors(r.id))
    for k, (e, X) in enumerate(cases):
        job = make_job(e, X)
        tot = None
        lines = []
        for sh in range(nshards):
            r, surv = out[100 * k + sh]
            assert r.status == 0
            d = r.counts.as_dict()
            tot = d if tot is None else {f: ([a + b for a, b in zip(tot[f], v)] if f == "hist" else tot[f] + v)
                                         for f, v in d.items()}
            lines += [E.survivor_line(job, s) for s in surv]
        check_entry(dict(e, expect=[_expect(e, X)]), [tot])
        want = [l for l in golden_lines(e) if l.startswith(f"SURVIVOR X={X} ")]
        assert sorted(lines) == want
