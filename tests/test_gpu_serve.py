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
