"""The device path's error statuses, made to happen without faulting or
hanging a GPU, and the context staying usable after each:

  * a frontier capacity too small for the search: E13_ERR_OVERFLOW (both
    kernels), then the same context runs the golden search;
  * the persistent kernel's one device-side wait (a warp that claimed a
    donation-pool slot waits for the donor's data) made to run out with
    e13_selftest_pool_wait: E13_ERR_TIMEOUT after the bounded wait, then the
    same context runs the golden search and a serve session.
"""
import pytest

import e13b200 as E
from gpu_common import check_entry, ctx, golden_lines, make_job

pytestmark = pytest.mark.gpu

KERNELS = {"plain": E.KERNEL_PLAIN, "persistent": E.KERNEL_PERSISTENT}


def _golden_f2_x8(searches):
    e = searches["local_edits_f2"]
    job = make_job(e, 8)
    c, surv = ctx().search(job)
    exp = next(x for x in e["expect"] if x["X"] == 8)
    assert c.as_dict() == {k: exp[k] for k in ("leaves", "survivors", "steps", "hist")}
    want = [l for l in golden_lines(e) if l.startswith("SURVIVOR X=8 ")]
    assert sorted(E.survivor_line(job, s) for s in surv) == want


@pytest.mark.parametrize("kernel", list(KERNELS))
def test_frontier_overflow_is_reported_and_the_context_recovers(searches, kernel):
    e = searches["local_edits_f3"]
    job = make_job(e, 11)  # 1.4e7 leaves: its frontier outgrows 2,000 nodes at once
    with pytest.raises(E.E13Error) as ei:
        # 1 ms epochs: the persistent kernel dumps its lanes and warp stacks onto the frontier at once
        ctx().search(job, E.tuning(kernel=KERNELS[kernel], stack_nodes=2000, epoch_us=1000))
    assert ei.value.code == -6  # E13_ERR_OVERFLOW
    _golden_f2_x8(searches)
    c, _ = ctx().search(job, E.tuning(kernel=KERNELS[kernel]))
    check_entry({"name": "f3 X=11", "expect": [e["expect"][11]]}, [c.as_dict()])


def test_pool_wait_runs_out_and_the_context_recovers(searches):
    import time
    t0 = time.perf_counter()
    assert ctx().selftest_pool_wait(2000) == -10  # E13_ERR_TIMEOUT after a 2 ms wait
    assert time.perf_counter() - t0 < 5.0
    _golden_f2_x8(searches)
    # a serve session on the same context
    e = searches["local_edits_f2"]
    jobs = [make_job(e, X) for X in (3, 8, 11)]
    with E.Server(ctx()) as srv:
        got = srv.run_all(jobs)
    for i, X in enumerate((3, 8, 11)):
        r, _ = got[i]
        exp = next(x for x in e["expect"] if x["X"] == X)
        assert r.status == 0
        assert r.counts.leaves == exp["leaves"] and list(r.counts.hist) == exp["hist"]
