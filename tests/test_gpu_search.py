"""Parity of the CUDA search (both kernels, through the C-ABI) with the
reference: golden counts and survivor sets from the reference's result logs,
and seeded random searches against the CPU oracle."""
import random

import pytest

import e13b200 as E
import oracle_lib as O
from gpu_common import check_entry, ctx, golden_lines, make_job, run_entry

pytestmark = pytest.mark.gpu

KERNELS = {"plain": E.KERNEL_PLAIN, "persistent": E.KERNEL_PERSISTENT}


@pytest.mark.parametrize("kernel", list(KERNELS))
@pytest.mark.parametrize("name", ["local_edits_f2", "doubling_X0", "doubling_X2", "split_test", "split_test_free",
                                  "counters_f2_base_01", "counters_f2_base_44"])
def test_small_golden(searches, name, kernel):
    e = searches[name]
    per_x, lines = run_entry(e, E.tuning(kernel=KERNELS[kernel]))
    check_entry(e, per_x)
    if "survivors_file" in e:
        assert lines == golden_lines(e)


@pytest.mark.parametrize("kernel", list(KERNELS))
def test_local_edits_f3(searches, kernel):
    e = searches["local_edits_f3"]
    per_x, lines = run_entry(e, E.tuning(kernel=KERNELS[kernel]))
    check_entry(e, per_x)
    assert lines == golden_lines(e)


@pytest.mark.parametrize("kernel", list(KERNELS))
def test_division_v4(searches, kernel):
    e = searches["division_v4"]
    per_x, lines = run_entry(e, E.tuning(kernel=KERNELS[kernel]))
    check_entry(e, per_x)
    assert lines == []


def test_counter_sym(searches):
    e = searches["counter_sym"]
    per_x, lines = run_entry(e, E.tuning(kernel=E.KERNEL_PERSISTENT))
    check_entry(e, per_x)
    assert lines == golden_lines(e)


def test_local_edits_f4(searches):
    """configs[1] at FMAX = 4: 5,986,617,022 leaves, 57 survivors."""
    e = searches["local_edits_f4"]
    per_x, lines = run_entry(e, E.tuning(kernel=E.KERNEL_PERSISTENT))
    check_entry(e, per_x)
    assert lines == golden_lines(e)


def _random_cases(n, seed):
    rng = random.Random(seed)
    base = O.load_machine("erdos_14.txt")
    cells = [f"{chr(65 + q)}{a}" for q in range(14) for a in (0, 1)]
    out = []
    while len(out) < n:
        X = rng.randrange(14)
        if rng.random() < 0.5:
            free = rng.sample([c for c in cells if ord(c[0]) - 65 != X], rng.randint(2, 4))
            r, job = O.setup(base, X, free_cells=free)
            if r >= 0:
                out.append(("free", X, free, None))
        else:
            fmax = rng.randint(1, 2)
            r, job = O.setup(base, X, fmax=fmax)
            if r >= 0:
                out.append(("delete", X, None, fmax))
    return out


@pytest.mark.parametrize("case", _random_cases(8, 13))
def test_random_searches_vs_oracle(case):
    mode, X, free, fmax = case
    base = O.load_machine("erdos_14.txt")
    if mode == "free":
        r, jo = O.setup(base, X, free_cells=free)
        _, job = E.setup(base, X, free_cells=free)
    else:
        r, jo = O.setup(base, X, fmax=fmax)
        _, job = E.setup(base, X, fmax=fmax)
    exp, recs = O.search(jo)
    exp_lines = sorted(O.survivor_line(X, rr, jo.nq) for rr in recs)
    for k in (E.KERNEL_PLAIN, E.KERNEL_PERSISTENT):
        c, surv = ctx().search(job, E.tuning(kernel=k))
        assert c.as_dict() == exp
        assert sorted(E.survivor_line(job, s) for s in surv) == exp_lines


def test_symmetric_vs_oracle():
    base = O.load_machine("erdos_14.txt")
    free = ["H0", "H1", "I0", "I1"]
    r, jo = O.setup(base, 9, free_cells=free, lo=3, hi=9)
    _, job = E.setup(base, 9, free_cells=free, lo=3, hi=9)
    exp, recs = O.search(jo)
    for k in (E.KERNEL_PLAIN, E.KERNEL_PERSISTENT):
        c, surv = ctx().search(job, E.tuning(kernel=k))
        assert c.as_dict() == exp


@pytest.mark.parametrize("tune", [dict(slice=1), dict(slice=7, warp_stack=1), dict(block=256, slice=64),
                                  dict(warp_stack=3, pool_low_pct=1, epoch_us=200), dict(warp_stack=2, pool_low_pct=100, epoch_us=50),
                                  dict(kernel=E.KERNEL_PLAIN, step_cap=50, batch=3)])
def test_tunings_do_not_change_results(searches, tune):
    e = searches["local_edits_f2"]
    per_x, lines = run_entry(e, E.tuning(**tune))
    check_entry(e, per_x)
    assert lines == golden_lines(e)


def test_base_and_mutants():
    import os
    gold = os.path.join(os.path.dirname(__file__), "golden")
    base = O.load_machine("erdos_14.txt")
    tabs, keys = [], []
    for i in range(28):
        for v in range(-1, 56):
            if v == base[i]:
                continue
            t = list(base)
            t[i] = v
            tabs.append(t)
            keys.append((i, v))
    out = ctx().run_full([base] + tabs, 14)
    r = out[0]
    assert r == [1, 9, 2, -2, 1, 0, 208864]
    got = [f"{i} {v} {o[1]} {o[0]}" for (i, v), o in zip(keys, out[1:])]
    exp = [l.rstrip("\n") for l in open(os.path.join(gold, "mutants.txt")) if l.strip() and not l.startswith("#")]
    assert got == exp


def test_survivor_cap_reports_overflow(searches):
    e = searches["split_test"]
    job = __import__("gpu_common").make_job(e, 14)
    c, surv = ctx().search(job, None, surv_cap=1)
    assert c.survivors == 3 and len(surv) == 1


@pytest.mark.parametrize("name", ["local_edits_f2", "split_test_free", "counters_f2_base_07"])
@pytest.mark.parametrize("kernel", [E.KERNEL_PERSISTENT, E.KERNEL_PLAIN])
def test_run_skip_is_exact(searches, name, kernel):
    """Advancing whole words across a self-loop run (always, or only in the
    slices of warps with an old machine) gives the same counts, steps and
    survivors as single steps."""
    e = searches[name]
    a = run_entry(e, E.tuning(kernel=kernel, run_skip=0))
    for rs in (1, 100, 4096):
        b = run_entry(e, E.tuning(kernel=kernel, run_skip=rs))
        assert a == b, rs
    check_entry(e, a[0])


def test_raw_simulator_vs_oracle():
    """Raw-simulator set (no filter, <= 2^18 steps, stop off the window): the
    device, drawing its own tables from seed 0, equals the oracle on the first
    3000 machines, and on tables passed in from the host."""
    n = 3000
    codes = O.raw_tables(0, n)
    exp = O.raw_run(codes, n)
    got, tot = ctx().raw_run(n, seed=0)
    assert got == exp and tot == sum(r[0] for r in exp)
    got2, _ = ctx().raw_run(n, codes=codes)
    assert got2 == exp


def test_raw_simulator_full_set_vs_reference_run_loop():
    """The whole raw set on the device (1e6 random 13-state machines from seed
    0, <= 2^18 steps each): its per-machine results aggregate exactly to
    tests/golden/raw_1e6.json, which make_raw_golden.py made by running the
    same tables through the reference's own run() (src/e13search.c:134-177)
    with the filter switched off -- total steps, machines by status, final
    heads by status, and an order-dependent checksum of every machine's row."""
    import json
    import os
    import sys

    import numpy as np
    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    sys.path.insert(0, gold)
    import make_raw_golden as G
    g = json.load(open(os.path.join(gold, "raw_1e6.json")))
    out, tot = ctx().raw_run(g["machines"], nq=g["nq"], max_steps=g["max_steps"], seed=g["seed"], as_array=True)
    rows = np.ctypeslib.as_array(out).reshape(-1, 4)
    agg = G.aggregates(rows)
    assert tot == g["total_steps"]
    for k in ("machines", "total_steps", "by_status", "head_hist_by_status", "sum_head", "sum_ones", "checksum"):
        assert agg[k] == g[k], k


def test_run_full_matches_oracle_random_tables():
    """Whole-table runs (with the filter) of random 13-state tables against
    the oracle."""
    codes = O.raw_tables(7, 2000)
    tabs = [list(codes[26 * i: 26 * i + 26]) for i in range(2000)]
    got = ctx().run_full(tabs, 13)
    for t, g in zip(tabs, got):
        assert g == O.run_full(t, 13)


def test_autotune_keeps_results(searches):
    """The autotuner times candidate launch shapes on shard 0 of 4 of a job;
    every candidate must reproduce the same counts, and the tuning it returns
    gives the golden totals on the whole job, on both the search and a serve
    session."""
    e = searches["local_edits_f3"]
    job = __import__("gpu_common").make_job(e, 12)
    best, ms = ctx().autotune(job, proxy_shards=4)
    assert ms > 0 and best.block in (512, 640, 768) and best.slice in (8, 12, 16, 24, 32)
    assert best.warp_stack in (64, 128, 256, 512) and best.pool_low_pct in (2, 5, 12, 25)
    assert best.run_skip in (1, 1024, 4096, 8192, 32768)
    c, _ = ctx().search(job, best)
    exp = e["expect"][12]
    assert c.leaves == exp["leaves"] and list(c.hist) == exp["hist"] and c.steps == exp["steps"]
    with E.Server(ctx(), best) as srv:
        got = srv.run_all([job])
    assert got[0][0].counts.leaves == exp["leaves"]


def _budget_symmetry_cases(n, seed):
    """Jobs that mix an FMAX budget with a symmetry range (the C-ABI allows it;
    the reference's estimate mode builds such jobs), plus the two symmetry
    corner cases of setup: no deleted state with LO = 0, and an empty range."""
    rng = random.Random(seed)
    base = O.load_machine("erdos_14.txt")
    out = [("free", -1, ["G0", "H0", "B0"], 0, 0, 9), ("free", 7, ["H0", "H1"], 0, 7, 7)]
    while len(out) < n:
        X = rng.randrange(14)
        lo = rng.randrange(1, 13)
        hi = rng.randrange(lo, 13)
        fmax = rng.randint(1, 2)
        r, job = O.setup(base, X, fmax=fmax, lo=lo, hi=hi)
        if r >= 0 and job.sym_lo >= 0:
            out.append(("delete", X, None, fmax, lo, hi))
    return out


@pytest.mark.parametrize("kernel", list(KERNELS))
@pytest.mark.parametrize("case", _budget_symmetry_cases(6, 99))
def test_budget_with_symmetry_vs_oracle(case, kernel):
    mode, X, free, fmax, lo, hi = case
    base = O.load_machine("erdos_14.txt")
    if mode == "free":
        r, jo = O.setup(base, X, free_cells=free, lo=lo, hi=hi)
        rd, job = E.setup(base, X, free_cells=free, lo=lo, hi=hi)
    else:
        r, jo = O.setup(base, X, fmax=fmax, lo=lo, hi=hi)
        rd, job = E.setup(base, X, fmax=fmax, lo=lo, hi=hi)
    assert r >= 0 and rd == 0
    exp, recs = O.search(jo)
    c, surv = ctx().search(job, E.tuning(kernel=KERNELS[kernel]))
    assert c.as_dict() == exp
    assert sorted(E.survivor_line(job, s) for s in surv) == sorted(O.survivor_line(X, rr, jo.nq) for rr in recs)


@pytest.mark.parametrize("kernel", list(KERNELS))
@pytest.mark.parametrize("name,X,nshards", [("counter_sym", 13, 4), ("local_edits_f3", 11, 3), ("local_edits_f2", 8, 5)])
def test_shards_add_up_to_the_search(searches, name, X, nshards, kernel):
    """e13_search_shard: the shards' counts add up to the golden totals and
    their survivors together are the golden survivor lines."""
    entry = searches[name]
    job = make_job(entry, X)
    tune = E.tuning(kernel=KERNELS[kernel])
    tot = None
    lines = []
    for s in range(nshards):
        c, surv = ctx().search_shard(job, s, nshards, tune)
        d = c.as_dict()
        tot = d if tot is None else {k: ([a + b for a, b in zip(tot[k], v)] if k == "hist" else tot[k] + v)
                                     for k, v in d.items()}
        lines += [E.survivor_line(job, sv) for sv in surv]
    exp = next(e for e in entry["expect"] if e["X"] == X)
    assert tot["leaves"] == exp["leaves"] and tot["survivors"] == exp["survivors"] and tot["hist"] == exp["hist"]
    if exp["steps"] is not None:
        assert tot["steps"] == exp["steps"]
    want = [l for l in golden_lines(entry) if l.startswith(f"SURVIVOR X={X} ")]
    assert sorted(lines) == want


def test_e13gpu_script_prints_the_reference_driver_text(searches):
    """erdos-machine-13_b200/e13gpu.py, the drop-in for src/e13gpu.py, on the
    V4 division search: its summary line is the reference driver's
    (src/e13gpu.py:454-457) with the golden counts."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    entry = searches["division_v4"]
    exp = entry["expect"][0]
    args = [os.path.join(root, "tests", "golden", "machines", entry["machine"]), str(exp["X"]), str(entry["lo"]),
            str(entry["hi"])] + entry["free"]
    p = subprocess.run([sys.executable, os.path.join(root, "erdos-machine-13_b200", "e13gpu.py")] + args,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    summary = [l for l in p.stderr.splitlines() if " gpu leaves=" in l]
    assert len(summary) == 1
    head = f"X={exp['X']} budget=0 gpu leaves={exp['leaves']} survivors={exp['survivors']} steps={exp['steps']} wall="
    tail = " dead-at-stage(0..9): " + " ".join(str(h) for h in exp["hist"])
    assert summary[0].startswith(head) and summary[0].endswith(tail)
    want = golden_lines(entry) if entry.get("survivors_file") else []
    assert sorted(l for l in p.stdout.splitlines() if l.strip()) == want
