"""The hash-free device checker against the reference's recheck.c and
deep.c outputs (golden) and against the CPU oracle's restatement."""
import gzip
import json
import os

import pytest

import e13b200 as E
import oracle_lib as O
from gpu_common import GOLD, ctx

pytestmark = pytest.mark.gpu


def v1_lines():
    with gzip.open(os.path.join(GOLD, "surv", "division_v1_1RD_fileorder.txt.gz"), "rt") as f:
        return [l.rstrip("\n") for l in f if l.strip()]


def test_recheck_v1_all_2868_at_15():
    lines = v1_lines()
    exp = json.load(gzip.open(os.path.join(GOLD, "recheck_1RD.json.gz"), "rt"))["verdicts"]
    ins = [E.parse_survivor_line(l) for l in lines]
    outs = ctx().check(ins, 15, 0)
    got = [E.format_recheck(o, 15) for o in outs]
    assert len(got) == len(exp) == 2868
    bad = [(i, g, x) for i, (g, x) in enumerate(zip(got, exp)) if g != x]
    assert not bad, bad[:3]


def test_recheck_counters_match_oracle_small():
    lines = v1_lines()[:3]
    ins = [E.parse_survivor_line(l) for l in lines]
    outs = ctx().check(ins, 15, 0)
    for line, o in zip(lines, outs):
        ok, verdict, counters = O.recheck_line(line, 15)
        assert E.format_recheck(o, 15) == verdict
        for n in range(1, o.stages_done + 1):
            got = "".join(f"{o.ones_cells[n][j]}," for j in range(min(o.nones[n], 64)))
            assert got == counters[n - 1], n


def test_deep_v2_and_erdos14():
    exp = [l.rstrip("\n") for l in open(os.path.join(GOLD, "deep", "deep_v2.txt")) if l.startswith("survivor")]
    lines = open(os.path.join(GOLD, "surv", "division_v2_fileorder.txt")).read().splitlines()
    nmax = max(int(tok[1:].split(":")[0]) for l in exp for tok in l.split() if tok.startswith("n") and ":" in tok)
    ins = [E.parse_survivor_line(l) for l in lines]
    outs = ctx().check(ins, nmax, 1)
    for i, (ci, o) in enumerate(zip(ins, outs)):
        assert f"survivor {i + 1} " + E.format_deep(ci, o, nmax) == exp[i]
    base_line = ("SURVIVOR X=-1 st0=2 head0=-2 abs=1 rel=0 steps=208864 table=1L1 1R0|1L2 1L1|0R3 0R0|1L12 0R4|"
                 "1L5 1R4|0L9 1L6|1R10 0L7|1R8 1L7|0L9 0R4|0R3 1L9|0L11 1R10|1R13 0L2|0L13 ---|0R10 0L12")
    ci = E.parse_survivor_line(base_line)
    o = ctx().check([ci], 14, 1)[0]
    exp14 = open(os.path.join(GOLD, "deep", "deep_base14.txt")).read().strip()
    assert "survivor 1 " + E.format_deep(ci, o, 14) == exp14


def test_deep15_v1_sample():
    with gzip.open(os.path.join(GOLD, "deep", "deep15_1RD.txt.gz"), "rt") as f:
        exp = [l.rstrip("\n") for l in f if l.startswith("survivor")]
    lines = v1_lines()
    idx = list(range(0, 2868, 97))
    ins = [E.parse_survivor_line(lines[i]) for i in idx]
    outs = ctx().check(ins, 15, 1)
    # the golden file was made in chunks whose ids restart: compare the text after the id
    for i, ci, o in zip(idx, ins, outs):
        assert E.format_deep(ci, o, 15) == exp[i].split(" ", 2)[2]


def test_search_feeds_device_recheck(searches):
    """The pipeline of the division and counter searches: survivors of a device
    search go straight to the device recheck.  The 61 counter survivors are all
    consistent to stage 15 (recheck.c on the reference's survivors says the
    same); the lines equal the golden survivors, so the verdicts are theirs."""
    from gpu_common import make_job
    e = searches["counter_sym"]
    job = make_job(e, 13)
    c, surv = ctx().search(job)
    lines = [E.survivor_line(job, s) for s in surv]
    assert len(lines) == 61
    outs = ctx().check([E.parse_survivor_line(l) for l in lines], 15, 0)
    verdicts = [E.format_recheck(o, 15) for o in outs]
    assert all(v.startswith("CONSISTENT to n=15") for v in verdicts), verdicts[:3]


def test_device_checker_on_survivor_mutants():
    """The device checker against the oracle on 60 seeded single-cell mutants
    of real survivors (the oracle equals the reference programs on the same
    set, tests/test_oracle.py): every recheck and deep verdict kind."""
    from test_oracle import _mutants
    lines = _mutants(60, 31)
    ins = [E.parse_survivor_line(l) for l in lines]
    outs = ctx().check(ins, 11, 0)
    for line, o in zip(lines, outs):
        assert E.format_recheck(o, 11) == O.recheck_line(line, 11)[1], line
    outs = ctx().check(ins, 11, 1)
    for ci, o, line in zip(ins, outs, lines):
        assert E.format_deep(ci, o, 11) == O.deep_line(line, 11), line
