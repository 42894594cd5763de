"""Shared helpers of the GPU parity tests: run a golden search entry through
libe13b200.so and compare with the expected counts and survivor lines."""
import gzip
import os

import e13b200 as E
import oracle_lib as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

_ctx = None


def ctx():
    global _ctx
    if _ctx is None:
        _ctx = E.Context(0)
    return _ctx


def golden_lines(entry):
    fn = os.path.join(GOLD, entry["survivors_file"])
    op = gzip.open if fn.endswith(".gz") else open
    with op(fn, "rt") as f:
        return sorted(l.rstrip("\n") for l in f if l.strip())


def make_job(entry, X):
    base = O.load_machine(entry["machine"])
    if entry["mode"] == "delete":
        r, job = E.setup(base, X, fmax=entry["fmax"])
    elif entry["mode"] == "freesym":
        r, job = E.setup(base, X, free_cells=entry["free"], lo=entry["lo"], hi=entry["hi"])
    else:
        r, job = E.setup(base, X, free_cells=entry["free"])
    assert r == 0, r
    return job


def run_entry(entry, tune=None, surv_cap=1 << 16):
    xs = entry["X"] if isinstance(entry["X"], list) else [entry["X"]]
    per_x, lines = [], []
    for X in xs:
        job = make_job(entry, X)
        c, surv = ctx().search(job, tune, surv_cap=surv_cap)
        per_x.append(c.as_dict())
        lines += [E.survivor_line(job, s) for s in surv]
    return per_x, sorted(lines)


def check_entry(entry, per_x):
    for got, exp in zip(per_x, entry["expect"]):
        assert got["leaves"] == exp["leaves"], (entry["name"], exp["X"], got, exp)
        assert got["survivors"] == exp["survivors"], (entry["name"], exp["X"])
        assert got["hist"] == exp["hist"], (entry["name"], exp["X"], got["hist"], exp["hist"])
        if exp["steps"] is not None:
            assert got["steps"] == exp["steps"], (entry["name"], exp["X"], got["steps"], exp["steps"])
