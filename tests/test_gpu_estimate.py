"""The device estimator (e13_estimate, bin/e13search estimate) against the
oracle's restatement of the reference's probe(): every probe's weighted
leaves, nodes, steps and survivors must be equal, bit for bit."""
import json
import os
import subprocess

import pytest

import e13b200 as E
import oracle_lib as O
from gpu_common import ctx

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
CASES = json.load(open(os.path.join(GOLD, "estimate_ref.json")))


def case_job(case):
    args = case["args"]
    X, fmax, lo, hi = int(args[3]), int(args[4]), int(args[5]), int(args[6])
    cells = args[7:] or None
    base = O.load_machine(args[1])
    r, job = E.setup(base, X, fmax=fmax, free_cells=cells, lo=lo if lo >= 0 else -1, hi=hi)
    ro, ojob = O.setup(base, X, fmax=fmax, free_cells=cells, lo=lo if lo >= 0 else -1, hi=hi)
    assert r == 0 and ro >= 0
    return job, ojob, int(args[2])


@pytest.mark.parametrize("i", range(len(CASES)))
def test_device_probes_equal_oracle(i):
    case = CASES[i]
    job, ojob, probes = case_job(case)
    probes = min(probes, 1500)
    out, rows = ctx().estimate(job, probes, seed=case["seed"], per_probe=True)
    want = O.estimate_per_probe(ojob, probes, seed=case["seed"])
    bad = [p for p in range(probes) if rows[p] != want[p]]
    assert not bad, (case["args"], bad[:5], rows[bad[0]], want[bad[0]])
    assert out.probes == probes
    lines = ["  %-9s %.3e  (+- %.1e standard error)" % (n, out.mean[j], out.std_error[j])
             for j, n in enumerate(("leaves", "nodes", "steps", "survivors"))]
    assert lines == O.lines_from_rows(want)


def test_cli_estimate_prints_the_reference_format():
    case = CASES[2]  # freesym counter search
    job, ojob, probes = case_job(case)
    exe = os.path.join(ROOT, "erdos-machine-13_b200", "bin", "e13search")
    args = list(case["args"])
    args[1] = os.path.join(GOLD, "machines", args[1])
    p = subprocess.run([exe] + args, capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, E13_SEED=str(case["seed"])))
    assert p.returncode == 0, p.stderr
    out = p.stdout.splitlines()
    assert out[0].startswith(case["header"] + " wall=")
    assert out[1:5] == O.lines_from_rows(O.estimate_per_probe(ojob, probes, seed=case["seed"]))


ORDER_SCRIPT = r"""
import sys
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[2])
import e13b200 as E, oracle_lib as O
base = O.load_machine("erdos_14.txt")
ctx = E.Context(0)
r, job = E.setup(base, 8, fmax=2)
ro, ojob = O.setup(base, 8, fmax=2)
def search():
    c, _ = ctx.search(job)
    assert (c.leaves, c.survivors, c.steps) == (19962, 1, 9400699), (c.leaves, c.survivors, c.steps)
def estimate():
    out, rows = ctx.estimate(job, 200, seed=1, per_probe=True)
    assert rows == O.estimate_per_probe(ojob, 200, seed=1)
for name in sys.argv[3:]:
    {"search": search, "estimate": estimate}[name]()
print("ok")
"""


@pytest.mark.parametrize("order", [("search", "estimate", "search"), ("estimate", "search", "estimate")])
def test_each_kernel_file_has_its_filter_tables(order, tmp_path):
    """A fresh process, kernels in either order: each .cu file uploads its
    own copy of the filter's constant tables."""
    script = tmp_path / "order.py"
    script.write_text(ORDER_SCRIPT)
    p = subprocess.run(["python", str(script), os.path.join(ROOT, "erdos-machine-13_b200"),
                        os.path.join(ROOT, "tests")] + list(order), capture_output=True, text=True, timeout=300)
    assert p.returncode == 0 and p.stdout.strip() == "ok", p.stdout + p.stderr


def test_device_probes_equal_oracle_on_random_jobs():
    """Device probes against the oracle on 6 seeded random jobs (delete with
    FMAX, free, freesym), every probe's four doubles."""
    import random
    rng = random.Random(404)
    base = O.load_machine("erdos_14.txt")
    done = 0
    while done < 6:
        X = rng.randrange(14)
        fmax = rng.randrange(0, 4)
        cells, lo, hi = [], -1, -1
        if rng.random() < 0.5:
            cells = sorted({f"{chr(65 + rng.randrange(14))}{rng.randrange(2)}" for _ in range(rng.randrange(2, 6))})
            if rng.random() < 0.5:
                lo = rng.randrange(1, 13)
                hi = rng.randrange(lo, 13)
        ro, ojob = O.setup(base, X, fmax=fmax, free_cells=cells or None, lo=lo, hi=hi)
        if ro < 0:
            continue
        r, job = E.setup(base, X, fmax=fmax, free_cells=cells or None, lo=lo, hi=hi)
        assert r == 0
        seed = rng.randrange(1000)
        out, rows = ctx().estimate(job, 400, seed=seed, per_probe=True)
        assert rows == O.estimate_per_probe(ojob, 400, seed=seed)
        done += 1
