"""src/check.py on the device (e13_check_crafted, bin/e13check): the verdict
lines must equal the reference's shipped check.py outputs and, on survivors
it never checked, the oracle's restatement of check.py."""
import glob
import os
import subprocess

import pytest

import oracle_lib as O
from gpu_common import ctx, golden_lines

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def test_device_equals_shipped_check_outputs():
    files = sorted(glob.glob(os.path.join(GOLD, "check", "*.txt")))
    pairs = [p for f in files for p in O.check_golden(f)]
    assert len(pairs) == 164
    got = ctx().check_crafted([line for line, _ in pairs])
    want = []
    for line, verdicts in pairs:
        want += [line.strip()] + verdicts
    assert got == want


def test_device_equals_oracle_on_new_survivors(searches):
    """Survivors the reference never ran through check.py (the FMAX = 4
    local-edit survivors and a sample of the 2868 V1 division survivors):
    device and oracle must agree line for line."""
    lines = golden_lines(searches["local_edits_f4"]) + golden_lines(searches["division_v1_1RD"])[::48]
    want = [l for line in lines for l in O.check_line(line)]
    assert len(want) > len(lines) + 50  # placements with verdicts
    assert ctx().check_crafted(lines) == want


def test_cli_equals_shipped_output(tmp_path):
    pairs = O.check_golden(os.path.join(GOLD, "check", "division_v2.txt"))
    src = tmp_path / "in.txt"
    src.write_text("# comment lines are skipped\n" + "\n".join(line for line, _ in pairs) + "\n")
    exe = os.path.join(ROOT, "erdos-machine-13_b200", "bin", "e13check")
    p = subprocess.run([exe, str(src)], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    want = []
    for line, verdicts in pairs:
        want += [line.strip()] + verdicts
    assert p.stdout.splitlines() == want


def test_device_equals_oracle_on_survivor_mutants():
    """check.py on 60 seeded single-cell mutants of real survivors: stage walks
    that fail early, halts placed in turn into never-read cells, crafted runs
    that halt, stop or run out."""
    from test_oracle import _mutants
    lines = _mutants(60, 31)
    want = [l for line in lines for l in O.check_line(line)]
    assert ctx().check_crafted(lines) == want
