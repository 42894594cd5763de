"""Checkpoint / resume of one search: e13_search_resumable and the CLI's
E13_CKPT (the reference's src/e13gpu.py:349-409, 462-465).  A search stopped
and resumed any number of times must give the whole run's exact counts and
survivor lines."""
import os
import shutil
import subprocess
import threading
import time

import pytest

import e13b200 as E
from gpu_common import check_entry, ctx, golden_lines, make_job

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FILES = ("", ".a.bin", ".a.meta", ".b.bin", ".b.meta", ".tmp")
CLI_CONFIG = "freesym erdos_14.txt 13 10 13 D0 G0 K0 K1 L1 M1"


def short_epochs():
    return E.tuning(epoch_us=50000, epochs_per_graph=1)


def run_to_end(job, path, config, stop_after_s, max_calls=200):
    """Calls e13_search_resumable until the search finishes; returns the final
    result and the number of calls."""
    for calls in range(1, max_calls + 1):
        r, counts, surv, wall, left = ctx().search_resumable(job, path, config, stop_after_s=stop_after_s,
                                                             tune=short_epochs())
        if r != E.STOPPED:
            return r, counts, surv, wall, calls
        assert left > 0 and os.path.exists(path)
    raise AssertionError("search did not finish")


def test_stop_and_resume_equals_whole_run(searches, tmp_path):
    entry = searches["counter_sym"]
    job = make_job(entry, 13)
    path = str(tmp_path / "ck")
    r, counts, surv, wall, calls = run_to_end(job, path, CLI_CONFIG, stop_after_s=0.3)
    assert r == 0 and calls >= 3
    check_entry(entry, [counts.as_dict()])
    assert sorted(E.survivor_line(job, s) for s in surv) == golden_lines(entry)
    assert wall > 0
    # a finished search leaves no checkpoint behind
    assert not any(os.path.exists(path + f) for f in FILES)


def test_checkpoint_of_another_run_is_refused(searches, tmp_path):
    entry = searches["counter_sym"]
    job = make_job(entry, 13)
    path = str(tmp_path / "ck")
    r, *_ = ctx().search_resumable(job, path, CLI_CONFIG, stop_after_s=0.2, tune=short_epochs())
    assert r == E.STOPPED
    with pytest.raises(E.E13Error) as ei:
        ctx().search_resumable(job, path, "another run", tune=short_epochs())
    assert ei.value.code == -13
    other = make_job(searches["local_edits_f3"], 11)
    with pytest.raises(E.E13Error) as ei:
        ctx().search_resumable(other, path, CLI_CONFIG, tune=short_epochs())
    assert ei.value.code == -13
    # the checkpoint itself is untouched by the refusals
    r, counts, surv, wall, calls = run_to_end(job, path, CLI_CONFIG, stop_after_s=0.0)
    assert r == 0
    check_entry(entry, [counts.as_dict()])


def test_crash_during_save_keeps_the_last_checkpoint(searches, tmp_path):
    """The slot the pointer file does not name may hold a half-written save:
    resuming ignores it.  A damaged named slot is an error, not a guess."""
    entry = searches["counter_sym"]
    job = make_job(entry, 13)
    path = str(tmp_path / "ck")
    r, *_ = ctx().search_resumable(job, path, CLI_CONFIG, stop_after_s=0.2, tune=short_epochs())
    assert r == E.STOPPED
    named = open(path).read().strip()
    other = "b" if named == "a" else "a"
    with open(f"{path}.{other}.bin", "wb") as f:
        f.write(b"\x5a" * 1000)
    with open(f"{path}.{other}.meta", "wb") as f:
        f.write(b"E13CKPT1 torn")
    keep = str(tmp_path / "copy")
    for f in FILES:
        if os.path.exists(path + f):
            shutil.copy(path + f, keep + f)
    r, counts, surv, wall, calls = run_to_end(job, path, CLI_CONFIG, stop_after_s=0.0)
    assert r == 0
    check_entry(entry, [counts.as_dict()])
    assert sorted(E.survivor_line(job, s) for s in surv) == golden_lines(entry)
    # the same checkpoint with its named slot truncated
    with open(f"{keep}.{named}.bin", "r+b") as f:
        f.truncate(os.path.getsize(f"{keep}.{named}.bin") - 320)
    with pytest.raises(E.E13Error) as ei:
        ctx().search_resumable(job, keep, CLI_CONFIG, tune=short_epochs())
    assert ei.value.code == -13


def test_stop_file_stops_cleanly(searches, tmp_path):
    """Creating <path>.stop during a run stops it with a checkpoint; the stop
    file is consumed."""
    entry = searches["counter_nosym"]
    job = make_job(entry, 13)
    path = str(tmp_path / "ck")
    # buffers allocated before the timed part, so the call below starts at once
    ctx().search(make_job(searches["local_edits_f2"], 3))
    open(path + ".stop", "w").close()  # left over: removed at the start, not obeyed
    out = {}

    def run():
        out["r"] = ctx().search_resumable(job, path, "free erdos_14.txt 13 D0 G0 K0 K1 L1 M1", tune=short_epochs())

    th = threading.Thread(target=run)
    th.start()
    time.sleep(1.5)
    assert th.is_alive()
    open(path + ".stop", "w").close()
    th.join(timeout=120)
    r, counts, surv, wall, left = out["r"]
    assert r == E.STOPPED and left > 0
    assert 0 < counts.leaves < entry["expect"][0]["leaves"]
    assert os.path.exists(path) and not os.path.exists(path + ".stop")


def test_cli_resumes_a_checkpoint(searches, tmp_path):
    """bin/e13search freesym with E13_CKPT finishes a run the C-ABI stopped,
    with the reference's survivor lines and summary counts."""
    entry = searches["counter_sym"]
    job = make_job(entry, 13)
    path = str(tmp_path / "ck")
    r, *_ = ctx().search_resumable(job, path, CLI_CONFIG, stop_after_s=0.3, tune=short_epochs())
    assert r == E.STOPPED
    exe = os.path.join(ROOT, "erdos-machine-13_b200", "bin", "e13search")
    machine = os.path.join(ROOT, "tests", "golden", "machines", "erdos_14.txt")
    env = dict(os.environ, E13_CKPT=path)
    p = subprocess.run([exe, "freesym", machine, "13", "10", "13", "D0", "G0", "K0", "K1", "L1", "M1"],
                       capture_output=True, text=True, env=env, timeout=300)
    assert p.returncode == 0, p.stderr
    assert "resuming from" in p.stderr
    assert sorted(l for l in p.stdout.splitlines() if l.strip()) == golden_lines(entry)
    exp = entry["expect"][0]
    assert f"leaves={exp['leaves']} survivors={exp['survivors']} steps={exp['steps']}" in p.stderr
    assert not os.path.exists(path)
