"""libe13b200.so without a GPU: it loads, exports every entry point that
include/e13.h declares, and its host-side helpers (keys, machine files,
candidate setup, text formats) agree with the oracle and the reference's
formats.  No compute call is made here."""
import os
import re

import pytest

import e13b200 as E
import oracle_lib as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "e13.h")).read()
    return sorted(set(re.findall(r"\b(e13_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = E.lib()
    for name in declared_symbols():
        assert hasattr(L, name), name
    assert set(declared_symbols()) >= set(E.EXPORTED)


def test_keys_equal_oracle():
    assert E.keys() == O.keys()


def test_machine_parsing():
    path = os.path.join(O.MACHINES, "erdos_14.txt")
    assert E.load_machine(path) == O.load_machine("erdos_14.txt")
    assert E.parse_machine(open(path).read()) == O.load_machine("erdos_14.txt")
    with pytest.raises(E.E13Error):
        E.load_machine("/nonexistent/machine.txt")


@pytest.mark.parametrize("machine", ["erdos_14.txt", "split_15.txt", "counters_3state/base_07.txt"])
def test_setup_delete_matches_oracle(machine):
    base = O.load_machine(machine)
    nq0 = len(base) // 2
    for X in range(-1, nq0):
        for fmax in (0, 1, 2, 4):
            r, job = E.setup(base, X, fmax=fmax)
            ro, jo = O.setup(base, X, fmax=fmax)
            if ro == -1:
                assert r == -2
                continue
            assert r == 0 and job.budget == ro
            assert list(job.tab)[: 2 * job.nq] == jo.tab
            assert job.nforced == jo.nforced


@pytest.mark.parametrize("X,lo,hi,free", [
    (13, 10, 13, ["D0", "G0", "K0", "K1", "L1", "M1"]),
    (9, 3, 9, ["F0", "F1", "G0", "G1", "H0", "H1", "I0", "I1"]),
    (9, 3, 9, ["F0", "F1"]),
    (13, 0, 13, ["A0", "A1"]),
    (2, -1, -1, ["A0", "A1", "B0", "B1"]),
])
def test_setup_free_matches_oracle(X, lo, hi, free):
    base = O.load_machine("erdos_14.txt")
    r, job = E.setup(base, X, free_cells=free, lo=lo, hi=hi)
    ro, jo = O.setup(base, X, free_cells=free, lo=lo, hi=hi)
    assert r == (0 if ro >= 0 else ro)
    if r == 0:
        assert list(job.tab)[: 2 * job.nq] == jo.tab
        assert (job.sym_lo, job.sym_hi, job.sym_n0) == (jo.sym_lo, jo.sym_hi, jo.sym_n0)


def test_format_survivor_matches_reference_text():
    line = open(os.path.join(os.path.dirname(__file__), "golden", "surv", "f2.txt")).read().strip()
    ci = E.parse_survivor_line(line)
    assert ci is not None and ci.nq == 13
    # rebuild the survivor record from the line and format it back
    base = O.load_machine("erdos_14.txt")
    _, job = E.setup(base, 8, fmax=2)
    s = E.Survivor()
    for i in range(26):
        s.tab[i] = -1 if ci.kind[i] else (ci.next[i] << 2) | ((ci.move[i] > 0) << 1) | ci.write[i]
    s.read_mask = (1 << 26) - 1
    s.st0, s.head0, s.abs_ok, s.rel_ok, s.steps = 2, -2, 1, 0, 208838
    assert E.survivor_line(job, s) == line


def test_survivor_check_in_equals_parsed_line():
    """e13_survivor_check_in gives the checker input that parsing the
    survivor's printed line gives, on 300 random survivor records (moves,
    halts, free cells, read masks, both head rules)."""
    import random

    rng = random.Random(5)
    base = O.load_machine("erdos_14.txt")
    _, job = E.setup(base, 9, free_cells=["F0", "F1", "G0", "G1", "H0", "H1", "I0", "I1"], lo=3, hi=9)
    fields = ("nq", "st0", "rel", "head0")
    for _ in range(300):
        s = E.Survivor()
        for i in range(2 * job.nq):
            r = rng.random()
            s.tab[i] = E.E13_FREE if r < 0.1 else (-1 if r < 0.2 else rng.randrange(4 * job.nq))
        s.read_mask = rng.getrandbits(26)
        s.st0, s.head0 = rng.randrange(job.nq), rng.randrange(-40, 3)
        s.abs_ok, s.rel_ok = rng.randrange(2), rng.randrange(2)
        s.steps = rng.randrange(1, 1 << 20)
        a = E.survivor_check_in(job, s)
        b = E.parse_survivor_line(E.survivor_line(job, s))
        assert [getattr(a, f) for f in fields] == [getattr(b, f) for f in fields]
        for arr in ("kind", "write", "move", "next"):
            assert list(getattr(a, arr)) == list(getattr(b, arr)), arr


def test_summary_format():
    base = O.load_machine("erdos_14.txt")
    _, job = E.setup(base, 9, free_cells=["F0", "F1", "G0", "G1", "H0", "H1", "I0", "I1"], lo=3, hi=9)
    c = E.Counts(830955779, 0, 96702705048, (E.ctypes.c_uint64 * 10)(0, 755283390, 74755943, 852182, 20270, 420,
                                                                         36, 0, 43538, 0))
    line = E.summary_line(job, c, 1.0)
    assert O.parse_summary(line) == dict(X=9, leaves=830955779, survivors=0, steps=96702705048,
                                         hist=[0, 755283390, 74755943, 852182, 20270, 420, 36, 0, 43538, 0])


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(E.E13Error) as ei:
        E.Context(0)
    assert ei.value.code in (-11, -5)


def test_resumable_search_checks_its_arguments():
    """e13_search_resumable rejects a missing context or checkpoint before
    touching a device or a file."""
    import ctypes
    base = O.load_machine("erdos_14.txt")
    r, job = E.setup(base, 13, free_cells=["D0", "G0", "K0", "K1", "L1", "M1"], lo=10, hi=13)
    counts, ns = E.Counts(), ctypes.c_int()
    ck = E.Checkpoint(b"/nonexistent/ckpt", b"cfg", 0.0, 0.0)
    L = E.lib()
    assert L.e13_search_resumable(None, ctypes.byref(job), None, ctypes.byref(ck), ctypes.byref(counts), None, 0,
                                  ctypes.byref(ns), None, None) == -1
    assert L.e13_search_resumable(None, ctypes.byref(job), None, None, ctypes.byref(counts), None, 0,
                                  ctypes.byref(ns), None, None) == -1


def test_setup_random_free_sets_match_oracle():
    """Candidate setup over 400 seeded random cases (machine, deleted state,
    free set, symmetry range): the library's status, table and symmetry
    fields equal the oracle's restatement of setup()/set_sym()."""
    import random
    rng = random.Random(13)
    machines = ["erdos_14.txt", "split_15.txt", "c0_1RD.txt", "counters_3state/base_07.txt",
                "counters_3state/base_33.txt"]
    checked = 0
    for _ in range(400):
        base = O.load_machine(rng.choice(machines))
        nq0 = len(base) // 2
        X = rng.randrange(-1, nq0)
        nq = nq0 - (1 if X >= 0 else 0)
        cells = rng.sample(range(2 * nq0), rng.randrange(1, 7))
        free = [chr(ord("A") + c // 2) + str(c % 2) for c in cells]
        if rng.random() < 0.5:
            lo = rng.randrange(0, nq)
            hi = rng.randrange(lo, nq)
        else:
            lo = hi = -1
        r, job = E.setup(base, X, free_cells=free, lo=lo, hi=hi)
        ro, jo = O.setup(base, X, free_cells=free, lo=lo, hi=hi)
        assert r == (0 if ro >= 0 else ro), (X, free, lo, hi, r, ro)
        if r == 0:
            assert list(job.tab)[: 2 * job.nq] == jo.tab
            assert (job.sym_lo, job.sym_hi, job.sym_n0) == (jo.sym_lo, jo.sym_hi, jo.sym_n0)
            checked += 1
    assert checked > 50


def test_survivor_lines_random_match_oracle():
    """e13_format_survivor against the oracle's restatement of report()
    (src/e13search.c:184-200) on 500 seeded random records: any moves, halts,
    free cells, read masks, heads and step counts."""
    import random
    rng = random.Random(7)
    base = O.load_machine("erdos_14.txt")
    for _ in range(500):
        nq = rng.randrange(1, 16)
        r, job = E.setup(base, rng.randrange(-1, 14), fmax=4)
        job.nq = nq
        tab = [rng.choice([E.E13_HALT, E.E13_FREE] + list(range(4 * nq))) for _ in range(2 * nq)]
        s = E.Survivor()
        for i, c in enumerate(tab):
            s.tab[i] = c
        s.read_mask = rng.getrandbits(2 * nq)
        s.st0, s.head0 = rng.randrange(0, nq), rng.randrange(-60, 1200)
        s.abs_ok, s.rel_ok = rng.randrange(2), rng.randrange(2)
        s.steps = rng.randrange(0, 835521)
        rec = dict(tab=tab, mask=s.read_mask, st0=s.st0, head0=s.head0, abs=s.abs_ok, rel=s.rel_ok, steps=s.steps)
        assert E.survivor_line(job, s) == O.survivor_line(job.X, rec, nq)


def test_machine_text_random_matches_oracle():
    """e13_parse_machine against load()/parse_cell() (src/e13search.c:105-121)
    on 300 seeded random machine texts with halts, odd spacing and blank lines."""
    import random
    rng = random.Random(11)
    for _ in range(300):
        nq = rng.randrange(1, 17)
        lines = []
        for q in range(nq):
            cells = []
            for a in range(2):
                if rng.random() < 0.1:
                    cells.append("---")
                else:
                    cells.append(f"{rng.randrange(2)}{rng.choice('LR')}{rng.randrange(16)}")
            lines.append((" " * rng.randrange(3)).join(["", ""]) + cells[0] + " " * rng.randrange(1, 4) + cells[1])
            if rng.random() < 0.1:
                lines.append("")
        text = "\n".join(lines) + "\n"
        assert E.parse_machine(text) == O.parse_machine_text(text)


def test_setup_random_delete_with_symmetry_matches_oracle():
    """Delete mode with a symmetry range (the reference's estimate mode allows
    it, src/e13search.c:478-480): 300 seeded random cases, status, table,
    budget and symmetry fields against the oracle."""
    import random
    rng = random.Random(5)
    machines = ["erdos_14.txt", "split_15.txt", "counters_3state/base_21.txt"]
    for _ in range(300):
        base = O.load_machine(rng.choice(machines))
        nq0 = len(base) // 2
        X = rng.randrange(-1, nq0)
        nq = nq0 - (1 if X >= 0 else 0)
        lo = rng.randrange(-1, nq)
        hi = rng.randrange(max(lo, 0), nq)
        fmax = rng.randrange(0, 5)
        r, job = E.setup(base, X, fmax=fmax, lo=lo, hi=hi)
        ro, jo = O.setup(base, X, fmax=fmax, lo=lo, hi=hi)
        assert r == (0 if ro >= 0 else (-2 if ro == -1 else ro)), (X, lo, hi, fmax, r, ro)
        if r == 0:
            assert job.budget == ro
            assert list(job.tab)[: 2 * job.nq] == jo.tab
            assert (job.sym_lo, job.sym_hi, job.sym_n0) == (jo.sym_lo, jo.sym_hi, jo.sym_n0)


def test_search_shard_checks_its_arguments():
    import ctypes
    base = O.load_machine("erdos_14.txt")
    r, job = E.setup(base, 11, fmax=2)
    counts, ns = E.Counts(), ctypes.c_int()
    L = E.lib()
    for shard, n in ((0, 0), (2, 2), (-1, 3)):
        assert L.e13_search_shard(None, ctypes.byref(job), None, shard, n, ctypes.byref(counts), None, 0,
                                  ctypes.byref(ns)) == -1


def _e13gpu(args):
    import subprocess
    import sys
    return subprocess.run([sys.executable, os.path.join(ROOT, "erdos-machine-13_b200", "e13gpu.py")] + args,
                          capture_output=True, text=True, timeout=120)


def test_e13gpu_script_refuses_like_the_reference():
    """The drop-in for src/e13gpu.py exits 1 with a message on a bad command
    line, a missing machine file and the symmetry preconditions, before any
    device work (src/e13gpu.py:79-94, 294-296)."""
    machine = os.path.join(ROOT, "tests", "golden", "machines", "erdos_14.txt")
    p = _e13gpu([])
    assert p.returncode == 1 and "usage" in p.stderr
    p = _e13gpu(["/nonexistent/m.txt", "9", "-1", "-1", "F0"])
    assert p.returncode == 1 and "cannot open" in p.stderr
    p = _e13gpu([machine, "13", "10", "13", "D0"])
    assert p.returncode == 1 and "named by a fixed cell" in p.stderr
    p = _e13gpu([machine, "13", "0", "13", "A0", "A1"])
    assert p.returncode == 1 and ("start state" in p.stderr or "named by a fixed cell" in p.stderr)


def test_tuning_ranges_are_checked():
    """e13_resolve_tuning (applied by every entry point that takes a tuning):
    zero fields take the defaults, a serve session defaults to 10 ms epochs on
    the persistent kernel, and each field out of range is E13_ERR_ARG --
    including a negative epoch bound (it would make one launch run a whole
    search, so checkpoints and stop files never fire) and a negative or zero
    graph length (an empty graph would never move the frontier)."""
    r, t = E.resolve_tuning(None)
    d = E.tuning()
    assert r == 0 and (t.block, t.slice, t.warp_stack, t.epoch_us, t.epochs_per_graph, t.pool_low_pct) == \
        (d.block, d.slice, d.warp_stack, d.epoch_us, d.epochs_per_graph, d.pool_low_pct)
    r, t = E.resolve_tuning(E.tuning(kernel=E.KERNEL_PLAIN, epoch_us=0), serve=True)
    assert r == 0 and t.kernel == E.KERNEL_PERSISTENT and t.epoch_us == 10000
    r, t = E.resolve_tuning(E.tuning(slice=9, block=256))
    assert r == 0 and t.slice == 9 and t.block == 256
    # run_skip is taken as given: 0 never, 1 always, N >= 2 from a machine age of N steps
    for rs in (0, 1, 2, 4096, 1 << 30):
        r, t = E.resolve_tuning(E.tuning(run_skip=rs))
        assert r == 0 and t.run_skip == rs
    bad = [dict(epoch_us=-1), dict(epochs_per_graph=-1), dict(pool_low_pct=-5), dict(pool_low_pct=101),
           dict(block=48), dict(block=800), dict(block=100), dict(slice=-1), dict(slice=5000),
           dict(warp_stack=-2), dict(warp_stack=5000), dict(epochs_per_graph=65), dict(epoch_us=60_000_001),
           dict(step_cap=-1), dict(batch=-1), dict(stack_nodes=-1), dict(kernel=2), dict(run_skip=-1)]
    for kw in bad:
        for serve in (False, True):
            r, _ = E.resolve_tuning(E.tuning(**kw), serve=serve)
            assert r == -1, (kw, serve)
