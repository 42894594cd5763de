"""The CPU oracle pinned against the reference's shipped results (golden
fixtures) and, where oracle/_ref exists, against the reference binaries.
No GPU needed."""
import gzip
import json
import os
import subprocess

import pytest

import oracle_lib as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def surv_lines(entry):
    fn = os.path.join(GOLD, entry["survivors_file"])
    op = gzip.open if fn.endswith(".gz") else open
    with op(fn, "rt") as f:
        return sorted(l.rstrip("\n") for l in f if l.strip())


def run_entry(entry, X):
    base = O.load_machine(entry["machine"])
    if entry["mode"] == "delete":
        r, job = O.setup(base, X, fmax=entry["fmax"])
    else:
        lo, hi = (entry["lo"], entry["hi"]) if entry["mode"] == "freesym" else (-1, -1)
        r, job = O.setup(base, X, free_cells=entry["free"], lo=lo, hi=hi)
    assert r >= 0
    c, recs = O.search(job, nthreads=8)
    return c, [O.survivor_line(X, rr, job.nq) for rr in recs]


def check_counts(c, exp):
    assert c["leaves"] == exp["leaves"]
    assert c["survivors"] == exp["survivors"]
    assert c["hist"] == exp["hist"]
    if exp["steps"] is not None:
        assert c["steps"] == exp["steps"]


def test_keys_match_reference_targets():
    k, t = O.keys()
    assert len(k) == 1364 and t[0] == 0
    # TGT[n] is the XOR of KEY over cells -1..2^n-2 (src/e13search.c:441-444)
    for n in range(1, 10):
        h = 0
        for c in range(-1, (1 << n) - 1):
            h ^= k[c + 64]
        assert h == t[n]


def test_base_erdos14():
    base = O.load_machine("erdos_14.txt")
    r = O.run_full(base, 14)
    # base states=14 result=SURV stage=9 st0=2 head0=-2 abs=1 rel=0 steps=208864
    line = open(os.path.join(GOLD, "base_erdos14.txt")).read().splitlines()[-1]
    assert line == (f"base states=14 result={'SURV' if r[0] else 'DEAD'} stage={r[1]} st0={r[2]} head0={r[3]} "
                    f"abs={r[4]} rel={r[5]} steps={r[6]}")


def test_mutants():
    base = O.load_machine("erdos_14.txt")
    got = []
    for i in range(28):
        for v in range(-1, 56):
            if v == base[i]:
                continue
            tab = list(base)
            tab[i] = v
            r = O.run_full(tab, 14)
            got.append(f"{i} {v} {r[1]} {r[0]}")
    exp = [l.rstrip("\n") for l in open(os.path.join(GOLD, "mutants.txt")) if l.strip() and not l.startswith("#")]
    assert got == exp


@pytest.mark.parametrize("name", ["local_edits_f2", "doubling_X0", "doubling_X1", "doubling_X2", "split_test",
                                  "split_test_free"])
def test_small_searches(searches, name):
    e = searches[name]
    xs = e["X"] if isinstance(e["X"], list) else [e["X"]]
    lines = []
    for X, exp in zip(xs, e["expect"]):
        assert exp["X"] == X
        c, l = run_entry(e, X)
        check_counts(c, exp)
        lines += l
    if "survivors_file" in e:
        assert sorted(lines) == surv_lines(e)


@pytest.mark.parametrize("k", [1, 17, 61])
def test_counters_f2(searches, k):
    e = searches[f"counters_f2_base_{k:02d}"]
    c, _ = run_entry(e, -1)
    check_counts(c, e["expect"][0])


def test_setup_errors():
    base = O.load_machine("erdos_14.txt")
    # X=2 has two forced cells: FMAX=1 skips it (src/e13search.c:353)
    r, _ = O.setup(base, 2, fmax=1)
    assert r == -1
    # a fixed cell naming a symmetric state beyond the first unnamed one
    r, _ = O.setup(base, 9, free_cells=["F0", "F1"], lo=3, hi=9)
    assert r == -3
    # start state inside the symmetric range
    r, _ = O.setup(base, 13, free_cells=["A0", "A1"], lo=0, hi=13)
    assert r in (-3, -4)


def test_recheck_golden_first_v1_survivor():
    lines = gzip.open(os.path.join(GOLD, "surv", "division_v1_1RD_fileorder.txt.gz"), "rt").read().splitlines()
    v = json.load(gzip.open(os.path.join(GOLD, "recheck_1RD.json.gz"), "rt"))["verdicts"]
    ok, verdict, _ = O.recheck_line(lines[0], 15)
    assert verdict == v[0]


def test_deep_golden():
    for fn, survfn, nmax in (("deep_v2.txt", "division_v2_fileorder.txt", 16),):
        exp = [l.rstrip("\n") for l in open(os.path.join(GOLD, "deep", fn)) if l.startswith("survivor")]
        lines = open(os.path.join(GOLD, "surv", survfn)).read().splitlines()
        # deep_v2 was run at some NMAX; take it from the longest line
        n = max(int(tok[1:].split(":")[0]) for l in exp for tok in l.split() if tok.startswith("n") and ":" in tok)
        for i, line in enumerate(lines[:2]):
            got = f"survivor {i + 1} " + O.deep_line(line, n)
            assert got == exp[i]


REFBIN = os.path.join(O.REF_DIR, "e13search")


@pytest.mark.skipif(not os.path.exists(REFBIN), reason="reference binaries not built here")
@pytest.mark.parametrize("args", [
    ["free", "erdos_14.txt", "5", "B0", "C1", "E0"],
    ["freesym", "erdos_14.txt", "9", "3", "9", "H0", "H1", "I0", "I1"],
    ["delete", "counters_3state/base_05.txt", "1", "-1"],
    ["delete", "split_15.txt", "2", "3"],
    # no deleted state: the reference shifts LO..HI down by one, so LO = 0 turns symmetry off
    ["freesym", "erdos_14.txt", "-1", "0", "9", "G0", "H0", "B0"],
    # an empty range after renumbering (7..6): accepted, no symmetry
    ["freesym", "erdos_14.txt", "7", "7", "7", "H0", "H1"],
])
def test_oracle_vs_reference_binary(args):
    mode = args[0]
    path = os.path.join(O.MACHINES, args[1])
    r = subprocess.run([REFBIN, mode, path] + args[2:], capture_output=True, text=True, check=True,
                       env=dict(os.environ, OMP_NUM_THREADS="4"))
    ref = [O.parse_summary(l) for l in r.stderr.splitlines() if "leaves=" in l]
    ref_surv = sorted(l for l in r.stdout.splitlines() if l.startswith("SURVIVOR"))
    base = O.load_machine(args[1])
    got_surv = []
    if mode == "delete":
        for X, exp in zip([int(x) for x in args[3:]], ref):
            st, job = O.setup(base, X, fmax=int(args[2]))
            c, recs = O.search(job)
            check_counts(c, exp)
            got_surv += [O.survivor_line(X, rr, job.nq) for rr in recs]
    else:
        X = int(args[2])
        if mode == "freesym":
            st, job = O.setup(base, X, free_cells=args[5:], lo=int(args[3]), hi=int(args[4]))
        else:
            st, job = O.setup(base, X, free_cells=args[3:])
        c, recs = O.search(job)
        check_counts(c, ref[0])
        got_surv = [O.survivor_line(X, rr, job.nq) for rr in recs]
    assert sorted(got_surv) == ref_surv


def test_raw_tables_are_splitmix_draws():
    """Machine m, cell i = draw m*26+i+1 of splitmix64 from seed 0, mod 52."""
    M = (1 << 64) - 1
    s = 0
    exp = []
    for _ in range(3 * 26):
        s = (s + 0x9E3779B97F4A7C15) & M
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        exp.append((z ^ (z >> 31)) % 52)
    assert list(O.raw_tables(0, 3)) == exp


def test_raw_run_small_known_cases():
    # A0 = 1RA: writes ones rightwards; leaves the window at 1299 (that step not counted)
    codes = bytes([2 | 1, 2 | 1]) + bytes([0] * 24)
    assert O.raw_run(codes, 1, nq=13)[0] == [1298, 1, 1299, 1299]
    # A0 = 0LA: walks left over blanks, leaves at -64 after 63 counted steps
    codes = bytes([0, 0]) + bytes([0] * 24)
    assert O.raw_run(codes, 1, nq=13)[0] == [63, 1, -64, 0]


REF_RAW = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "ref_raw")


@pytest.mark.skipif(not os.path.exists(REF_RAW), reason="oracle/_ref/ref_raw not built (no reference checkout)")
def test_raw_run_equals_reference_run_loop():
    """The raw-simulator restatement against the reference's own step loop:
    oracle/_ref/ref_raw runs run() of src/e13search.c with the filter switched
    off from outside.  Per machine (steps, status, final head, ones), on 20,000
    machines of the set and on 2,000 machines of an 8-state set with a short cap."""
    import numpy as np
    for seed, m0, n, nq, cap in ((0, 0, 20000, 13, 1 << 18), (5, 777, 2000, 8, 5000)):
        p = subprocess.run([REF_RAW, str(seed), str(m0), str(n), str(nq), str(cap)], capture_output=True, check=True)
        ref = np.frombuffer(p.stdout, dtype=np.int64).reshape(-1, 4)
        codes = O.raw_tables(seed, m0 + n, nq)[m0 * 2 * nq:]
        got = np.array(O.raw_run(codes, n, nq=nq, max_steps=cap), dtype=np.int64).reshape(-1, 4)
        assert (got == ref).all()


def test_raw_golden_fixture_matches_its_first_machines():
    """raw_1e6.json (made by tests/golden/make_raw_golden.py from the
    reference's run()) is consistent with the oracle: the histogram counts add
    up, and the oracle's first 2,000 machines have the checksum the generator's
    function gives them."""
    import sys
    sys.path.insert(0, GOLD)
    import make_raw_golden as G
    g = json.load(open(os.path.join(GOLD, "raw_1e6.json")))
    assert g["machines"] == 1000000 and sum(g["by_status"].values()) == 1000000
    for s, h in g["head_hist_by_status"].items():
        assert sum(h.values()) == g["by_status"][s]
    codes = O.raw_tables(0, 2000)
    out = O.raw_run(codes, 2000)
    agg = G.aggregates(out)
    assert agg["machines"] == 2000 and agg["total_steps"] == sum(r[0] for r in out)


def _estimate_job(case):
    args = case["args"]
    X, fmax, lo, hi = int(args[3]), int(args[4]), int(args[5]), int(args[6])
    cells = args[7:] or None
    base = O.load_machine(args[1])
    r, job = O.setup(base, X, fmax=fmax, free_cells=cells, lo=lo if lo >= 0 else -1, hi=hi)
    assert r >= 0
    return job, int(args[2])


def test_estimate_equals_reference_binary():
    """The restated probe() draws and adds exactly as the reference: on one
    thread's stream its printed estimate is the reference binary's, digit for
    digit (fixtures made by tests/golden/make_golden.py)."""
    import json
    cases = json.load(open(os.path.join(GOLD, "estimate_ref.json")))
    assert len(cases) >= 4
    for case in cases:
        job, probes = _estimate_job(case)
        assert case["header"].startswith(f"estimate X={job.X} budget={job.budget} probes={probes}")
        assert O.estimate_lines(job, probes, case["seed"]) == case["lines"], case["args"]


def test_estimate_probe_streams_are_independent():
    """Per-probe streams: probe p's result depends only on (seed, p)."""
    base = O.load_machine("erdos_14.txt")
    r, job = O.setup(base, 11, fmax=3)
    a = O.estimate_per_probe(job, 50, seed=5)
    b = [O.probe(job, O.probe_stream(5, p))[0] for p in reversed(range(50))][::-1]
    assert a == b
    assert O.estimate_per_probe(job, 50, seed=6) != a


def test_check_py_restatement_equals_shipped_outputs():
    """The oracle's restatement of src/check.py prints, for every survivor
    line of the reference's shipped check.py outputs, the same verdict lines
    (stages to n = 11, counters per c, crafted-start fails)."""
    import glob
    files = sorted(glob.glob(os.path.join(GOLD, "check", "*.txt")))
    assert len(files) == 6
    n = 0
    for f in files:
        for line, verdicts in O.check_golden(f):
            got = O.check_line(line)
            assert got[0] == line.strip()
            assert got[1:] == verdicts, (f, line[:80])
            n += 1
    assert n == 164


def _random_free_cases(n, seed):
    """Seeded small free / freesym searches on erdos_14 and a counter base:
    (args for the reference binary)."""
    import random
    rng = random.Random(seed)
    out = []
    while len(out) < n:
        machine = rng.choice(["erdos_14.txt", "counters_3state/base_12.txt"])
        nq0 = len(O.load_machine(machine)) // 2
        X = rng.randrange(-1, nq0)
        cells = sorted(rng.sample(range(2 * nq0), rng.randrange(2, 4)))
        names = [chr(ord("A") + c // 2) + str(c % 2) for c in cells]
        if rng.random() < 0.5:
            lo = rng.randrange(1, nq0)
            hi = rng.randrange(lo, nq0)
            base = O.load_machine(machine)
            if O.setup(base, X, free_cells=names, lo=lo, hi=hi)[0] < 0:
                continue  # the reference exits 1 on these; the setup tests cover them
            out.append(["freesym", machine, str(X), str(lo), str(hi)] + names)
        else:
            out.append(["free", machine, str(X)] + names)
    return out


@pytest.mark.skipif(not os.path.exists(REFBIN), reason="reference binaries not built here")
@pytest.mark.parametrize("args", _random_free_cases(12, 2026))
def test_oracle_vs_reference_binary_random(args):
    """The oracle against the reference program on seeded random free-cell
    searches: leaves, survivors, steps, deaths per stage, survivor lines."""
    test_oracle_vs_reference_binary(args)


def _mutants(n, seed):
    """Seeded single-cell mutants of V1 and V2 survivor lines: a cell gets a
    random move or a halt, a fixed cell may become a never-read free one."""
    import random
    rng = random.Random(seed)
    src = [l.rstrip("\n") for l in gzip.open(os.path.join(GOLD, "surv", "division_v1_1RD.txt.gz"), "rt") if "table=" in l]
    src += [l.rstrip("\n") for l in open(os.path.join(GOLD, "surv", "division_v2_fileorder.txt")) if "table=" in l]
    out = []
    for _ in range(n):
        line = rng.choice(src)
        head, table = line.split("table=")
        rows = [r.split() for r in table.split("|")]
        q = rng.randrange(len(rows))
        a = rng.randrange(2)
        u = rng.random()
        if u < 0.15:
            rows[q][a] = "---"
        elif u < 0.25:
            rows[q][a] = "?---"
        else:
            rows[q][a] = f"{rng.randrange(2)}{rng.choice('LR')}{rng.randrange(len(rows))}"
        out.append(head + "table=" + "|".join(" ".join(r) for r in rows))
    return out


@pytest.mark.skipif(not os.path.exists(os.path.join(O.REF_DIR, "recheck")), reason="reference binaries not built here")
def test_recheck_and_deep_vs_reference_binaries_on_mutants():
    """The oracle's recheck.c / deep.c restatements against the reference
    programs on 60 seeded mutants of real survivors, which fail at every kind
    of point (counter change, limit, off tape, halt, free cell read)."""
    lines = _mutants(60, 31)
    nmax = 11
    data = "\n".join(lines) + "\n"
    rr = subprocess.run([os.path.join(O.REF_DIR, "recheck"), str(nmax)], input=data, capture_output=True, text=True,
                        check=True, timeout=600)
    ref = [l.split(": ", 1)[1] for l in rr.stdout.splitlines() if ": " in l]
    assert len(ref) == len(lines)
    kinds = set()
    for line, want in zip(lines, ref):
        ok, got, _ = O.recheck_line(line, nmax)
        assert got == want, (line, got, want)
        kinds.add(want.split(" ")[0])
    assert len(kinds) >= 3  # several verdict kinds were exercised
    rd = subprocess.run([os.path.join(O.REF_DIR, "deep"), str(nmax)], input=data, capture_output=True, text=True,
                        check=True, timeout=600)
    dref = [l for l in rd.stdout.splitlines() if l.startswith("survivor")]
    assert len(dref) == len(lines)
    for i, (line, want) in enumerate(zip(lines, dref)):
        assert f"survivor {i + 1} " + O.deep_line(line, nmax) == want


@pytest.mark.skipif(not os.path.exists(REFBIN), reason="reference binaries not built here")
def test_estimate_vs_reference_binary_random():
    """The restated probe() against the reference binary's estimate mode on one
    thread, for 6 seeded random jobs (delete with FMAX, free, freesym)."""
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
        r, job = O.setup(base, X, fmax=fmax, free_cells=cells or None, lo=lo, hi=hi)
        if r < 0:
            continue
        seed = rng.randrange(1000)
        args = [REFBIN, "estimate", os.path.join(O.MACHINES, "erdos_14.txt"), "400", str(X), str(fmax), str(lo),
                str(hi)] + cells
        p = subprocess.run(args, capture_output=True, text=True, timeout=300,
                           env=dict(os.environ, OMP_NUM_THREADS="1", E13_SEED=str(seed)))
        assert p.returncode == 0, p.stderr
        assert O.estimate_lines(job, 400, seed) == p.stdout.splitlines()[1:5], args
        done += 1
