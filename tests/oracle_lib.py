"""ctypes access to the CPU oracle (oracle/e13_oracle.c), for tests and for
bench.py's cpu_baseline leg only.  The oracle is the checker, never the thing
measured as the product.

Also holds the text helpers the tests share: survivor-line formatting in the
reference's format (src/e13search.c:184-200 ``report``) and the parsing of the
summary lines the reference prints (src/e13search.c:413-416).
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "_build", "libe13oracle.so")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")
MACHINES = os.path.join(ROOT, "tests", "golden", "machines")

REC_INTS = 40
FREE = -2
HALT = -1

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-s", "-C", ORACLE_DIR, "oracle"], check=True)
        L = ctypes.CDLL(ORACLE_SO)
        I = ctypes.c_int
        P = ctypes.POINTER
        L.oracle_keys.argtypes = [P(ctypes.c_uint64), P(ctypes.c_uint64)]
        L.oracle_parse_cell.argtypes = [ctypes.c_char_p]
        L.oracle_load.argtypes = [ctypes.c_char_p, P(I)]
        L.oracle_setup.argtypes = [P(I), I, I, I, ctypes.c_char_p, I, I, P(I), P(I), P(I), P(I), P(I)]
        L.oracle_search.argtypes = [P(I), I, I, I, I, I, I, P(ctypes.c_longlong), P(I), I, P(I)]
        L.oracle_search_shard.argtypes = [P(I), I, I, I, I, I, I, I, I, P(ctypes.c_longlong), P(I), I, P(I)]
        L.oracle_run_full.argtypes = [P(I), I, P(ctypes.c_longlong)]
        L.oracle_recheck_line.argtypes = [ctypes.c_char_p, I, ctypes.c_char_p, I, ctypes.c_char_p, I]
        L.oracle_deep_line.argtypes = [ctypes.c_char_p, I, ctypes.c_char_p, I]
        L.oracle_raw_tables.argtypes = [ctypes.c_uint64, ctypes.c_long, I, ctypes.c_char_p]
        L.oracle_raw_run.argtypes = [ctypes.c_char_p, ctypes.c_long, I, ctypes.c_long, P(ctypes.c_longlong)]
        L.oracle_probe_stream.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.oracle_probe_stream.restype = ctypes.c_uint64
        L.oracle_probe.argtypes = [P(I), I, I, I, I, I, P(ctypes.c_uint64), P(ctypes.c_double)]
        L.oracle_probe.restype = None
        L.oracle_check_line.argtypes = [ctypes.c_char_p, ctypes.c_char_p, I]
        _lib = L
    return _lib


def keys():
    k = (ctypes.c_uint64 * 1364)()
    t = (ctypes.c_uint64 * 10)()
    lib().oracle_keys(k, t)
    return list(k), list(t)


def parse_machine_text(text: str) -> list[int]:
    """Cells of a machine file, two per line, first 16 lines
    (src/e13search.c:105-121)."""
    base = []
    toks = text.split()
    for i in range(0, min(len(toks) // 2, 16) * 2, 2):
        for s in (toks[i], toks[i + 1]):
            base.append(lib().oracle_parse_cell(s.encode()))
    return base


def load_machine(name_or_path: str) -> list[int]:
    path = name_or_path if os.path.exists(name_or_path) else os.path.join(MACHINES, name_or_path)
    with open(path) as f:
        return parse_machine_text(f.read())


def cell_index(name: str) -> int:
    """'D0' -> 2*3+0 (src/e13search.c:471)."""
    return 2 * (ord(name[0]) - ord("A")) + int(name[1])


class Job:
    def __init__(self, tab, nq, budget, sym_lo, sym_hi, sym_n0, nforced, X):
        self.tab, self.nq, self.budget = tab, nq, budget
        self.sym_lo, self.sym_hi, self.sym_n0, self.nforced, self.X = sym_lo, sym_hi, sym_n0, nforced, X


def setup(base, X, fmax=0, free_cells=None, lo=-1, hi=-1):
    """Returns (status, Job).  status >= 0 is the budget; <0 see
    oracle_setup()."""
    nq0 = len(base) // 2
    b = (ctypes.c_int * 32)(*(base + [HALT] * (32 - len(base))))
    fb = None
    if free_cells is not None:
        arr = bytearray(32)
        for c in free_cells:
            arr[cell_index(c)] = 1
        fb = bytes(arr)
    tab = (ctypes.c_int * 32)()
    slo, shi, n0, nf = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    r = lib().oracle_setup(b, nq0, X, fmax, fb, lo, hi, tab, ctypes.byref(slo), ctypes.byref(shi),
                           ctypes.byref(n0), ctypes.byref(nf))
    nq = nq0 - (1 if X >= 0 else 0)
    return r, Job(list(tab)[: 2 * nq], nq, r, slo.value, shi.value, n0.value, nf.value, X)


def search(job: Job, nthreads: int = 8, surv_cap: int = 100000, shard: int = 0, nshards: int = 1):
    """Runs the oracle search (with nshards > 1, one share of it, see
    oracle_search_shard); returns (counts dict, list of survivor records)."""
    tab = (ctypes.c_int * 32)(*(job.tab + [HALT] * (32 - len(job.tab))))
    counts = (ctypes.c_longlong * 13)()
    surv = (ctypes.c_int * (REC_INTS * surv_cap))()
    ns = ctypes.c_int()
    lib().oracle_search_shard(tab, job.nq, max(job.budget, 0), job.sym_lo, job.sym_hi, job.sym_n0, nthreads, shard,
                              nshards, counts, surv, surv_cap, ctypes.byref(ns))
    c = list(counts)
    recs = []
    for k in range(min(ns.value, surv_cap)):
        r = surv[REC_INTS * k: REC_INTS * (k + 1)]
        recs.append(dict(tab=list(r[: 2 * job.nq]), mask=r[32] & 0xFFFFFFFF, st0=r[33], head0=r[34], abs=r[35],
                         rel=r[36], steps=r[37]))
    return dict(leaves=c[0], survivors=c[1], steps=c[2], hist=c[3:13]), recs


def run_full(tab, nq):
    out = (ctypes.c_longlong * 7)()
    t = (ctypes.c_int * 32)(*(list(tab) + [HALT] * (32 - len(tab))))
    lib().oracle_run_full(t, nq, out)
    return list(out)


def recheck_line(line: str, nmax: int):
    v = ctypes.create_string_buffer(512)
    cl = 2048
    ctr = ctypes.create_string_buffer(cl * 20)
    ok = lib().oracle_recheck_line(line.encode(), nmax, v, 512, ctr, cl)
    counters = [ctr.raw[i * cl: (i + 1) * cl].split(b"\0", 1)[0].decode() for i in range(nmax)]
    return ok, v.value.decode(), counters


def deep_line(line: str, nmax: int):
    out = ctypes.create_string_buffer(8192)
    lib().oracle_deep_line(line.encode(), nmax, out, 8192)
    return out.value.decode()


# ---------------------------------------------------------------------------
# text formats of the reference


def cell_str(code: int) -> str:
    """src/e13search.c:179-182."""
    if code < 0:
        return "---"
    return f"{code & 1}{'R' if code & 2 else 'L'}{code >> 2}"


def survivor_line(X: int, rec: dict, nq: int) -> str:
    """src/e13search.c:184-200."""
    rows = []
    for q in range(nq):
        cells = []
        for a in (0, 1):
            i = 2 * q + a
            mark = "" if (rec["mask"] >> i) & 1 else "?"
            code = rec["tab"][i]
            cells.append(mark + cell_str(-1 if code == FREE else code))
        rows.append(" ".join(cells))
    return (f"SURVIVOR X={X} st0={rec['st0']} head0={rec['head0']} abs={rec['abs']} rel={rec['rel']} "
            f"steps={rec['steps']} table=" + "|".join(rows))


SUMMARY_RE = re.compile(r"X=(-?\d+) .*?leaves=(\d+) survivors=(\d+)(?: steps=(\d+))?.*?dead-at-stage\(0\.\.9\):((?: \d+){10})")


def parse_summary(line: str):
    m = SUMMARY_RE.search(line)
    if not m:
        return None
    return dict(X=int(m.group(1)), leaves=int(m.group(2)), survivors=int(m.group(3)),
                steps=int(m.group(4)) if m.group(4) else None, hist=[int(x) for x in m.group(5).split()])


def raw_tables(seed: int, n: int, nq: int = 13) -> bytes:
    """Random tables of the raw-simulator set (splitmix64 draws, mod 4nq)."""
    buf = ctypes.create_string_buffer(n * 2 * nq)
    lib().oracle_raw_tables(seed, n, nq, buf)
    return buf.raw


def raw_run(codes: bytes, n: int, nq: int = 13, max_steps: int = 1 << 18):
    out = (ctypes.c_longlong * (4 * n))()
    lib().oracle_raw_run(codes, n, nq, max_steps, out)
    return [list(out[4 * i: 4 * i + 4]) for i in range(n)]


def probe(job: Job, rng_state: int):
    """One estimator probe (src/e13search.c:262-313) from the given splitmix64
    state; returns ([leaves, nodes, steps, survivors], the state after it)."""
    tab = (ctypes.c_int * 32)(*(job.tab + [HALT] * (32 - len(job.tab))))
    out = (ctypes.c_double * 4)()
    st = ctypes.c_uint64(rng_state)
    lib().oracle_probe(tab, job.nq, max(job.budget, 0), job.sym_lo, job.sym_hi, job.sym_n0, ctypes.byref(st), out)
    return list(out), st.value


def probe_stream(seed: int, k: int) -> int:
    """The splitmix64 state the reference gives OpenMP thread k (src/e13search.c:486-491)."""
    return lib().oracle_probe_stream(seed, k)


def estimate_per_probe(job: Job, probes: int, seed: int = 0):
    """Per-probe results with probe p on stream k = p (the device's layout)."""
    return [probe(job, probe_stream(seed, p))[0] for p in range(probes)]


def estimate_lines(job: Job, probes: int, seed: int = 0) -> list[str]:
    """The four result lines the reference prints for `estimate` run on one
    OpenMP thread (src/e13search.c:505-509): all probes on thread 0's stream."""
    st = probe_stream(seed, 0)
    rows = []
    for _ in range(probes):
        o, st = probe(job, st)
        rows.append(o)
    return lines_from_rows(rows)


def lines_from_rows(rows) -> list[str]:
    """Mean and standard error lines of per-probe results, summed in order
    (src/e13search.c:500-509)."""
    import math
    n = len(rows)
    s, q = [0.0] * 4, [0.0] * 4
    for o in rows:
        for j in range(4):
            s[j] += o[j]
            q[j] += o[j] * o[j]
    lines = []
    for j, name in enumerate(("leaves", "nodes", "steps", "survivors")):
        m = s[j] / n
        var = q[j] / n - m * m
        se = math.sqrt(var / n) if var > 0 else 0.0
        lines.append("  %-9s %.3e  (+- %.1e standard error)" % (name, m, se))
    return lines


def check_line(line: str) -> list[str]:
    """check.py's output lines for one input line (src/check.py:165-173)."""
    buf = ctypes.create_string_buffer(1 << 16)
    n = lib().oracle_check_line(line.encode(), buf, len(buf))
    return buf.value.decode().splitlines() if n else []


def check_golden(path: str) -> list[tuple[str, list[str]]]:
    """(input line, verdict lines) pairs of a shipped check.py output."""
    pairs = []
    for line in open(path):
        line = line.rstrip("\n")
        if "table=" in line:
            pairs.append([line, []])
        elif line.startswith("   halt@") and pairs:
            pairs[-1][1].append(line)
    return [(l, v) for l, v in pairs if v]
