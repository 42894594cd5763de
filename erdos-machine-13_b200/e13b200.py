"""Python access to libe13b200.so through its C-ABI (include/e13.h).

This module only marshals arguments; all search work runs in the CUDA kernels
of the shared library.  There is no CPU fallback: without the built library or
without a CUDA device the calls raise.

The function names follow the reference's program structure
(src/e13search.c: load, setup, run_delete, run_full, report; src/recheck.c).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libe13b200.so")

E13_MAXCELLS = 32
E13_HALT = -1
E13_FREE = -2
KERNEL_PLAIN = 0
KERNEL_PERSISTENT = 1

ERRORS = {
    -1: "bad argument", -2: "forced cells exceed FMAX", -3: "symmetric state named by a fixed cell or has one",
    -4: "start state in the symmetric states", -5: "CUDA error", -6: "frontier stack overflow",
    -7: "survivor buffer too small", -8: "too many states", -9: "cannot open machine file",
    -10: "device wait timed out", -11: "no CUDA device", -12: "more than the fixed no-allocation memory holds",
    -13: "checkpoint unreadable or of another run",
}
STOPPED = 3  # e13_search_resumable stopped cleanly with a checkpoint
E13_CHECK_NOALLOC_MAX = 16


class E13Error(RuntimeError):
    def __init__(self, code, what=""):
        super().__init__(f"{what}: {ERRORS.get(code, code)} ({code})")
        self.code = code


class Checkpoint(ctypes.Structure):
    _fields_ = [("path", ctypes.c_char_p), ("config", ctypes.c_char_p), ("interval_s", ctypes.c_double),
                ("stop_after_s", ctypes.c_double)]


class EstimateOut(ctypes.Structure):
    _fields_ = [("mean", ctypes.c_double * 4), ("std_error", ctypes.c_double * 4), ("probes", ctypes.c_int64)]


class Job(ctypes.Structure):
    _fields_ = [("X", ctypes.c_int32), ("nq", ctypes.c_int32), ("tab", ctypes.c_int32 * E13_MAXCELLS),
                ("budget", ctypes.c_int32), ("nforced", ctypes.c_int32), ("sym_lo", ctypes.c_int32),
                ("sym_hi", ctypes.c_int32), ("sym_n0", ctypes.c_int32)]


class Counts(ctypes.Structure):
    _fields_ = [("leaves", ctypes.c_uint64), ("survivors", ctypes.c_uint64), ("steps", ctypes.c_uint64),
                ("hist", ctypes.c_uint64 * 10)]

    def as_dict(self):
        return dict(leaves=self.leaves, survivors=self.survivors, steps=self.steps, hist=list(self.hist))


class Survivor(ctypes.Structure):
    _fields_ = [("tab", ctypes.c_int32 * E13_MAXCELLS), ("read_mask", ctypes.c_uint32), ("st0", ctypes.c_int32),
                ("head0", ctypes.c_int32), ("abs_ok", ctypes.c_int32), ("rel_ok", ctypes.c_int32),
                ("steps", ctypes.c_int64)]


class Tuning(ctypes.Structure):
    _fields_ = [("kernel", ctypes.c_int32), ("block", ctypes.c_int32), ("slice", ctypes.c_int32),
                ("warp_stack", ctypes.c_int32), ("step_cap", ctypes.c_int32), ("batch", ctypes.c_int32),
                ("epoch_us", ctypes.c_int32), ("epochs_per_graph", ctypes.c_int32), ("pool_low_pct", ctypes.c_int32),
                ("run_skip", ctypes.c_int32), ("stack_nodes", ctypes.c_int64)]


class Stats(ctypes.Structure):
    _fields_ = [("device_ms", ctypes.c_double), ("launches", ctypes.c_int64), ("epochs", ctypes.c_int64),
                ("peak_nodes", ctypes.c_int64), ("search_kernel_launches", ctypes.c_int64),
                ("search_kernel_ms", ctypes.c_double), ("lane_occupancy", ctypes.c_double),
                ("warp_rounds", ctypes.c_int64), ("donations", ctypes.c_int64), ("pool_claims", ctypes.c_int64),
                ("idle_polls", ctypes.c_int64), ("h2d_bytes", ctypes.c_int64), ("d2h_bytes", ctypes.c_int64)]


class ServeResult(ctypes.Structure):
    _fields_ = [("id", ctypes.c_int64), ("status", ctypes.c_int32), ("nsurv", ctypes.c_int32), ("counts", Counts),
                ("t_submit", ctypes.c_double), ("t_start", ctypes.c_double), ("t_done", ctypes.c_double)]


E13_CHECK_MAX_NMAX = 20
E13_CHECK_MAX_ONES = 64


class CheckIn(ctypes.Structure):
    _fields_ = [("nq", ctypes.c_int32), ("st0", ctypes.c_int32), ("rel", ctypes.c_int32), ("head0", ctypes.c_int64),
                ("kind", ctypes.c_int8 * E13_MAXCELLS), ("write", ctypes.c_int8 * E13_MAXCELLS),
                ("move", ctypes.c_int8 * E13_MAXCELLS), ("next", ctypes.c_int8 * E13_MAXCELLS)]


class CheckOut(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("fail_stage", ctypes.c_int32), ("free_state", ctypes.c_int32),
                ("free_sym", ctypes.c_int32), ("fail_t", ctypes.c_int64), ("fail_head", ctypes.c_int64),
                ("stages_done", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("stage_t", ctypes.c_int64 * (E13_CHECK_MAX_NMAX + 1)),
                ("minhead", ctypes.c_int64 * (E13_CHECK_MAX_NMAX + 1)),
                ("nones", ctypes.c_int32 * (E13_CHECK_MAX_NMAX + 1)),
                ("leftmost", ctypes.c_int64 * (E13_CHECK_MAX_NMAX + 1)),
                ("ones_cells", (ctypes.c_int32 * E13_CHECK_MAX_ONES) * (E13_CHECK_MAX_NMAX + 1))]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    """Loads libe13b200.so (building it first if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        I = ctypes.c_int
        L.e13_keys.argtypes = [P(ctypes.c_uint64), P(ctypes.c_uint64)]
        L.e13_keys.restype = None
        L.e13_parse_cell.argtypes = [ctypes.c_char_p]
        L.e13_load_machine.argtypes = [ctypes.c_char_p, P(ctypes.c_int32)]
        L.e13_parse_machine.argtypes = [ctypes.c_char_p, P(ctypes.c_int32)]
        L.e13_setup.argtypes = [P(ctypes.c_int32), I, I, I, ctypes.c_char_p, I, I, P(Job)]
        L.e13_format_survivor.argtypes = [P(Job), P(Survivor), ctypes.c_char_p, ctypes.c_size_t]
        L.e13_format_summary.argtypes = [P(Job), P(Counts), ctypes.c_double, ctypes.c_char_p, ctypes.c_size_t]
        L.e13_default_tuning.argtypes = [P(Tuning)]
        L.e13_default_tuning.restype = None
        L.e13_resolve_tuning.argtypes = [P(Tuning), I, P(Tuning)]
        L.e13_selftest_pool_wait.argtypes = [ctypes.c_void_p, ctypes.c_int32]
        L.e13_ctx_create.argtypes = [I, P(ctypes.c_void_p)]
        L.e13_ctx_destroy.argtypes = [ctypes.c_void_p]
        L.e13_ctx_destroy.restype = None
        L.e13_search.argtypes = [ctypes.c_void_p, P(Job), P(Tuning), P(Counts), P(Survivor), I, P(I)]
        L.e13_search_resumable.argtypes = [ctypes.c_void_p, P(Job), P(Tuning), P(Checkpoint), P(Counts),
                                           P(Survivor), I, P(I), P(ctypes.c_double), P(ctypes.c_int64)]
        L.e13_last_stats.argtypes = [ctypes.c_void_p, P(Stats)]
        L.e13_search_shard.argtypes = [ctypes.c_void_p, P(Job), P(Tuning), I, I, P(Counts), P(Survivor), I, P(I)]
        L.e13_check_crafted.argtypes = [ctypes.c_void_p, P(ctypes.c_char_p), I, ctypes.c_char_p, ctypes.c_size_t,
                                        P(ctypes.c_size_t)]
        L.e13_estimate.argtypes = [ctypes.c_void_p, P(Job), ctypes.c_int64, ctypes.c_uint64, P(EstimateOut),
                                   P(ctypes.c_double)]
        L.e13_autotune.argtypes = [ctypes.c_void_p, P(Job), ctypes.c_int32, P(Tuning), P(Tuning), P(ctypes.c_double)]
        L.e13_autotune_jobs.argtypes = [ctypes.c_void_p, P(Job), I, ctypes.c_int32, P(Tuning), P(Tuning),
                                        P(ctypes.c_double)]
        L.e13_serve_create.argtypes = [ctypes.c_void_p, P(Tuning), ctypes.c_int64, P(ctypes.c_void_p)]
        L.e13_serve_destroy.argtypes = [ctypes.c_void_p]
        L.e13_serve_destroy.restype = None
        L.e13_serve_clock.argtypes = [ctypes.c_void_p]
        L.e13_serve_clock.restype = ctypes.c_double
        L.e13_serve_submit.argtypes = [ctypes.c_void_p, P(Job), ctypes.c_int64, ctypes.c_double]
        L.e13_serve_step.argtypes = [ctypes.c_void_p, P(ServeResult), I, P(I)]
        L.e13_serve_submit_shard.argtypes = [ctypes.c_void_p, P(Job), ctypes.c_int64, ctypes.c_double, I, I]
        L.e13_serve_pending.argtypes = [ctypes.c_void_p]
        L.e13_serve_pending.restype = ctypes.c_int64
        L.e13_serve_survivors.argtypes = [ctypes.c_void_p, ctypes.c_int64, P(Survivor), I, P(I)]
        L.e13_serve_stats.argtypes = [ctypes.c_void_p, P(ctypes.c_double), P(ctypes.c_int64), P(ctypes.c_int64),
                                      P(ctypes.c_int64), P(ctypes.c_int64)]
        L.e13_serve_preempt.argtypes = [ctypes.c_void_p, ctypes.c_int64]
        L.e13_run_full.argtypes = [ctypes.c_void_p, P(ctypes.c_int32), I, I, P(ctypes.c_int64)]
        L.e13_check.argtypes = [ctypes.c_void_p, P(CheckIn), I, I, I, P(CheckOut)]
        L.e13_check_noalloc.argtypes = [I, P(CheckIn), I, I, I, P(CheckOut)]
        L.e13_raw_run.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int64, I,
                                  ctypes.c_int64, P(ctypes.c_int64), P(ctypes.c_uint64)]
        L.e13_parse_survivor_line.argtypes = [ctypes.c_char_p, P(CheckIn)]
        L.e13_survivor_check_in.argtypes = [P(Job), P(Survivor), P(CheckIn)]
        L.e13_format_recheck.argtypes = [P(CheckOut), I, ctypes.c_char_p, ctypes.c_size_t]
        L.e13_format_deep.argtypes = [P(CheckIn), P(CheckOut), I, ctypes.c_char_p, ctypes.c_size_t]
        _lib = L
    return _lib


EXPORTED = ["e13_keys", "e13_parse_cell", "e13_load_machine", "e13_parse_machine", "e13_setup",
            "e13_format_survivor", "e13_format_summary", "e13_default_tuning", "e13_ctx_create", "e13_ctx_destroy",
            "e13_search", "e13_search_shard", "e13_search_resumable", "e13_estimate", "e13_last_stats", "e13_run_full", "e13_check", "e13_parse_survivor_line",
            "e13_format_recheck", "e13_format_deep", "e13_check_crafted", "e13_raw_run", "e13_autotune", "e13_check_noalloc",
            "e13_serve_create", "e13_serve_destroy", "e13_serve_clock", "e13_serve_submit", "e13_serve_step",
            "e13_serve_pending", "e13_serve_survivors", "e13_serve_stats", "e13_resolve_tuning",
            "e13_selftest_pool_wait", "e13_serve_submit_shard", "e13_serve_preempt", "e13_autotune_jobs",
            "e13_survivor_check_in"]


def keys():
    k = (ctypes.c_uint64 * 1364)()
    t = (ctypes.c_uint64 * 10)()
    lib().e13_keys(k, t)
    return list(k), list(t)


def load_machine(path: str) -> list[int]:
    base = (ctypes.c_int32 * E13_MAXCELLS)()
    nq = lib().e13_load_machine(path.encode(), base)
    if nq < 0:
        raise E13Error(nq, path)
    return list(base)[: 2 * nq]


def parse_machine(text: str) -> list[int]:
    base = (ctypes.c_int32 * E13_MAXCELLS)()
    nq = lib().e13_parse_machine(text.encode(), base)
    return list(base)[: 2 * nq]


def cell_index(name: str) -> int:
    return 2 * (ord(name[0]) - ord("A")) + int(name[1])


def setup(base, X, fmax=0, free_cells=None, lo=-1, hi=-1):
    """Returns (status, Job); status 0 or a negative e13 error (the job is
    still filled as far as the reference's setup() gets)."""
    b = (ctypes.c_int32 * E13_MAXCELLS)(*(list(base) + [E13_HALT] * (E13_MAXCELLS - len(base))))
    fb = None
    if free_cells is not None:
        arr = bytearray(E13_MAXCELLS)
        for c in free_cells:
            arr[cell_index(c) if isinstance(c, str) else c] = 1
        fb = bytes(arr)
    job = Job()
    r = lib().e13_setup(b, len(base) // 2, X, fmax, fb, lo, hi, ctypes.byref(job))
    return r, job


def tuning(**kw) -> Tuning:
    t = Tuning()
    lib().e13_default_tuning(ctypes.byref(t))
    for k, v in kw.items():
        setattr(t, k, v)
    return t


def resolve_tuning(tune: Tuning | None, serve: bool = False):
    """(status, Tuning): the tuning a search or serve session would run with
    (e13_resolve_tuning); status E13_ERR_ARG for a field out of range."""
    out = Tuning()
    r = lib().e13_resolve_tuning(ctypes.byref(tune) if tune else None, 1 if serve else 0, ctypes.byref(out))
    return r, out


class Context:
    """A device context (one CUDA device, one stream, reusable buffers)."""

    def __init__(self, device: int = 0):
        self.h = ctypes.c_void_p()
        r = lib().e13_ctx_create(device, ctypes.byref(self.h))
        if r:
            raise E13Error(r, "e13_ctx_create")

    def close(self):
        if self.h:
            lib().e13_ctx_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def search(self, job: Job, tune: Tuning | None = None, surv_cap: int = 1 << 16):
        counts = Counts()
        surv = (Survivor * max(surv_cap, 1))()
        ns = ctypes.c_int()
        r = lib().e13_search(self.h, ctypes.byref(job), ctypes.byref(tune) if tune else None, ctypes.byref(counts),
                             surv, surv_cap, ctypes.byref(ns))
        if r and r != -7:
            raise E13Error(r, "e13_search")
        return counts, [surv[i] for i in range(min(ns.value, surv_cap))]

    def selftest_pool_wait(self, wait_us: int) -> int:
        """Status of e13_selftest_pool_wait: E13_ERR_TIMEOUT (-10) when the
        persistent kernel's bounded pool wait runs out as it should."""
        return lib().e13_selftest_pool_wait(self.h, wait_us)

    def search_shard(self, job: Job, shard: int, nshards: int, tune: Tuning | None = None, surv_cap: int = 1 << 16):
        """Shard `shard` of `nshards` of the search for `job` (e13_search_shard)."""
        counts = Counts()
        surv = (Survivor * max(surv_cap, 1))()
        ns = ctypes.c_int()
        r = lib().e13_search_shard(self.h, ctypes.byref(job), ctypes.byref(tune) if tune else None, shard, nshards,
                                   ctypes.byref(counts), surv, surv_cap, ctypes.byref(ns))
        if r and r != -7:
            raise E13Error(r, "e13_search_shard")
        return counts, [surv[i] for i in range(min(ns.value, surv_cap))]

    def search_resumable(self, job: Job, path: str, config: str, interval_s: float = 0.0,
                         stop_after_s: float = 0.0, tune: Tuning | None = None, surv_cap: int = 1 << 16):
        """e13_search with checkpoints at `path`.  Returns (status, counts,
        survivors, wall seconds over all calls, frontier nodes left); status is
        0 when the search finished, STOPPED when it stopped with a checkpoint."""
        ck = Checkpoint(path.encode(), config.encode(), interval_s, stop_after_s)
        counts = Counts()
        surv = (Survivor * max(surv_cap, 1))()
        ns = ctypes.c_int()
        wall = ctypes.c_double()
        left = ctypes.c_int64()
        r = lib().e13_search_resumable(self.h, ctypes.byref(job), ctypes.byref(tune) if tune else None,
                                       ctypes.byref(ck), ctypes.byref(counts), surv, surv_cap, ctypes.byref(ns),
                                       ctypes.byref(wall), ctypes.byref(left))
        if r not in (0, -7, STOPPED):
            raise E13Error(r, "e13_search_resumable")
        return r, counts, [surv[i] for i in range(min(ns.value, surv_cap))], wall.value, left.value

    def estimate(self, job: Job, probes: int, seed: int = 0, per_probe: bool = False):
        """Knuth size estimate of the search for `job`; returns (EstimateOut,
        per-probe [leaves, nodes, steps, survivors] rows or None)."""
        out = EstimateOut()
        buf = (ctypes.c_double * (4 * probes))() if per_probe else None
        r = lib().e13_estimate(self.h, ctypes.byref(job), probes, seed, ctypes.byref(out), buf)
        if r:
            raise E13Error(r, "e13_estimate")
        rows = [list(buf[4 * p: 4 * p + 4]) for p in range(probes)] if per_probe else None
        return out, rows

    def check_crafted(self, lines):
        """src/check.py on the device: its output lines for these input lines."""
        arr = (ctypes.c_char_p * max(len(lines), 1))(*[l.encode() for l in lines])
        need = ctypes.c_size_t()
        size = 1 << 16
        for _ in range(2):
            buf = ctypes.create_string_buffer(size)
            r = lib().e13_check_crafted(self.h, arr, len(lines), buf, size, ctypes.byref(need))
            if r == -1 and need.value > size:
                size = need.value
                continue
            if r:
                raise E13Error(r, "e13_check_crafted")
            return buf.value.decode().splitlines()
        raise E13Error(-1, "e13_check_crafted")

    def autotune(self, job: Job, start: Tuning | None = None, proxy_shards: int = 1):
        """Coordinate-descent tuning of the persistent kernel, timed on shard 0 of
        proxy_shards of `job`; returns (Tuning, best proxy ms)."""
        best = Tuning()
        ms = ctypes.c_double()
        r = lib().e13_autotune(self.h, ctypes.byref(job), proxy_shards, ctypes.byref(start) if start else None,
                               ctypes.byref(best), ctypes.byref(ms))
        if r:
            raise E13Error(r, "e13_autotune")
        return best, ms.value

    def autotune_jobs(self, jobs, start: Tuning | None = None, proxy_shards: int = 1):
        """Coordinate-descent tuning timed on shard 0 of proxy_shards of every job,
        all in one serve session; returns (Tuning, best proxy ms)."""
        arr = (Job * len(jobs))(*jobs)
        best = Tuning()
        ms = ctypes.c_double()
        r = lib().e13_autotune_jobs(self.h, arr, len(jobs), proxy_shards, ctypes.byref(start) if start else None,
                                    ctypes.byref(best), ctypes.byref(ms))
        if r:
            raise E13Error(r, "e13_autotune_jobs")
        return best, ms.value

    def stats(self) -> Stats:
        s = Stats()
        lib().e13_last_stats(self.h, ctypes.byref(s))
        return s

    def run_full(self, tabs, nq):
        n = len(tabs)
        arr = (ctypes.c_int32 * (E13_MAXCELLS * max(n, 1)))()
        for i, t in enumerate(tabs):
            for j, v in enumerate(t):
                arr[E13_MAXCELLS * i + j] = v
        out = (ctypes.c_int64 * (7 * max(n, 1)))()
        r = lib().e13_run_full(self.h, arr, n, nq, out)
        if r:
            raise E13Error(r, "e13_run_full")
        return [list(out[7 * i: 7 * i + 7]) for i in range(n)]

    def raw_run(self, n, nq=13, max_steps=1 << 18, seed=0, codes: bytes | None = None, want_out=True,
                as_array=False):
        """Raw-simulator set; returns (per-machine [steps, status, head, ones] or None, total steps).
        as_array: the rows as one flat ctypes int64 array (4 per machine) instead of lists."""
        out = (ctypes.c_int64 * (4 * n))() if want_out else None
        tot = ctypes.c_uint64()
        r = lib().e13_raw_run(self.h, codes, seed, n, nq, max_steps, out, ctypes.byref(tot))
        if r:
            raise E13Error(r, "e13_raw_run")
        if as_array or not want_out:
            return out, tot.value
        return [list(out[4 * i: 4 * i + 4]) for i in range(n)], tot.value

    def check(self, ins, nmax, mode=0):
        n = len(ins)
        arr = (CheckIn * max(n, 1))(*ins)
        out = (CheckOut * max(n, 1))()
        r = lib().e13_check(self.h, arr, n, nmax, mode, out)
        if r:
            raise E13Error(r, "e13_check")
        return [out[i] for i in range(n)]


def survivor_line(job: Job, s: Survivor) -> str:
    buf = ctypes.create_string_buffer(1024)
    n = lib().e13_format_survivor(ctypes.byref(job), ctypes.byref(s), buf, 1024)
    if n < 0:
        raise E13Error(n, "e13_format_survivor")
    return buf.value.decode()


def summary_line(job: Job, c: Counts, wall: float) -> str:
    buf = ctypes.create_string_buffer(512)
    lib().e13_format_summary(ctypes.byref(job), ctypes.byref(c), wall, buf, 512)
    return buf.value.decode()


def parse_survivor_line(line: str) -> CheckIn | None:
    ci = CheckIn()
    return ci if lib().e13_parse_survivor_line(line.encode(), ctypes.byref(ci)) else None


def survivor_check_in(job: Job, s: Survivor) -> CheckIn:
    """The checker input of a survivor a search returned (e13_survivor_check_in)."""
    ci = CheckIn()
    r = lib().e13_survivor_check_in(ctypes.byref(job), ctypes.byref(s), ctypes.byref(ci))
    if r:
        raise E13Error(r, "e13_survivor_check_in")
    return ci


def format_recheck(o: CheckOut, nmax: int) -> str:
    buf = ctypes.create_string_buffer(8192)
    lib().e13_format_recheck(ctypes.byref(o), nmax, buf, 8192)
    return buf.value.decode()


def format_deep(ci: CheckIn, o: CheckOut, nmax: int) -> str:
    buf = ctypes.create_string_buffer(8192)
    lib().e13_format_deep(ctypes.byref(ci), ctypes.byref(o), nmax, buf, 8192)
    return buf.value.decode()


def check_noalloc(device: int, ins, nmax: int, mode: int = 0):
    """e13_check_noalloc(): the deep check with no device allocation (at most
    E13_CHECK_NOALLOC_MAX machines per call)."""
    n = len(ins)
    arr = (CheckIn * max(n, 1))(*ins)
    out = (CheckOut * max(n, 1))()
    r = lib().e13_check_noalloc(device, arr, n, nmax, mode, out)
    if r:
        raise E13Error(r, "e13_check_noalloc")
    return [out[i] for i in range(n)]


class Server:
    """Continuous batching of search jobs in one persistent kernel (e13_serve_*)."""

    def __init__(self, ctx: Context, tune: Tuning | None = None, reserve_nodes: int = 0):
        self.h = ctypes.c_void_p()
        r = lib().e13_serve_create(ctx.h, ctypes.byref(tune) if tune else None, reserve_nodes, ctypes.byref(self.h))
        if r:
            raise E13Error(r, "e13_serve_create")

    def close(self):
        if self.h:
            lib().e13_serve_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def clock(self) -> float:
        return lib().e13_serve_clock(self.h)

    def submit(self, job: Job, job_id: int, t_submit: float = -1.0):
        r = lib().e13_serve_submit(self.h, ctypes.byref(job), job_id, t_submit)
        if r:
            raise E13Error(r, "e13_serve_submit")

    def submit_shard(self, job: Job, job_id: int, shard: int, nshards: int, t_submit: float = -1.0):
        r = lib().e13_serve_submit_shard(self.h, ctypes.byref(job), job_id, t_submit, shard, nshards)
        if r:
            raise E13Error(r, "e13_serve_submit_shard")

    def step(self):
        res = (ServeResult * 16)()
        n = ctypes.c_int()
        r = lib().e13_serve_step(self.h, res, 16, ctypes.byref(n))
        if r:
            raise E13Error(r, "e13_serve_step")
        return [res[i] for i in range(n.value)]

    def pending(self) -> int:
        return lib().e13_serve_pending(self.h)

    def survivors(self, job_id: int, cap: int = 1 << 16):
        out = (Survivor * cap)()
        n = ctypes.c_int()
        r = lib().e13_serve_survivors(self.h, job_id, out, cap, ctypes.byref(n))
        if r and r != -7:
            raise E13Error(r, "e13_serve_survivors")
        return [out[i] for i in range(min(n.value, cap))]

    def stats(self):
        """(device ms of all epochs, epochs)."""
        ms = ctypes.c_double()
        ep = ctypes.c_int64()
        lib().e13_serve_stats(self.h, ctypes.byref(ms), ctypes.byref(ep), None, None, None)
        return ms.value, ep.value

    def swapped_out(self) -> int:
        """Times a job was swapped out to host memory to make room."""
        n = ctypes.c_int64()
        lib().e13_serve_stats(self.h, None, None, ctypes.byref(n), None, None)
        return n.value

    def peaks(self):
        """(largest frontier after an epoch, largest share of it one job held), in nodes."""
        a, b = ctypes.c_int64(), ctypes.c_int64()
        lib().e13_serve_stats(self.h, None, None, None, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def preempt(self, job_id: int):
        r = lib().e13_serve_preempt(self.h, job_id)
        if r:
            raise E13Error(r, "e13_serve_preempt")

    def run_all(self, jobs, arrivals=None, shard=0, nshards=1):
        """Submits jobs (with optional arrival times; with nshards > 1 this
        rank's share of each) and steps until all are done; returns
        {id: (ServeResult, [Survivor])}."""
        for i, job in enumerate(jobs):
            t = -1.0 if arrivals is None else arrivals[i]
            if nshards > 1:
                self.submit_shard(job, i, shard, nshards, t)
            else:
                self.submit(job, i, t)
        out = {}
        while self.pending():
            for r in self.step():
                out[r.id] = (r, self.survivors(r.id))
        return out
