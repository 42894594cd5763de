#!/usr/bin/env python
"""Benchmark of the TNF enumeration search on B200 (one JSON line on rank 0).

A step is one whole search of the workload: by default the local-edit search
with FMAX = 4 (delete each of erdos_14's 14 states, <= 4 changed cells; the
<=4-cell half of the local-edit config, 5,986,617,022 leaves).  The metric is
simulated Turing-machine steps per second (leaves/s is reported beside it).

  value     steps of the K timed searches / their device time (CUDA events on
            the library's stream, summed over the searches of each step)
  e2e       the same through the public C-ABI call e13_search() timed on the
            host: root node H2D, control block and survivors D2H included
  roofline  integer-issue bound of the search kernel: 16 lane-ops per step
            against SMs x 128 lanes x the SM clock sampled during the run
  cpu_baseline  the reference's own e13search (OpenMP, all host threads) on a
            bounded sample: the FMAX = 3 local-edit search

--impl reference runs that reference CPU program instead (the reference arm).
Under torchrun (N > 1) rank r runs every N-th X starting at r (the search
splits into independent per-X jobs; e13shard.py sums the totals and takes the
maximum of the times over ranks).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "erdos-machine-13_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
MACHINES = os.path.join(ROOT, "tests", "golden", "machines")
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "e13search")

WORKLOADS = {
    "local_edits_f4": dict(desc="delete erdos_14 FMAX=4 X=0..13", machine="erdos_14.txt", mode="delete", fmax=4,
                           X=list(range(14)), leaves=5986617022),
    "local_edits_f3": dict(desc="delete erdos_14 FMAX=3 X=0..13", machine="erdos_14.txt", mode="delete", fmax=3,
                           X=list(range(14)), leaves=36383467),
    "counter_sym": dict(desc="freesym erdos_14 13 10 13 D0 G0 K0 K1 L1 M1", machine="erdos_14.txt", mode="freesym",
                        X=[13], free=["D0", "G0", "K0", "K1", "L1", "M1"], lo=10, hi=13, leaves=3078656272),
    "division_v4": dict(desc="freesym erdos_14 9 3 9 F0..I1", machine="erdos_14.txt", mode="freesym", X=[9],
                        free=["F0", "F1", "G0", "G1", "H0", "H1", "I0", "I1"], lo=3, hi=9, leaves=830955779),
}
WORKLOADS["serving_mix"] = dict(desc="seeded Poisson stream of 40 search jobs on erdos_14 (seed 2026, 25 jobs/s): "
                                    "random deleted state, random free set of 2-5 cells (symmetry where setup "
                                    "allows) or FMAX 2-4, plus counter_sym and FMAX=4 X=11",
                               machine="erdos_14.txt", mode="mix", X=[], leaves=None)
CPU_SAMPLE = "local_edits_f3"


def serving_mix(seed=2026, n=40, rate=25.0):
    """The serving-mix job stream: (kind, X, cells, fmax, lo, hi) and arrival times."""
    import random

    import oracle_lib as O

    rng = random.Random(seed)
    base = O.load_machine("erdos_14.txt")
    cells_all = [f"{chr(65 + q)}{a}" for q in range(14) for a in (0, 1)]
    out, t = [], 0.0
    while len(out) < n:
        t += rng.expovariate(rate)
        X = rng.randrange(14)
        if len(out) == n // 3:
            out.append((("free", 13, ["D0", "G0", "K0", "K1", "L1", "M1"], 0, 10, 13), t))  # counter_sym
            continue
        if len(out) == 2 * n // 3:
            out.append((("delete", 11, None, 4, -1, -1), t))
            continue
        if rng.random() < 0.5:
            cells = rng.sample([c for c in cells_all if ord(c[0]) - 65 != X], rng.randint(2, 5))
            lo = hi = -1
            if rng.random() < 0.5:
                lo, hi = sorted(rng.sample(range(1, 14), 2))
                if not (lo <= X <= hi) or O.setup(base, X, free_cells=cells, lo=lo, hi=hi)[0] < 0:
                    lo = hi = -1  # symmetry only where setup() accepts it
            if O.setup(base, X, free_cells=cells, lo=lo, hi=hi)[0] < 0:
                continue
            out.append((("free", X, cells, 0, lo, hi), t))
        else:
            fmax = rng.randint(2, 4)
            if fmax == 4 and rng.random() < 0.7:
                fmax = 3  # keep most jobs small: the stream spans 1e3 .. 1e9 leaves
            if O.setup(base, X, fmax=fmax)[0] < 0:
                continue
            out.append((("delete", X, None, fmax, -1, -1), t))
    return out
# DRAM bytes (read + write) of one 200 ms epoch launch of the persistent search
# kernel, from the ncu capture summarised in
# profiles/search_kernel_persistent_local_edits_f4.md
PROFILED_TRAFFIC = {"local_edits_f4": 386.7e6}
OPS_PER_STEP = 16  # integer lane-ops per simulated step (hash test 2, deadline 1, address 1, load+extract 2,
#                    index 1, table 2, fork test 1, halt test 1, write test 1, head 2, bounds 2)


def ref_args(w):
    path = os.path.join(MACHINES, w["machine"])
    if w["mode"] == "delete":
        return ["delete", path, str(w["fmax"])] + [str(x) for x in w["X"]]
    if w["mode"] == "freesym":
        return ["freesym", path, str(w["X"][0]), str(w["lo"]), str(w["hi"])] + w["free"]
    return ["free", path, str(w["X"][0])] + w["free"]


def run_reference_cpu(w, threads):
    """The reference's e13search on the host cores; returns (steps, leaves, seconds, kind)."""
    import oracle_lib as O

    if os.path.exists(REF_BIN):
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        t0 = time.perf_counter()
        r = subprocess.run([REF_BIN] + ref_args(w), capture_output=True, text=True, env=env, check=True)
        dt = time.perf_counter() - t0
        s = [O.parse_summary(l) for l in r.stderr.splitlines() if "leaves=" in l]
        return sum(x["steps"] for x in s), sum(x["leaves"] for x in s), dt, "reference"
    # no reference build on this machine: the oracle's restatement (same algorithm, pthreads)
    base = O.load_machine(w["machine"])
    steps = leaves = 0
    t0 = time.perf_counter()
    for X in w["X"]:
        if w["mode"] == "delete":
            st, job = O.setup(base, X, fmax=w["fmax"])
        else:
            st, job = O.setup(base, X, free_cells=w["free"], lo=w.get("lo", -1), hi=w.get("hi", -1))
        if st < 0:
            continue
        c, _ = O.search(job, nthreads=threads)
        steps += c["steps"]
        leaves += c["leaves"]
    return steps, leaves, time.perf_counter() - t0, "port"


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        rows = [l.strip().split(", ") for l in self.f.read().splitlines() if l.strip()]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return ws, rank, local, pg


def reference_arm(args, w, ws, rank, pg):
    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return
    threads = os.cpu_count() or 1
    sample = WORKLOADS[CPU_SAMPLE]
    for _ in range(args.warmup):
        run_reference_cpu(sample, threads)
    tot_steps = tot_leaves = 0
    tot_t = 0.0
    kind = "reference"
    for _ in range(args.steps):
        s, l, dt, kind = run_reference_cpu(sample, threads)
        tot_steps += s
        tot_leaves += l
        tot_t += dt
    v = tot_steps / tot_t
    line = {"metric": "TM steps/s", "value": v, "unit": "steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * tot_t / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "int32+u64", "data": "synthetic (reference searches)",
            "impl": "reference", "leaves_per_s": tot_leaves / tot_t,
            "config": {"workload": f"{CPU_SAMPLE}: {sample['desc']} (bounded sample of {w['desc']})",
                       "sample_of": args.workload},
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": threads, "kind": kind,
                             "sample": f"{sample['desc']} per step"},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


def serving_bench(args, w, ws, rank, local, pg):
    """The serving workload: search jobs arrive as a Poisson stream and join the
    running persistent kernel as job slots and frontier memory free up."""
    import torch

    import e13b200 as E
    import oracle_lib as O

    base = O.load_machine("erdos_14.txt")
    stream = serving_mix()
    jobs, arrivals = [], []
    for (kind, X, cells, fmax, lo, hi), t in stream:
        if kind == "free":
            r, job = E.setup(base, X, free_cells=cells, lo=lo, hi=hi)
        else:
            r, job = E.setup(base, X, fmax=fmax)
        assert r == 0
        jobs.append(job)
        arrivals.append(t)
    ctx = E.Context(local)
    lat, steps, dev_ms, wall, leaves, epochs, launches = [], 0, 0.0, 0.0, [], 0, 0
    for it in range(args.warmup + args.steps):
        with E.Server(ctx) as srv:
            t0 = time.perf_counter()
            got = srv.run_all(jobs, arrivals)
            dt = time.perf_counter() - t0
            ms, ep = srv.stats()
        if it >= args.warmup:
            wall += dt
            dev_ms += ms
            epochs += ep
            launches += ctx.stats().launches
            for r, surv in got.values():
                steps += r.counts.steps
                lat.append(r.t_done - r.t_submit)
                leaves.append(r.counts.leaves)
    lat.sort()
    p = lambda q: lat[min(len(lat) - 1, int(q * len(lat)))]
    line = {"metric": "TM steps/s", "value": steps / wall, "unit": "steps/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * wall / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "int32+u64", "data": "synthetic (seeded job stream)",
            "config": {"workload": f"serving_mix: {w['desc']}", "kernel": "persistent (serve)",
                       "jobs": len(jobs), "leaves_min": min(leaves), "leaves_max": max(leaves)},
            "latency_p50_s": p(0.50), "latency_p99_s": p(0.99),
            "device_busy_frac": dev_ms / 1000 / wall, "gpu_launches": launches,
            "note": "value = steps of all jobs / wall time from the first arrival to the last completion; "
                    "jobs arrive on the host clock, so idle gaps between arrivals count"}
    print(json.dumps(line), flush=True)
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="local_edits_f4", choices=list(WORKLOADS))
    ap.add_argument("--kernel", default="persistent", choices=["persistent", "plain"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    ws, rank, local, pg = dist_setup()
    if args.impl == "reference":
        return reference_arm(args, w, ws, rank, pg)

    import torch

    import e13b200 as E
    import oracle_lib as O

    torch.cuda.set_device(local)
    if args.workload == "serving_mix":
        return serving_bench(args, w, ws, rank, local, pg)
    import e13shard as S

    base = O.load_machine(w["machine"])
    jobs = []
    for X in S.share(w["X"], rank, ws):
        if w["mode"] == "delete":
            r, job = E.setup(base, X, fmax=w["fmax"])
        else:
            r, job = E.setup(base, X, free_cells=w["free"], lo=w.get("lo", -1), hi=w.get("hi", -1))
        if r == 0:
            jobs.append(job)
    kernel = E.KERNEL_PERSISTENT if args.kernel == "persistent" else E.KERNEL_PLAIN
    tune = E.tuning(kernel=kernel)
    ctx = E.Context(local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    kstats = dict(epochs=0, jobs=len(jobs))

    def one_step():
        """One whole search of the workload.  Persistent kernel: all of its jobs
        (one per deleted state X) run concurrently in one serve session.  Plain
        kernel: the jobs run one after another, one launch per frontier batch."""
        steps = leaves = 0
        dev_ms = 0.0
        launches = 0
        surv_bytes = 0
        if kernel == E.KERNEL_PERSISTENT:
            with E.Server(ctx, E.tuning(epoch_us=200000)) as srv:
                got = srv.run_all(jobs)
                ms, epochs = srv.stats()
            for r, surv in got.values():
                steps += r.counts.steps
                leaves += r.counts.leaves
                surv_bytes += 64 * len(surv)
            dev_ms = ms
            launches = ctx.stats().launches  # search, move, finish, node count per epoch; frontier order
            kstats["epochs"] += epochs
        else:
            for job in jobs:
                c, surv = ctx.search(job, tune)
                st = ctx.stats()
                steps += c.steps
                leaves += c.leaves
                dev_ms += st.device_ms
                launches += st.launches
                surv_bytes += 64 * len(surv)
                kstats["epochs"] += st.epochs
        return steps, leaves, dev_ms, launches, surv_bytes

    for _ in range(args.warmup):
        one_step()
    torch.cuda.synchronize()
    tot = dict(steps=0, leaves=0, dev_ms=0.0, wall=0.0, launches=0, d2h=0)
    sampler = ClockSampler(local)
    if pg:
        pg.barrier()
    with sampler:
        for _ in range(args.steps):
            flush.zero_()  # evict L2 (126 MB) between timed steps
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s, l, ms, nl, d2h = one_step()
            torch.cuda.synchronize()
            tot["wall"] += time.perf_counter() - t0
            tot["steps"] += s
            tot["leaves"] += l
            tot["dev_ms"] += ms
            tot["launches"] += nl
            tot["d2h"] += d2h
    if pg:
        pg.barrier()
    clocks = sampler.summary()
    if pg:
        sums, maxes = S.reduce_totals(pg, {k: tot[k] for k in ("steps", "leaves", "launches", "d2h")},
                                      {k: tot[k] for k in ("dev_ms", "wall")}, device=f"cuda:{local}")
        tot.update(sums)
        tot.update(maxes)
    parity = tot["leaves"] == w["leaves"] * args.steps
    dev_s = tot["dev_ms"] / 1000.0
    value = tot["steps"] / dev_s
    sm_mhz = clocks["sm_mhz"] or 1965.0
    nsm = torch.cuda.get_device_properties(local).multi_processor_count
    peak_gops = nsm * 128 * sm_mhz * 1e6 / 1e9
    ach_gops = OPS_PER_STEP * tot["steps"] / dev_s / 1e9
    line = {"metric": "TM steps/s", "value": value, "unit": "steps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot["dev_ms"] / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "int32+u64", "data": "synthetic (reference searches)",
            "leaves_per_s": tot["leaves"] / dev_s, "parity": parity,
            "config": {"workload": f"{args.workload}: {w['desc']}", "kernel": args.kernel,
                       "jobs": "concurrent in one persistent kernel" if kernel == E.KERNEL_PERSISTENT
                       else "one after another",
                       "leaves_per_step": w["leaves"], "l2": "flushed between steps (256 MiB write)",
                       "parallelism": f"X sharded over {ws} rank(s)"},
            "roofline": {"bound": "int-issue", "achieved": ach_gops, "peak": peak_gops, "unit": "Gop/s",
                         "frac": ach_gops / peak_gops, "traffic": PROFILED_TRAFFIC.get(args.workload),
                         "note": f"{OPS_PER_STEP} integer lane-ops per step; peak = {nsm} SMs x 128 lanes x "
                                 f"{sm_mhz:.0f} MHz (median SM clock sampled during the timed region)"},
            "e2e": {"value": tot["steps"] / tot["wall"], "unit": "steps/s",
                    "h2d_bytes_per_step": 288 * len(jobs) + 160 * len(jobs),
                    "d2h_bytes_per_step": tot["d2h"] // args.steps + 160 * len(jobs)},
            "gpu_launches": tot["launches"], "clocks": clocks,
            "kernel_stats": {"epochs": kstats["epochs"], "jobs_per_step": kstats["jobs"],
                             "note": "epochs over all warmup and timed steps"}}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        s, l, dt, kind = run_reference_cpu(WORKLOADS[CPU_SAMPLE], threads)
        line["cpu_baseline"] = {"value": s / dt, "unit": "steps/s", "cores": threads, "kind": kind,
                                "sample": WORKLOADS[CPU_SAMPLE]["desc"] + " (4.0e9 steps)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
