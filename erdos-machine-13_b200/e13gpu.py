"""Drop-in for the reference's GPU driver, `python src/e13gpu.py`, on B200.

    python erdos-machine-13_b200/e13gpu.py machine.txt X LO HI CELL...   (LO = -1: no symmetry)

The same command line, environment and text as src/e13gpu.py:293-465, with
the search run by libe13b200.so (the persistent kernel) instead of a CuPy
kernel:
  stdout   SURVIVOR lines in the C format (src/e13search.c:184-200)
  stderr   the start line, "resumed from ...", the summary
           "X=.. budget=0 gpu leaves=.. survivors=.. steps=.. wall=..s
           dead-at-stage(0..9): ..." and the "launches= peak stack=" line
  E13_CKPT, E13_CKPT_SEC, <E13_CKPT>.stop   checkpoints, clean stop (exit 3)
  E13_SLICE  iterations (of up to two actions per lane) between refill rounds
             (the kernel's slice)
  E13_DEVICE the CUDA device (default 0)

One difference: with X = -1 (nothing deleted) the reference driver renumbers
next states as if state 0 were deleted (`n - (n > X)`, src/e13gpu.py:76-77);
this follows e13search.c instead (`n - (X >= 0 && n > X)`,
src/e13search.c:329-330).  The reference's GPU runs all have X >= 0, where the
two agree.
"""
from __future__ import annotations

import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import e13b200 as E  # noqa: E402

NODE_BYTES = 320


def main(argv: list[str]) -> int:
    t0 = time.time()
    if len(argv) < 5:
        print("usage: e13gpu.py machine.txt X LO HI CELL...   (LO = -1: no symmetry)", file=sys.stderr)
        return 1
    path, X, lo, hi = argv[1], int(argv[2]), int(argv[3]), int(argv[4])
    cells = argv[5:]
    try:
        base = E.load_machine(path)
    except E.E13Error:
        print(f"cannot open {path}", file=sys.stderr)
        return 1
    r, job = E.setup(base, X, free_cells=cells, lo=lo, hi=hi)
    if r == -3:
        print("a symmetric state is named by a fixed cell or has one", file=sys.stderr)
        return 1
    if r == -4:
        print("start state in the symmetric states", file=sys.stderr)
        return 1
    if r:
        print(f"setup failed ({E.ERRORS.get(r, r)})", file=sys.stderr)
        return 1
    kw = {}
    if os.environ.get("E13_SLICE"):
        kw["slice"] = int(os.environ["E13_SLICE"])
    tune = E.tuning(**kw)
    ctx = E.Context(int(os.environ.get("E13_DEVICE", "0")))
    print(f"X={X} nq={job.nq} free={len(cells)} sym={job.sym_lo}..{job.sym_hi} n0={job.sym_n0} "
          f"node={NODE_BYTES}B block={tune.block}", file=sys.stderr, flush=True)
    ckpt = os.environ.get("E13_CKPT")
    if ckpt:
        if os.path.exists(ckpt):
            slot = open(ckpt).read().strip()
            print(f"resumed from {ckpt}.{slot}", file=sys.stderr, flush=True)
        config = " ".join(argv[2:]) + f" {os.path.basename(path)} NB={NODE_BYTES}"
        rc, counts, surv, wall, left = ctx.search_resumable(
            job, ckpt, config, interval_s=float(os.environ.get("E13_CKPT_SEC", "1800")), tune=tune)
        if rc == E.STOPPED:
            print(f"STOPPED cleanly at wall={wall:.0f}s steps={counts.steps:.3e} survivors={counts.survivors} "
                  f"stack={left}; run the same command to resume", file=sys.stderr, flush=True)
            return 3
    else:
        counts, surv = ctx.search(job, tune)
        wall = time.time() - t0
    st = ctx.stats()
    for s in surv:
        print(E.survivor_line(job, s))
    sys.stdout.flush()
    hist = " ".join(str(h) for h in counts.hist)
    print(f"X={X} budget=0 gpu leaves={counts.leaves} survivors={counts.survivors} steps={counts.steps} "
          f"wall={wall:.1f}s dead-at-stage(0..9): {hist}", file=sys.stderr)
    print(f"  launches={st.launches} peak stack={st.peak_nodes} nodes ({st.peak_nodes * NODE_BYTES / 1e9:.2f} GB) "
          f"{counts.steps / max(wall, 1e-9):.2e} steps/s", file=sys.stderr)
    if counts.survivors > len(surv):
        print(f"WARNING: {counts.survivors} survivors, only {len(surv)} printed", file=sys.stderr)
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
