"""Makes tests/golden/raw_1e6.json: the whole raw-simulator set (1e6 random
13-state tables drawn from seed 0, at most 2^18 steps each) run through the
reference's own step loop, run() of src/e13search.c, by oracle/_ref/ref_raw
(built by ``make -C oracle ref`` from the reference source; see
oracle/ref_raw.c for how the filter is switched off from outside).

    python tests/golden/make_raw_golden.py

The fixture holds aggregates of the per-machine results (steps, status, final
head, ones): total steps, machines by status, a histogram of final heads by
status, sums, and an order-dependent checksum (raw_checksum below) that the GPU
test recomputes from the device's per-machine output.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_RAW = os.path.join(ROOT, "oracle", "_ref", "ref_raw")
N, NQ, MAX_STEPS, SEED = 1_000_000, 13, 1 << 18, 0


def raw_checksum(out: np.ndarray) -> int:
    """Order-dependent 64-bit checksum of per-machine rows (steps, status,
    head, ones): sum over m of a splitmix64 finaliser of (m, row), mod 2^64."""
    out = np.asarray(out, dtype=np.int64).reshape(-1, 4).astype(np.uint64)
    m = np.arange(out.shape[0], dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (m * np.uint64(0x9E3779B97F4A7C15) + out[:, 0] * np.uint64(0xBF58476D1CE4E5B9) +
             out[:, 1] * np.uint64(0x94D049BB133111EB) + out[:, 2] * np.uint64(0xD6E8FEB86659FD93) +
             out[:, 3] * np.uint64(0xA0761D6478BD642F))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
        return int(z.sum(dtype=np.uint64))


def aggregates(out: np.ndarray) -> dict:
    out = np.asarray(out, dtype=np.int64).reshape(-1, 4)
    by_status = {str(s): int((out[:, 1] == s).sum()) for s in (0, 1, 2)}
    heads = {}
    for s in (0, 1, 2):
        sel = out[out[:, 1] == s, 2]
        vals, cnt = np.unique(sel, return_counts=True)
        # final heads of machines that stop in the window spread over it; bucket them by 64 cells
        if s == 0:
            b, c = np.unique((sel + 64) // 64, return_counts=True)
            heads[str(s)] = {str(int(k)): int(v) for k, v in zip(b, c)}
        else:
            heads[str(s)] = {str(int(k)): int(v) for k, v in zip(vals, cnt)}
    return {"machines": int(out.shape[0]), "total_steps": int(out[:, 0].sum()), "by_status": by_status,
            "head_hist_by_status": heads, "sum_head": int(out[:, 2].sum()), "sum_ones": int(out[:, 3].sum()),
            "checksum": raw_checksum(out)}


def run_chunk(m0: int, n: int) -> np.ndarray:
    p = subprocess.run([REF_RAW, str(SEED), str(m0), str(n), str(NQ), str(MAX_STEPS)], capture_output=True,
                       check=True)
    return np.frombuffer(p.stdout, dtype=np.int64).reshape(-1, 4)


def main():
    if not os.path.exists(REF_RAW):
        sys.exit("oracle/_ref/ref_raw missing: run make -C oracle ref where the reference is checked out")
    chunk = 25_000
    starts = list(range(0, N, chunk))
    with ThreadPoolExecutor(os.cpu_count() or 4) as ex:
        parts = list(ex.map(lambda m0: run_chunk(m0, min(chunk, N - m0)), starts))
    out = np.concatenate(parts)
    agg = aggregates(out)
    agg.update({"seed": SEED, "nq": NQ, "max_steps": MAX_STEPS,
                "source": "oracle/_ref/ref_raw: run() of src/e13search.c with the filter switched off"})
    with open(os.path.join(HERE, "raw_1e6.json"), "w") as f:
        json.dump(agg, f, indent=1, sort_keys=True)
    print(json.dumps({k: agg[k] for k in ("machines", "total_steps", "by_status", "checksum")}))


if __name__ == "__main__":
    main()
