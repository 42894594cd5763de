"""Makes tests/golden/recheck15_counter_sym.txt: the reference recheck's
verdicts (src/recheck.c, stage limit NMAX = 15) on the 61 survivors of the
3-state counter search with symmetry (freesym erdos_14 13 10 13 D0 G0 K0 K1
L1 M1), in the order of the sorted SURVIVOR lines of surv/counter_sym.txt.

The reference's recheck takes about 330 s on one core for these machines, so
the lines go to it in 16 chunks run side by side; each chunk numbers its
machines from 1 again, and this script numbers them through.  Needs the
reference binary built by ``make -C oracle ref`` (oracle/_ref/recheck).

    python tests/golden/make_pipeline_golden.py
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
RECHECK = os.path.join(ROOT, "oracle", "_ref", "recheck")
NMAX = 15


def main():
    with open(os.path.join(HERE, "surv", "counter_sym.txt")) as f:
        lines = sorted(l.rstrip("\n") for l in f if l.strip())
    chunks = [lines[i::16] for i in range(16)]

    def run(chunk):
        r = subprocess.run([RECHECK, str(NMAX)], input="\n".join(chunk) + "\n", capture_output=True, text=True,
                           check=True)
        return [l.split(": ", 1)[1] for l in r.stdout.splitlines() if ": " in l]

    with ThreadPoolExecutor(16) as ex:
        outs = list(ex.map(run, chunks))
    verdicts = [None] * len(lines)
    for i, out in enumerate(outs):
        assert len(out) == len(chunks[i])
        for j, v in enumerate(out):
            verdicts[i + 16 * j] = v
    with open(os.path.join(HERE, f"recheck{NMAX}_counter_sym.txt"), "w") as f:
        for k, v in enumerate(verdicts):
            f.write(f"{k + 1}: {v}\n")
    print(f"{len(verdicts)} verdicts", file=sys.stderr)


if __name__ == "__main__":
    main()
