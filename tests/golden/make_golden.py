"""Makes the golden fixtures under tests/golden/ from the reference project.

Run in a container that has the reference checked out (default
/root/reference) and, for the step counts that older logs lack, the reference
binaries built by ``make -C oracle ref`` (oracle/_ref/e13search):

    python tests/golden/make_golden.py [REFERENCE_DIR]

Outputs (all small text / gzip files, committed):
  machines/...             the machine tables the searches start from
  searches.json            per search: command, per-X expected counts
                           (leaves, survivors, steps when known, deaths per
                           stage), survivor file, source log
  surv/*.txt(.gz)          sorted SURVIVOR lines of each search
  recheck_1RD.json.gz      recheck.c 15 verdicts for the 2868 V1 survivors
  deep/*.txt(.gz)          deep.c outputs (V1 at 15, V2, erdos_14)
  mutants.txt              e13search mutant on erdos_14
  base_erdos14.txt         e13search base on erdos_14
  check/*.txt              src/check.py's shipped outputs (the survivor line,
                           then one "halt@<place>: PASS|FAIL ..." line per
                           placement), copied from the reference's results
  estimate_ref.json        e13search estimate printed by the reference binary
                           on one OpenMP thread (so every probe draws from
                           thread 0's stream, in order): args, E13_SEED and
                           the four result lines

``python tests/golden/make_golden.py [REFERENCE_DIR] estimates`` remakes only
estimate_ref.json, ``... checks`` only check/.

Every number comes from the reference's own result logs except the step
counts marked "steps_source": "reference binary" -- those were printed by the
reference e13search.c compiled here from its own source and run on the same
arguments (its logs for those searches predate the steps= field).
"""
from __future__ import annotations

import gzip
import json
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
ARGS = [a for a in sys.argv[1:] if a not in ("estimates", "checks")]
REF = ARGS[0] if ARGS else os.environ.get("E13_REF", "/root/reference")
RES = os.path.join(REF, "results")
REFBIN = os.path.join(REPO, "oracle", "_ref", "e13search")

SUMMARY_RE = re.compile(
    r"X=(-?\d+) .*?leaves=(\d+) survivors=(\d+)(?: steps=(\d+))?.*?dead-at-stage\(0\.\.9\):((?: \d+){10})")
ERDOS14 = "erdos_14.txt"
DIV = ["D0", "D1", "E0", "E1", "F0", "F1", "G0", "G1", "H0", "H1", "I0", "I1"]


def summaries(path):
    out = []
    for line in open(path):
        m = SUMMARY_RE.search(line)
        if m and "leaves=" in line and "dead-at-stage" in line:
            out.append(dict(X=int(m.group(1)), leaves=int(m.group(2)), survivors=int(m.group(3)),
                            steps=int(m.group(4)) if m.group(4) else None,
                            hist=[int(x) for x in m.group(5).split()]))
    return out


def survivor_lines(path, strip_prefix=False):
    lines = []
    for line in open(path):
        line = line.rstrip("\n")
        if "SURVIVOR" not in line:
            continue
        if strip_prefix:
            line = line[line.index("SURVIVOR"):]
        lines.append(line)
    return sorted(lines)


def write_surv(name, lines):
    os.makedirs(os.path.join(HERE, "surv"), exist_ok=True)
    body = "".join(l + "\n" for l in lines)
    if len(body) > 16000:
        fn = name + ".txt.gz"
        with gzip.open(os.path.join(HERE, "surv", fn), "wt") as f:
            f.write(body)
    else:
        fn = name + ".txt"
        with open(os.path.join(HERE, "surv", fn), "w") as f:
            f.write(body)
    return "surv/" + fn


def ref_steps(args):
    """Per-X step counts printed by the reference binary on these args."""
    if not os.path.exists(REFBIN):
        return None
    r = subprocess.run([REFBIN] + args, capture_output=True, text=True, check=True,
                       env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count())))
    return {s["X"]: s["steps"] for s in summaries_from_text(r.stderr)}


def summaries_from_text(text):
    out = []
    for line in text.splitlines():
        m = SUMMARY_RE.search(line)
        if m:
            out.append(dict(X=int(m.group(1)), steps=int(m.group(4)) if m.group(4) else None))
    return out


ESTIMATE_CASES = [
    (["estimate", ERDOS14, "2000", "8", "2", "-1", "-1"], 0),
    (["estimate", ERDOS14, "1000", "11", "3", "-1", "-1"], 0),
    (["estimate", ERDOS14, "3000", "13", "0", "10", "13", "D0", "G0", "K0", "K1", "L1", "M1"], 7),
    (["estimate", ERDOS14, "2000", "13", "0", "-1", "-1", "D0", "G0", "K0", "K1", "L1", "M1"], 3),
]


CHECK_FILES = {
    "erdos14.txt": "validation/check_erdos14.txt",
    "f4_unread.txt": "1_local_edits/check_f4_unread.txt",
    "counter_plus_f2.txt": "5_counter_plus/f2_f3/check_f2.txt",
    "counter_plus_f3.txt": "5_counter_plus/f2_f3/check_f3.txt",
    "counter_plus_cx.txt": "5_counter_plus/extra_cell/check_cx.txt",
    "division_v2.txt": "4_division_6/v2/check_v2.txt",
}


def check_outputs():
    """check.py's outputs as the reference ships them (comment lines dropped)."""
    os.makedirs(os.path.join(HERE, "check"), exist_ok=True)
    for name, src in CHECK_FILES.items():
        with open(os.path.join(RES, src)) as f, open(os.path.join(HERE, "check", name), "w") as g:
            for line in f:
                if not line.startswith("#"):
                    g.write(line)


def estimates():
    """The reference's estimate mode (src/e13search.c:473-510) on one thread."""
    out = []
    for args, seed in ESTIMATE_CASES:
        run = [REFBIN, args[0], os.path.join(HERE, "machines", args[1])] + args[2:]
        r = subprocess.run(run, capture_output=True, text=True, check=True,
                           env=dict(os.environ, OMP_NUM_THREADS="1", E13_SEED=str(seed)))
        lines = r.stdout.splitlines()
        head = re.sub(r" wall=\S+", "", lines[0])
        out.append(dict(args=args, seed=seed, threads=1, header=head, lines=lines[1:5]))
    with open(os.path.join(HERE, "estimate_ref.json"), "w") as f:
        json.dump(out, f, indent=1)


def main():
    # machine tables
    mdir = os.path.join(HERE, "machines")
    os.makedirs(os.path.join(mdir, "counters_3state"), exist_ok=True)
    for fn in ["erdos_14.txt", "split_15.txt", "c0_0LD.txt", "c0_1LD.txt", "c0_1RD.txt"]:
        shutil.copy(os.path.join(REF, "machines", fn), os.path.join(mdir, fn))
    for fn in sorted(os.listdir(os.path.join(REF, "machines", "counters_3state"))):
        shutil.copy(os.path.join(REF, "machines", "counters_3state", fn), os.path.join(mdir, "counters_3state", fn))

    searches = []

    def add(name, mode, machine, per_x, src, surv=None, fmax=None, X=None, free=None, lo=-1, hi=-1,
            steps_source="log", note=None):
        e = dict(name=name, mode=mode, machine=machine, fmax=fmax, X=X, free=free, lo=lo, hi=hi, expect=per_x,
                 source=src, steps_source=steps_source)
        if surv is not None:
            e["survivors_file"] = surv
        if note:
            e["note"] = note
        e["leaves_total"] = sum(p["leaves"] for p in per_x)
        searches.append(e)

    # 1. local edits, FMAX = 2, 3, 4 (delete mode, X = 0..13)
    for fmax in (2, 3, 4):
        s = summaries(os.path.join(RES, "1_local_edits", f"log_f{fmax}.txt"))
        s.sort(key=lambda d: d["X"])
        src = "steps: none"
        if fmax <= 3:
            st = ref_steps(["delete", os.path.join(REF, "machines", ERDOS14), str(fmax)] +
                           [str(x) for x in range(14)])
            if st:
                for d in s:
                    d["steps"] = st[d["X"]]
                src = "reference binary"
        surv = write_surv(f"f{fmax}", survivor_lines(os.path.join(RES, "1_local_edits", f"surv_f{fmax}.txt")))
        add(f"local_edits_f{fmax}", "delete", ERDOS14, s, f"results/1_local_edits/log_f{fmax}.txt", surv, fmax=fmax,
            X=list(range(14)), steps_source=src)

    # 2. counter in 3 states, with and without symmetry
    s = summaries(os.path.join(RES, "2_counter_3", "log_modsym.txt"))
    surv = write_surv("counter_sym", survivor_lines(os.path.join(RES, "2_counter_3", "surv_modsym.txt")))
    add("counter_sym", "freesym", ERDOS14, s, "results/2_counter_3/log_modsym.txt", surv, X=13,
        free=["D0", "G0", "K0", "K1", "L1", "M1"], lo=10, hi=13)
    s = summaries(os.path.join(RES, "2_counter_3", "log_mod.txt"))
    surv = write_surv("counter_nosym", survivor_lines(os.path.join(RES, "2_counter_3", "surv_mod.txt")))
    add("counter_nosym", "free", ERDOS14, s, "results/2_counter_3/log_mod.txt", surv, X=13,
        free=["D0", "G0", "K0", "K1", "L1", "M1"], steps_source="none")

    # 3. doubling in 2 states
    for X, free in ((0, ["B0", "B1", "C0", "C1"]), (1, ["A0", "A1", "C0", "C1"]), (2, ["A0", "A1", "B0", "B1"])):
        s = summaries(os.path.join(RES, "3_doubling_2", f"dbl_X{X}.log"))
        add(f"doubling_X{X}", "free", ERDOS14, s, f"results/3_doubling_2/dbl_X{X}.log", X=X, free=free)

    # 4. division in 6 states
    s = summaries(os.path.join(RES, "4_division_6", "v4", "log_v4.txt"))
    add("division_v4", "freesym", ERDOS14, s, "results/4_division_6/v4/log_v4.txt", X=9, free=DIV[4:], lo=3, hi=9)
    s = summaries(os.path.join(RES, "4_division_6", "v3", "log_v3.txt"))
    add("division_v3", "freesym", ERDOS14, s, "results/4_division_6/v3/log_v3.txt", X=9, free=DIV[2:], lo=3, hi=9)
    s = summaries(os.path.join(RES, "4_division_6", "v2", "log_v2.txt"))[-1:]
    surv = write_surv("division_v2", survivor_lines(os.path.join(RES, "4_division_6", "v2", "surv_v2.txt")))
    add("division_v2", "freesym", ERDOS14, s, "results/4_division_6/v2/log_v2.txt", surv, X=9, free=DIV, lo=3, hi=9)
    for c0 in ("1RD", "1LD", "0LD"):
        s = summaries(os.path.join(RES, "4_division_6", "v1", f"log_{c0}.txt"))[-1:]
        surv = None
        if c0 == "1RD":
            surv = write_surv("division_v1_1RD", survivor_lines(os.path.join(RES, "4_division_6", "v1", "surv_1RD.txt")))
        add(f"division_v1_{c0}", "freesym", f"c0_{c0}.txt", s, f"results/4_division_6/v1/log_{c0}.txt", surv, X=9,
            free=DIV, lo=3, hi=9)

    # 5a. around each three-state counter, X = -1, FMAX = 2 and 3
    for fmax in (2, 3):
        s = summaries(os.path.join(RES, "5_counter_plus", "f2_f3", f"log_f{fmax}_all.txt"))
        for k, d in enumerate(s):
            add(f"counters_f{fmax}_base_{k + 1:02d}", "delete", f"counters_3state/base_{k + 1:02d}.txt", [d],
                f"results/5_counter_plus/f2_f3/log_f{fmax}_all.txt (line {k + 1} of the summaries)", fmax=fmax,
                X=[-1])
    # 5b. counter + one more cell
    for extra in ("C1", "D1", "C0", "G1"):
        s = summaries(os.path.join(RES, "5_counter_plus", "extra_cell", f"log_cx_{extra}.txt"))[-1:]
        surv = write_surv(f"counter_plus_{extra}",
                          survivor_lines(os.path.join(RES, "5_counter_plus", "extra_cell", f"surv_cx_{extra}.txt")))
        add(f"counter_plus_{extra}", "freesym", ERDOS14, s, f"results/5_counter_plus/extra_cell/log_cx_{extra}.txt",
            surv, X=13, free=["K0", "K1", "L0", "L1", "M0", "M1", "D0", "G0", extra], lo=10, hi=13)

    # split tests (validation)
    s = summaries(os.path.join(RES, "validation", "split_test.txt"))
    surv = write_surv("split_test", survivor_lines(os.path.join(RES, "validation", "split_test.txt")))
    add("split_test", "delete", "split_15.txt", s, "results/validation/split_test.txt", surv, fmax=1, X=[14])
    s = summaries(os.path.join(RES, "validation", "split_test_free.txt"))
    surv = write_surv("split_test_free", survivor_lines(os.path.join(RES, "validation", "split_test_free.txt")))
    add("split_test_free", "free", "split_15.txt", s, "results/validation/split_test_free.txt", surv, X=14,
        free=["K0", "K1", "L1"])

    with open(os.path.join(HERE, "searches.json"), "w") as f:
        json.dump(searches, f, indent=1)

    # recheck.c 15 verdicts for the 2868 V1 survivors (ids restart per chunk)
    verdicts = []
    for line in open(os.path.join(RES, "validation", "recheck_1RD.txt")):
        if line.startswith("#"):
            continue
        m = re.match(r"(\d+): (.*)$", line.rstrip("\n"))
        if m:
            verdicts.append(m.group(2))
    with gzip.open(os.path.join(HERE, "recheck_1RD.json.gz"), "wt") as f:
        json.dump(dict(nmax=15, survivors="surv/division_v1_1RD.txt.gz (in file order of results/4_division_6/"
                                            "v1/surv_1RD.txt)", verdicts=verdicts), f)
    # the recheck order is the file order of surv_1RD.txt, not the sorted one
    with gzip.open(os.path.join(HERE, "surv", "division_v1_1RD_fileorder.txt.gz"), "wt") as f:
        for line in open(os.path.join(RES, "4_division_6", "v1", "surv_1RD.txt")):
            if "SURVIVOR" in line:
                f.write(line)
    with open(os.path.join(HERE, "surv", "division_v2_fileorder.txt"), "w") as f:
        for line in open(os.path.join(RES, "4_division_6", "v2", "surv_v2.txt")):
            if "SURVIVOR" in line:
                f.write(line)

    os.makedirs(os.path.join(HERE, "deep"), exist_ok=True)
    with gzip.open(os.path.join(HERE, "deep", "deep15_1RD.txt.gz"), "wt") as f:
        f.write(open(os.path.join(RES, "4_division_6", "v1", "deep15_1RD.txt")).read())
    shutil.copy(os.path.join(RES, "4_division_6", "v2", "deep_v2.txt"), os.path.join(HERE, "deep", "deep_v2.txt"))
    shutil.copy(os.path.join(RES, "validation", "deep_base14.txt"), os.path.join(HERE, "deep", "deep_base14.txt"))
    shutil.copy(os.path.join(RES, "validation", "mutants.txt"), os.path.join(HERE, "mutants.txt"))
    shutil.copy(os.path.join(RES, "validation", "base_erdos14.txt"), os.path.join(HERE, "base_erdos14.txt"))
    check_outputs()
    print(f"{len(searches)} searches, {len(verdicts)} recheck verdicts")


if __name__ == "__main__":
    if "estimates" in sys.argv[1:]:
        estimates()
    elif "checks" in sys.argv[1:]:
        check_outputs()
    else:
        main()
        estimates()
