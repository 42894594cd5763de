"""Parity of the CUDA search with the reference's larger result logs: the
routine cases of the counter (cfg 2) and division (cfg 3) families that fit a
test run on one B200.

  division V3      freesym erdos_14 9 3 9 E0..I1   53,282,072,641 leaves, 0 survivors
                   (results/4_division_6/v3/log_v3.txt:1)
  counter, no sym  free erdos_14 13 D0 G0 K0 K1 L1 M1   18,471,584,227 leaves, 366 survivors
                   (results/2_counter_3/log_mod.txt:1, surv_mod.txt)
  counter + C1     freesym erdos_14 13 10 13 K0..M1 D0 G0 C1   90,976,928,448 leaves, 61 survivors
                   (results/5_counter_plus/extra_cell/log_cx_C1.txt, surv_cx_C1.txt)
  61 x FMAX 2 / 3  the neighbourhoods of the 61 three-state counters
                   (results/5_counter_plus/f2_f3/log_f{2,3}_all.txt)

and the survivor pipeline on the device: the counter search's survivors,
as the search returns them, go straight into the hash-free deep check to
stage 15, whose verdicts must equal the reference recheck's
(golden/recheck15_counter_sym.txt, made by make_pipeline_golden.py).
"""
import os

import pytest

import e13b200 as E
from gpu_common import GOLD, check_entry, ctx, golden_lines, make_job, run_entry

pytestmark = pytest.mark.gpu

KERNELS = {"plain": E.KERNEL_PLAIN, "persistent": E.KERNEL_PERSISTENT}


@pytest.mark.slow
@pytest.mark.parametrize("kernel", list(KERNELS))
def test_division_v3(searches, kernel):
    e = searches["division_v3"]
    per_x, lines = run_entry(e, E.tuning(kernel=KERNELS[kernel]))
    check_entry(e, per_x)
    assert lines == []


@pytest.mark.slow
def test_counter_no_symmetry(searches):
    e = searches["counter_nosym"]
    per_x, lines = run_entry(e, E.tuning(kernel=E.KERNEL_PERSISTENT))
    check_entry(e, per_x)
    assert len(lines) == 366
    assert lines == golden_lines(e)


@pytest.mark.slow
def test_counter_plus_c1(searches):
    e = searches["counter_plus_C1"]
    per_x, lines = run_entry(e, E.tuning(kernel=E.KERNEL_PERSISTENT))
    check_entry(e, per_x)
    assert lines == golden_lines(e)


@pytest.mark.parametrize("kernel", list(KERNELS))
def test_counter_neighbourhoods_f2(searches, kernel):
    """All 61 FMAX = 2 neighbourhoods: leaves, survivors, steps and deaths by
    stage of each equal its line of log_f2_all.txt."""
    names = sorted(n for n in searches if n.startswith("counters_f2_base_"))
    assert len(names) == 61
    for n in names:
        per_x, _ = run_entry(searches[n], E.tuning(kernel=KERNELS[kernel]))
        check_entry(searches[n], per_x)


def test_counter_neighbourhoods_f3(searches):
    """All 61 FMAX = 3 neighbourhoods (4.15e11 steps) against log_f3_all.txt."""
    names = sorted(n for n in searches if n.startswith("counters_f3_base_"))
    assert len(names) == 61
    for n in names:
        per_x, _ = run_entry(searches[n], E.tuning(kernel=E.KERNEL_PERSISTENT))
        check_entry(searches[n], per_x)


@pytest.mark.slow
def test_counter_search_feeds_the_deep_check(searches):
    """Enumeration feeding the deep check: the 61 survivors of the counter
    search with symmetry, taken from e13_search's records with
    e13_survivor_check_in (no text in between), are rechecked on the device
    to stage 15; the verdicts, in sorted survivor-line order, equal the
    reference recheck's on the reference's survivor file."""
    e = searches["counter_sym"]
    job = make_job(e, 13)
    c, surv = ctx().search(job, E.tuning(kernel=E.KERNEL_PERSISTENT))
    assert c.survivors == 61 and len(surv) == 61
    pairs = sorted((E.survivor_line(job, s), s) for s in surv)
    assert [l for l, _ in pairs] == golden_lines(e)
    outs = ctx().check([E.survivor_check_in(job, s) for _, s in pairs], 15, 0)  # mode 0: recheck.c
    got = [f"{k + 1}: {E.format_recheck(o, 15)}" for k, o in enumerate(outs)]
    with open(os.path.join(GOLD, "recheck15_counter_sym.txt")) as f:
        assert got == f.read().splitlines()
