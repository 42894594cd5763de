"""e13_check_noalloc(): the deep check for callers that cannot allocate device
memory (their GPU memory belongs to another allocator, or they cannot afford
cudaMalloc's implicit synchronisation).  Its output must equal e13_check's
(integer results, so exactly) on two calls in a row, which also shows that the
fixed arrays it reuses are cleared between calls.  Kept in its own file so it
is collected last."""
import gzip
import os

import pytest

import e13b200 as E

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _survivors(k, start):
    with gzip.open(os.path.join(GOLD, "surv", "division_v1_1RD_fileorder.txt.gz"), "rt") as f:
        lines = [l for l in f if l.strip()]
    return [E.parse_survivor_line(l) for l in lines[start:start + k]]


def _same(a, b):
    return bytes(a) == bytes(b)


@pytest.mark.parametrize("mode", [0, 1])
def test_noalloc_check_matches_e13_check_twice(mode):
    ctx = E.Context(0)
    for call, start in enumerate((0, 500)):  # two calls in a row, different machines
        ins = _survivors(E.E13_CHECK_NOALLOC_MAX, start)
        ref = ctx.check(ins, 12, mode)
        got = E.check_noalloc(0, ins, 12, mode)
        assert all(_same(a, b) for a, b in zip(ref, got)), (mode, call)
        assert all(E.format_recheck(o, 12) == E.format_recheck(r, 12) for o, r in zip(got, ref))
    ctx.close()


def test_noalloc_rejects_too_many_machines():
    ins = _survivors(E.E13_CHECK_NOALLOC_MAX + 1, 0)
    with pytest.raises(E.E13Error) as ei:
        E.check_noalloc(0, ins, 12, 0)
    assert ei.value.code == -12
