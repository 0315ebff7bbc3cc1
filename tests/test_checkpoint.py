"""The binomial checkpoint plan behind dgb_forward_record / dgb_backward, on
the CPU: replaying the plan on step indices must reverse every step exactly
once, in order, each time with the right state in the work buffer, never use
more buffers than allowed, and recompute exactly the minimal number of steps
(a brute-force dynamic programme over all split points for small cases, the
closed form for large ones)."""
from functools import lru_cache
from math import comb

import pytest

import dgpr_b200 as dg


@lru_cache(None)
def dp_cost(t, f):
    if t <= 1:
        return 0
    if f == 0:
        return t * (t - 1) // 2
    return min(m + dp_cost(t - m, f - 1) + dp_cost(m, f) for m in range(1, t))


def closed_cost(t, f):
    if t <= 1:
        return 0
    s = f + 1
    r = 0
    while comb(s + r, s) < t:
        r += 1
    return r * t - comb(s + r, s + 1)


def replay(nsteps, slots):
    ops, forward, peak = dg.checkpoint_plan(nsteps, slots)
    nbuf = min(slots, nsteps)
    bufs = {}
    work = 0
    reversed_steps = []
    advanced = 0
    first_rev = next(k for k, (kind, _) in enumerate(ops) if kind == "reverse")
    assert ops[0] == ("store", 0)
    for k, (kind, arg) in enumerate(ops):
        if kind == "store":
            assert 0 <= arg < nbuf
            bufs[arg] = work
        elif kind == "restore":
            assert k > first_rev, "the recorded forward run never restores"
            assert arg in bufs
            work = bufs[arg]
        elif kind == "forward":
            assert arg >= 1
            work += arg
            advanced += arg
            assert work <= nsteps - 1
        else:
            if k == first_rev:
                assert work == nsteps - 1
            assert arg == work, "reverse step i needs U_i in the work buffer"
            reversed_steps.append(arg)
    assert reversed_steps == list(range(nsteps - 1, -1, -1))
    assert advanced == forward
    assert peak <= nbuf and len(bufs) <= nbuf
    return forward, peak


@pytest.mark.parametrize("nsteps", [1, 2, 3, 5, 8, 13, 21, 40, 64])
@pytest.mark.parametrize("slots", [1, 2, 3, 4, 6, 100])
def test_plan_is_valid_and_minimal(nsteps, slots):
    forward, _ = replay(nsteps, slots)
    assert forward == dp_cost(nsteps, min(slots, nsteps) - 1)


@pytest.mark.parametrize("nsteps,slots", [(400, 10), (400, 20), (1000, 12), (500, 3), (400, 400)])
def test_plan_at_adjoint_horizons(nsteps, slots):
    forward, peak = replay(nsteps, slots)
    assert forward == closed_cost(nsteps, min(slots, nsteps) - 1)
    if slots >= nsteps:
        assert forward == nsteps - 1 and peak == nsteps


def test_closed_form_matches_dynamic_programme():
    for f in range(0, 6):
        for t in range(1, 90):
            assert closed_cost(t, f) == dp_cost(t, f), (t, f)


def test_bad_arguments():
    with pytest.raises(dg.DgbError):
        dg.checkpoint_plan(0, 3)
    with pytest.raises(dg.DgbError):
        dg.checkpoint_plan(10, 0)
