"""The batched solver's step schedule (zolo_batch_schedule, host only) against PQDWHFACS's
loop control (pqdwhfacs.f90:359-372, restated by the oracle's _qdwh_loop): the weights of
every step bitwise equal to the oracle's qdwh_weights, each step's form the QR form exactly
when a member scheduled there has c > 100, and the unconditional steps plus the gated
conditional step reproducing the loop's iteration count for any error sequence."""
import math

import numpy as np
import pytest

import zolo_svd_b200 as zb
from oracle import zolo_oracle as zo

EPS = zo.EPS
TOL1 = 10.0 * EPS / 2.0
TOL2 = math.exp(math.log(TOL1) / 3.0)


def member_steps(l0, maxit=12):
    """The oracle loop's weights per step, stopping on L alone: (weights of the unconditional
    steps, weights of the conditional step or None)."""
    steps, l = [], l0
    while True:
        ak, bk, ck, l = zo.qdwh_weights(l)
        steps.append((ak, bk, ck))
        if len(steps) > maxit:
            return steps, None
        if not abs(1.0 - l) > TOL1:
            return steps, zo.qdwh_weights(l)[:3]


def expected_row(w, qr):
    ak, bk, ck = w
    sck = math.sqrt(ck)
    return (1.0 / sck if qr else ck), bk / ck, ((ak - bk / ck) / sck if qr else ak - bk / ck)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_schedule_matches_oracle_weights_and_forms(seed):
    rng = np.random.default_rng(seed)
    l0 = list(10 ** rng.uniform(-15, -0.3, 37)) + [1.0, 0.999999, 1e-16]
    S = zb.batch_schedule(l0)
    K = S["steps"]
    per = [member_steps(l) for l in l0]
    assert K == max(len(u) + (c is not None) for u, c in per)
    for b, (u, c) in enumerate(per):
        assert S["count"][b] == len(u)
        assert S["last"][b] == len(u) - 1
        assert S["cond"][b] == (len(u) if c is not None else -1)
    for k in range(K):
        ws = []
        for u, c in per:
            if k < len(u):
                ws.append(u[k])
            elif c is not None and k == len(u):
                ws.append(c)
        qr = any(w[2] > 100.0 for w in ws)
        assert S["qr"][k] == int(qr), k
        tab = S["table"][k]
        for b, (u, c) in enumerate(per):
            if k < len(u) or (c is not None and k == len(u)):
                w = u[k] if k < len(u) else c
                assert tuple(tab[:3, b]) == expected_row(w, qr), (k, b)  # bitwise
                assert tab[4, b] == (1.0 if k == len(u) else 0.0)
            else:
                assert tuple(tab[:3, b]) == ((1.0 if qr else 0.0), 1.0, 0.0)
            assert tab[3, b] == 0.0


def loop_count(l0, errs, maxit=12):
    """Iterations of the oracle loop's control for a member whose k-th step has error errs[k]."""
    it, l, err = 0, l0, 1.0
    while (it == 0 or err > TOL2 or abs(1.0 - l) > TOL1) and it <= maxit:
        l = zo.qdwh_weights(l)[3]
        err = errs[it]
        it += 1
    return it


@pytest.mark.parametrize("seed", [3, 4])
def test_gated_conditional_step_reproduces_loop_counts(seed):
    """For error sequences falling by 10^U[1, 6] per step from 10^U[-8, 0], the member's steps in
    the scheduled run (its unconditional steps, plus the conditional one when the error of its
    last unconditional step is above TOL1^(1/3), the gate's test) equal the loop's count
    whenever the loop stops within them; otherwise the solver continues in the loop."""
    rng = np.random.default_rng(seed)
    l0 = list(10 ** rng.uniform(-15, -0.3, 200))
    S = zb.batch_schedule(l0)
    matched = 0
    for b, l in enumerate(l0):
        errs = [10 ** rng.uniform(-8, 0)]
        for _ in range(20):
            errs.append(errs[-1] * 10 ** -rng.uniform(1, 6))
        cnt, cond = S["count"][b], S["cond"][b]
        took = cond >= 0 and errs[cnt - 1] > TOL2
        sched = cnt + took
        want = loop_count(l, errs)
        if want <= cnt + (cond >= 0):
            assert sched == want, (b, sched, want)
            matched += 1
        else:  # the continuation case: the error is still high after the conditional step
            assert took and errs[cnt] > TOL2
    assert matched >= 150


def test_schedule_edge_members():
    """Members with no valid bound take no step; an empty bucket has no steps; a too small
    max_steps reports the needed count."""
    S = zb.batch_schedule([0.5, 0.0, float("nan"), 2.0])
    assert S["count"][1:] == [0, 0, 0] and S["last"][1:] == [-1, -1, -1] and S["cond"][1:] == [-1, -1, -1]
    assert S["count"][0] >= 1
    assert zb.batch_schedule([])["steps"] == 0
    import ctypes as C
    l = (C.c_double * 1)(1e-10)
    steps = C.c_int()
    assert zb.lib().zolo_batch_schedule(1, l, 12, 1, C.byref(steps), None, None, None, None, None) == -4
    assert steps.value > 1
