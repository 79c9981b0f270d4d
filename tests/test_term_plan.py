"""The term plan's host logic (ZOLO_OPT_TERM_PLAN, zolo_plan_terms; no GPU): the plans the
GPU runs take at n = 8192 for the bench's condition numbers, and invariants over a grid of
CON, rk and shapes (terms within 1..rk, the QR form only while CON > 12 and never after a
Cholesky-form iteration, a few iterations to convergence)."""
import pytest

import zolo_svd_b200 as zb


@pytest.mark.parametrize("con,plan,ns", [
    (1.41e14, [(4, "QR"), (1, "CH"), (4, "CH")], 0),   # kappa = 1e12, Frobenius beta
    (2.88e8, [(3, "QR"), (3, "CH")], 2),                # kappa = 1e6
    (8.83e4, [(2, "QR"), (5, "CH")], 1),                # kappa = 1e2
    (1.0, [], 0),
])
def test_plans_at_n8192(con, plan, ns):
    assert zb.plan_terms(con, 8, 8192, 8192) == (plan, ns)


@pytest.mark.parametrize("rk", [1, 2, 3, 5, 8])
@pytest.mark.parametrize("mn", [(512, 512), (8192, 8192), (16384, 8192)])
def test_plan_invariants(rk, mn):
    m, n = mn
    for e in range(0, 21):
        con = 1.5 * 10.0 ** e
        plan, ns = zb.plan_terms(con, rk, m, n)
        assert 1 <= len(plan) <= 8
        assert all(1 <= r <= rk for r, _ in plan)
        forms = [f for _, f in plan]
        # QR while CON > 12, then Cholesky: never QR after a Cholesky-form iteration
        assert forms == sorted(forms, key=lambda f: f == "CH")
        assert (forms[0] == "QR") == (con > 12)
        assert 0 <= ns <= 12
        if rk == 1:
            assert all(r == 1 for r, _ in plan)


def test_plan_rejects_bad_arguments():
    with pytest.raises(zb.ZoloError):
        zb.plan_terms(10.0, 9, 100, 100)
    with pytest.raises(zb.ZoloError):
        zb.plan_terms(10.0, 8, 50, 100)
    with pytest.raises(zb.ZoloError):
        zb.plan_terms(0.5, 8, 100, 100)
