"""Pipelined state evaluations (btam_mf_eval_state_async / _wait) against
the one-call form btam_mf_eval_state.

Tolerance: none.  The pipelined call runs the same update and evaluation
kernels on the same stream as btam_mf_eval_state; only the copies move to
the copy streams and through the call's device slot.  So every result of a
sequence of states must equal, bit for bit, the one-call result of the same
state, whether the calls overlap or not; a rejected state must give the
one-call status and leave the state as the one-call form does."""
import numpy as np
import pytest
import torch

import btam
from btam import lattice

pytestmark = pytest.mark.gpu
KEYS = ("rho", "V0", "S0", "Rq", "Rs", "Rx", "totals")


def pinned(shape):
    return torch.zeros(shape, dtype=torch.float64).pin_memory().numpy()


def states(s, k, seed=3):
    g = np.random.default_rng(seed)
    for _ in range(k):
        yield (s["q"] + g.normal(0.0, 0.01, s["q"].shape),
               s["sigma"] * g.uniform(0.95, 1.05, s["sigma"].shape),
               np.where(s["species"] == 1, np.clip(s["x"] + g.normal(0, 0.02, s["x"].shape),
                                                   0.0, 0.9), s["x"]))


def system():
    # a free cluster: moved sites never leave a periodic cell
    return lattice.sphere(11.0, T=400.0, h_fraction=0.4, seed=17)


@pytest.mark.parametrize("prec", [btam.FP64, btam.FP32C])
def test_pipelined_states_equal_one_call_form(gpu_tables, prec):
    s = system()
    n = len(s["x"])
    A = btam.System(gpu_tables, s)
    B = btam.System(gpu_tables, s)
    for S in (A, B):
        S.build_neighbors()
        S.set_variants(prec, 16 | 8 | 3, 16 | 8 | 3)
    seq = list(states(s, 7))
    want = [B.evaluate_state(prec, q=q, sigma=sg, x=x) for q, sg, x in seq]
    shapes = dict(rho=(n,), V0=(n,), S0=(n,), Rq=(n, 3), Rs=(n,), Rx=(n,), totals=(4,))
    bufs = [{k: pinned(v) for k, v in shapes.items()} for _ in range(2)]
    got, tickets = [], []
    for k, (q, sg, x) in enumerate(seq):
        tickets.append(A.evaluate_state_async(prec, q=q, sigma=sg, x=x, out=bufs[k % 2]))
        if k >= 1:  # two in flight: wait for the previous one, then keep its results
            A.wait_state(tickets[k - 1])
            got.append({key: v.copy() for key, v in bufs[(k - 1) % 2].items()})
    A.wait_state(tickets[-1])
    got.append({key: v.copy() for key, v in bufs[(len(seq) - 1) % 2].items()})
    for k in range(len(seq)):
        for key in KEYS:
            assert np.array_equal(got[k][key], want[k][key]), (k, key)
    # a ticket is waited for once
    with pytest.raises(btam.BtamError):
        A.wait_state(tickets[0])


def test_third_call_retires_the_first_and_keeps_its_status(gpu_tables):
    s = system()
    S = btam.System(gpu_tables, s)
    S.build_neighbors()
    q0 = s["q"].copy()
    bad = q0.copy()
    bad[3, 1] = np.nan
    outs = [dict(totals=np.zeros(4)) for _ in range(3)]
    t1 = S.evaluate_state_async(btam.FP64, q=bad, out=outs[0])       # rejected
    t2 = S.evaluate_state_async(btam.FP64, q=q0 + 0.001, out=outs[1])
    t3 = S.evaluate_state_async(btam.FP64, q=q0, out=outs[2])         # retires t1
    with pytest.raises(btam.BtamError) as e:
        S.wait_state(t1)
    assert e.value.code == 6  # BTAM_ERR_NONFINITE
    S.wait_state(t3)
    S.wait_state(t2)
    # the rejected update left the state: t1 evaluated the initial state
    R = btam.System(gpu_tables, s)
    R.build_neighbors()
    ref0 = R.evaluate(btam.FP64)["totals"]
    ref2 = R.evaluate_state(btam.FP64, q=q0)["totals"]
    assert np.array_equal(outs[0]["totals"], ref0)
    assert np.array_equal(outs[2]["totals"], ref2)
