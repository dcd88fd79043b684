"""GPU: the schedule picker's network (hand-written forward / backward / Adam
kernels) against its float64 restatement, and what the trained picker gains
over the fixed default schedule on fresh held-out cases, judged by the
exhaustive autotuner."""
import os

import numpy as np
import pytest

from oracle import mlp_ref

ap = pytest.importorskip("anionpy_b200")
pytestmark = pytest.mark.gpu

from anionpy_b200 import picker, workloads  # noqa: E402
from anionpy_b200._batch import DEFAULT_INDEX, NUM_SCHEDULES  # noqa: E402


def test_forward_and_gradients_match_float64_reference():
    nin, h, nout, B = picker.NFEAT, picker.HIDDEN, NUM_SCHEDULES, 300
    mlp = picker.Mlp(nin, h, nout, seed=3)
    rng = np.random.default_rng(1)
    x = rng.standard_normal((B, nin)).astype(np.float32)
    t = rng.standard_normal((B, nout)).astype(np.float32)
    p = mlp.params()
    y = mlp.forward(x)
    yref, _ = mlp_ref.forward(p, x, nin, h, nout)
    assert np.max(np.abs(y - yref)) <= 1e-4 * np.max(np.abs(yref))
    loss, g = mlp.gradients(x, t)
    lref, gref = mlp_ref.loss_and_grads(p, x, t, nin, h, nout)
    assert abs(loss - lref) <= 1e-5 * abs(lref)
    # FP32 sums over the batch against float64: tolerance relative to the
    # largest gradient entry
    assert np.max(np.abs(g - gref)) <= 1e-4 * np.max(np.abs(gref))
    mask = (rng.random((B, nout)) < 0.5).astype(np.float32)
    loss_m, g_m = mlp.gradients(x, t, mask)
    lref_m, gref_m = mlp_ref.loss_and_grads(p, x, t, nin, h, nout, mask)
    assert abs(loss_m - lref_m) <= 1e-5 * abs(lref_m)
    assert np.max(np.abs(g_m - gref_m)) <= 1e-4 * np.max(np.abs(gref_m))


def test_training_is_deterministic_and_learns():
    rng = np.random.default_rng(5)
    x = rng.standard_normal((4096, picker.NFEAT)).astype(np.float32)
    w = rng.standard_normal((picker.NFEAT, NUM_SCHEDULES)).astype(np.float32) * 0.3
    t = np.tanh(x @ w).astype(np.float32)
    runs = []
    for _ in range(2):
        mlp = picker.Mlp(seed=11)
        losses = mlp.fit(x, t, epochs=40, batch=256, lr=3e-3)
        runs.append((losses, mlp.params()))
    assert runs[0][1].tobytes() == runs[1][1].tobytes(), "training is not deterministic"
    assert runs[0][0][-1] < 0.5 * runs[0][0][0]


@pytest.mark.skipif(not os.path.exists(picker.DEFAULT_WEIGHTS), reason="picker weights not trained yet")
def test_learned_picker_beats_the_fixed_schedule():
    """Fresh cases (a seed the study never used), every schedule timed by the
    autotuner: the trained network's picks lose less time to the best
    schedule than the fixed default schedule does."""
    sp = picker.SchedulePicker()
    calls = workloads.picker_cases(160, seed=7 + 3)
    pools = workloads.DevicePools(ap, pool_elems=1 << 21, seed=33)
    b, _ = workloads.build_batch(ap, calls, pools)
    times = np.stack([b.time_call(i, reps=3) for i in range(len(b))])
    picks = sp.pick(b, fallback=False)
    learned = picker.regret(times, picks)
    fixed = picker.regret(times, np.full(len(b), DEFAULT_INDEX))
    assert learned["total"] < fixed["total"], (learned, fixed)
    assert learned["mean"] < fixed["mean"], (learned, fixed)


def test_default_schedule_is_near_the_best_single_schedule_on_a_fresh_stream():
    """A mixed stream no study used (seed 13), every call on one schedule,
    for each of the 48: the batch's default schedule is within 2 % of the
    fastest. (Per-call choices inside the persistent kernel, learned or
    tuned, moved whole streams by about their run-to-run noise; the single
    schedule is the choice that counts.)"""
    sp = picker.StreamPicker() if os.path.exists(picker.STREAM_WEIGHTS) else None
    res = picker.stream_evaluate(sp, 10000, seed=13, reps=6)
    assert res["default_ms"] <= 1.02 * res["best_uniform_ms"], res
