"""Autotuner and learned schedule picker for batched calls.

* The **autotuner** times a call under every one of the 48 schedules
  (``Batch.time_call``: the call queued enough times in one persistent launch
  to fill the GPU, every copy on its own operand region so that the copies
  stream from HBM like the distinct calls of a real batch; CUDA events, time
  per copy) and keeps the fastest. It is exact but costs 48 timed runs per
  call.
* The **picker** is a 3-layer perceptron (width 64, FP32; forward, backward
  and Adam are this library's own CUDA kernels, ``ionp_mlp_*``) that maps a
  call's features (``ionp_batch_features``: op class, call kind, operand
  widths, merged shape, stride class, reduction geometry) to a predicted
  log-time for each schedule, and picks the argmin. It is trained on the
  autotuner's own timings. Calls whose features fall outside the box seen in
  training go to the autotuner instead (the fallback), and the autotuner's
  timings are the judge of the picker's regret.

Schedules never change results (every schedule computes the same bits), so
the picker only moves time.

Command line (the study that produced ``data/picker.npz``)::

    python -m anionpy_b200.picker study --train 50000 --test 5000
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import time

import numpy as np

from . import _lib
from ._batch import DEFAULT_INDEX, NUM_SCHEDULES, Batch

NFEAT = 32
HIDDEN = 64
HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "data", "picker.npz")


def features(batch: Batch) -> np.ndarray:
    """[calls, 32] feature matrix of a batch's calls."""
    L = _lib.lib()
    out = np.zeros((len(batch), NFEAT), np.float32)
    for i in range(len(batch)):
        _lib.check(L.ionp_batch_features(batch._h, i, out[i].ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
    return out


class _Dev:
    """A device float32 buffer (from the engine's allocator)."""

    def __init__(self, host: np.ndarray):
        from ._array import from_numpy
        self.arr = from_numpy(np.ascontiguousarray(host, np.float32))

    @property
    def ptr(self):
        return self.arr.data_ptr


class Mlp:
    """The picker's network on the device (``ionp_mlp_*``)."""

    def __init__(self, nin=NFEAT, hidden=HIDDEN, nout=NUM_SCHEDULES, seed=0):
        self.nin, self.hidden, self.nout = nin, hidden, nout
        self._h = ctypes.c_void_p()
        _lib.check(_lib.lib().ionp_mlp_create(ctypes.byref(self._h), nin, hidden, nout, seed))
        n = ctypes.c_int64()
        _lib.check(_lib.lib().ionp_mlp_num_params(self._h, ctypes.byref(n)))
        self.nparam = n.value

    def __del__(self):
        try:
            if self._h:
                _lib.lib().ionp_mlp_destroy(self._h)
        except Exception:
            pass
        self._h = None

    def params(self) -> np.ndarray:
        p = np.zeros(self.nparam, np.float32)
        _lib.check(_lib.lib().ionp_mlp_get(self._h, 0, p.ctypes.data, self.nparam))
        return p

    def grads(self) -> np.ndarray:
        g = np.zeros(self.nparam, np.float32)
        _lib.check(_lib.lib().ionp_mlp_get(self._h, 1, g.ctypes.data, self.nparam))
        return g

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.nparam
        _lib.check(_lib.lib().ionp_mlp_set_params(self._h, p.ctypes.data, self.nparam))

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        dx = _Dev(x)
        from ._array import ndarray
        y = ndarray.empty((x.shape[0], self.nout), np.float32)
        _lib.check(_lib.lib().ionp_mlp_forward(self._h, dx.ptr, x.shape[0], y.data_ptr, None))
        return y.get()

    def gradients(self, x, t, mask=None):
        """(loss, flat gradient) of the mean squared error on one batch."""
        dx, dt = _Dev(x), _Dev(t)
        dm = _Dev(mask) if mask is not None else None
        loss = ctypes.c_float()
        _lib.check(_lib.lib().ionp_mlp_gradients(self._h, dx.ptr, dt.ptr, dm.ptr if dm else None, x.shape[0],
                                                 ctypes.byref(loss), None))
        return loss.value, self.grads()

    def fit(self, x, t, epochs=40, batch=1024, lr=2e-3, weight_decay=0.0, seed=0, log=None):
        """Adam on the mean squared error of log-times; the data stay on the
        device, minibatches are contiguous slices of a per-epoch permutation."""
        rng = np.random.default_rng(seed)
        n = x.shape[0]
        batch = min(batch, n)
        losses = []
        L = _lib.lib()
        for ep in range(epochs):
            perm = rng.permutation(n)
            dx, dt = _Dev(x[perm]), _Dev(t[perm])
            ep_loss = []
            lr_ep = lr * (0.5 * (1 + np.cos(np.pi * ep / epochs)))
            starts = list(range(0, n - batch + 1, batch))
            for s0 in starts:
                loss = ctypes.c_float()
                want = s0 == starts[-1]  # the loss is read back once per epoch
                _lib.check(L.ionp_mlp_train_step(self._h, dx.ptr + s0 * self.nin * 4, dt.ptr + s0 * self.nout * 4,
                                                 None, batch, float(lr_ep), float(weight_decay),
                                                 ctypes.byref(loss) if want else None, None))
                if want:
                    ep_loss.append(loss.value)
            losses.append(float(np.mean(ep_loss)) if ep_loss else float("nan"))
            if log:
                log(f"epoch {ep}: loss {losses[-1]:.4f}")
        return losses


def stream_schedules() -> np.ndarray:
    """Schedules a call may take inside a mixed stream: at least 256 threads'
    worth of block tile, at most 1024 16-byte units of work per tile, no
    reduction split. The autotuner times a call alone (many copies of it),
    where long tiles amortise per-tile costs; in a persistent kernel shared
    by thousands of different calls, long tiles and split reductions made the
    whole stream slower (10,000-call stream, every call on one schedule: these
    7 schedules took 11.2-12.3 ms, tiles of 2048-16384 units 12.6-15.9 ms,
    block tile 128 14.6-21.2 ms, each split variant 1.5-2.6 ms more), so the
    picker chooses among these."""
    from ._batch import BLOCK_TILES, ELEMS_PER_THREAD, RED_SPLITS, VEC_WIDTHS, schedule_index
    keep = []
    for bt in BLOCK_TILES:
        for vw in VEC_WIDTHS:
            for ept in ELEMS_PER_THREAD:
                if bt >= 256 and bt * vw * ept <= 1024:
                    keep.append(schedule_index(bt, vw, ept, RED_SPLITS[0]))
    return np.array(sorted(keep))


class SchedulePicker:
    """Picks one schedule per call: the network's argmin (over `allowed`
    schedules when given), or the autotuner for calls outside the training
    feature box."""

    def __init__(self, path=DEFAULT_WEIGHTS):
        d = np.load(path)
        self.mlp = Mlp(int(d["nin"]), int(d["hidden"]), int(d["nout"]))
        self.mlp.set_params(d["params"])
        self.lo, self.hi = d["feat_lo"], d["feat_hi"]
        self.fallbacks = 0

    def predict(self, feats: np.ndarray) -> np.ndarray:
        return self.mlp.forward(feats)

    def pick(self, batch: Batch, fallback=True, reps=3, allowed=None) -> np.ndarray:
        f = features(batch)
        pred = self.predict(f)
        cols = np.arange(pred.shape[1]) if allowed is None else np.asarray(allowed)
        picks = cols[np.argmin(pred[:, cols], axis=1)]
        outside = np.any((f < self.lo - 1e-6) | (f > self.hi + 1e-6), axis=1)
        self.fallbacks = int(outside.sum())
        if fallback:
            for i in np.nonzero(outside)[0]:
                picks[i] = int(cols[np.argmin(batch.time_call(int(i), scheds=cols, reps=reps))])
        return picks


# ---------------------------------------------------------------------------
# the study: collect autotuner timings, train, evaluate regret
# ---------------------------------------------------------------------------
def collect(ncases, seed, reps=3, chunk=500, log=None):
    """(features [n, 32], microseconds [n, 48]) of `ncases` picker-study cases,
    every schedule timed by the autotuner."""
    import anionpy_b200 as ap
    from . import workloads
    calls = workloads.picker_cases(ncases, seed)
    pools = workloads.DevicePools(ap, pool_elems=1 << 22, seed=seed + 5)
    X = np.zeros((ncases, NFEAT), np.float32)
    T = np.zeros((ncases, NUM_SCHEDULES), np.float32)
    t0 = time.time()
    for c0 in range(0, ncases, chunk):
        part = calls[c0: c0 + chunk]
        b, _ = workloads.build_batch(ap, part, pools)
        X[c0: c0 + len(part)] = features(b)
        for i in range(len(part)):
            T[c0 + i] = b.time_call(i, reps=reps)
        del b
        if log:
            log(f"collected {min(c0 + chunk, ncases)}/{ncases} cases, {time.time() - t0:.0f} s")
    return X, T


def regret(times: np.ndarray, picks: np.ndarray) -> dict:
    """Regret of picks against the exhaustive autotuner's best, per case
    (mean and percentiles of t_pick/t_best - 1) and over the whole set
    (sum t_pick / sum t_best - 1)."""
    best = times.min(axis=1)
    chosen = times[np.arange(len(times)), picks]
    r = chosen / best - 1.0
    return {"mean": float(r.mean()), "p50": float(np.median(r)), "p90": float(np.percentile(r, 90)),
            "total": float(chosen.sum() / best.sum() - 1.0), "exact_best": float(np.mean(r == 0))}


def study(ntrain, ntest, seed=7, reps=3, epochs=60, out=DEFAULT_WEIGHTS, log=print):
    Xtr, Ttr = collect(ntrain, seed + 1, reps=reps, log=log)
    Xte, Tte = collect(ntest, seed + 2, reps=reps, log=log)
    ytr = np.log(np.maximum(Ttr, 1e-3))
    mlp = Mlp(seed=seed)
    losses = mlp.fit(Xtr, ytr, epochs=epochs, log=log)
    params = mlp.params()
    lo, hi = Xtr.min(axis=0), Xtr.max(axis=0)
    os.makedirs(os.path.dirname(out), exist_ok=True)
    np.savez_compressed(out, params=params, nin=NFEAT, hidden=HIDDEN, nout=NUM_SCHEDULES, feat_lo=lo, feat_hi=hi)
    pred = mlp.forward(Xte)
    picks = np.argmin(pred, axis=1)
    inside = ~np.any((Xte < lo - 1e-6) | (Xte > hi + 1e-6), axis=1)
    picks_fb = np.where(inside, picks, np.argmin(Tte, axis=1))  # fallback = the autotuner's own best
    res = {
        "train_cases": ntrain, "test_cases": ntest, "schedules": NUM_SCHEDULES, "reps": reps, "epochs": epochs,
        "final_train_loss": losses[-1], "fallback_cases": int((~inside).sum()),
        "regret_learned": regret(Tte, picks_fb),
        "regret_learned_no_fallback": regret(Tte, picks),
        "regret_fixed_heuristic": regret(Tte, np.full(len(Tte), DEFAULT_INDEX)),
        "regret_random": regret(Tte, np.random.default_rng(0).integers(0, NUM_SCHEDULES, len(Tte))),
        "test_total_us": {"autotuner_best": float(Tte.min(axis=1).sum()),
                          "learned": float(Tte[np.arange(len(Tte)), picks_fb].sum()),
                          "fixed_heuristic": float(Tte[:, DEFAULT_INDEX].sum())},
    }
    return res, (Xtr, Ttr, Xte, Tte)


def stream_sweep(ncalls=10000, seed=7, steps=4, warmup=2):
    """Device milliseconds of the mixed stream (persistent kernel, CUDA graph)
    with every call on one schedule, for each of the 48, and with the learned
    picks over all schedules and over `stream_schedules()`."""
    import anionpy_b200 as ap
    from . import workloads
    check = _lib.check
    L = _lib.lib()
    calls, _ = workloads.mixed_stream(ncalls=ncalls, seed=seed)
    pools = workloads.DevicePools(ap, pool_elems=1 << 22, seed=17)
    b, _ = workloads.build_batch(ap, calls, pools)
    e0, e1 = ctypes.c_void_p(), ctypes.c_void_p()
    check(L.ionp_event_create(ctypes.byref(e0)))
    check(L.ionp_event_create(ctypes.byref(e1)))

    def timed(sched):
        b.set_schedules(sched)
        for _ in range(warmup):
            b.run(graph=True)
        check(L.ionp_device_synchronize())
        check(L.ionp_event_record(e0, None))
        for _ in range(steps):
            b.run(graph=True)
        check(L.ionp_event_record(e1, None))
        check(L.ionp_device_synchronize())
        ms = ctypes.c_float()
        check(L.ionp_event_elapsed_ms(e0, e1, ctypes.byref(ms)))
        return {"ms": round(ms.value / steps, 3), "tiles": b.info()["tiles"]}

    n = len(b)
    res = {f"schedule_{k}": timed(np.full(n, k)) for k in range(NUM_SCHEDULES)}
    if os.path.exists(DEFAULT_WEIGHTS):
        sp = SchedulePicker()
        res["learned_all"] = timed(sp.pick(b, fallback=False))
        res["learned_stream_set"] = timed(sp.pick(b, fallback=False, allowed=stream_schedules()))
    return res


# ---------------------------------------------------------------------------
# the in-stream study: labels from mixed sub-streams instead of lone calls
# ---------------------------------------------------------------------------
STREAM_WEIGHTS = os.path.join(HERE, "data", "picker_stream.npz")


def class_keys(F: np.ndarray) -> list:
    """Coarse call classes of a feature matrix: call kind, element count
    (log2 in steps of 4) and output width -- few enough classes, each with
    enough calls, that moving one class to another schedule changes the
    whole stream's time by far more than its run-to-run noise."""
    kind = np.argmax(F[:, 8:11], axis=1)
    size = np.clip((F[:, 20] * 20 / 4).astype(int), 0, 5)
    wout = np.rint(F[:, 13] * 3).astype(int)
    return list(zip(kind.tolist(), size.tolist(), wout.tolist()))


def _stream_timer():
    L = _lib.lib()
    e0, e1 = ctypes.c_void_p(), ctypes.c_void_p()
    _lib.check(L.ionp_event_create(ctypes.byref(e0)))
    _lib.check(L.ionp_event_create(ctypes.byref(e1)))

    def timed(b: Batch, sched, reps=3, warmup=1) -> float:
        """Device ms of one graph replay of the whole batch, `sched` a
        schedule index per call."""
        b.set_schedules(sched)
        for _ in range(warmup):
            b.run(graph=True)
        _lib.check(L.ionp_device_synchronize())
        _lib.check(L.ionp_event_record(e0, None))
        for _ in range(reps):
            b.run(graph=True)
        _lib.check(L.ionp_event_record(e1, None))
        _lib.check(L.ionp_device_synchronize())
        ms = ctypes.c_float()
        _lib.check(L.ionp_event_elapsed_ms(e0, e1, ctypes.byref(ms)))
        return ms.value / reps
    return timed


def stream_collect(ncalls, seed, reps=3, accept=0.002, log=None):
    """(features [n, 32], targets [n, 48], classes) from one mixed stream,
    labelled by the WHOLE stream's device time (persistent kernel, CUDA
    graph): first the best single schedule for every call, then one pass of
    coordinate descent over the call classes (`class_keys`, largest total
    work first) -- each class tried on every schedule with the others fixed,
    its best kept when it makes the stream at least `accept` (relative)
    faster. Each call's target is 0 for its class's final schedule and 1 for
    the others, so the network learns the assignment the stream measured."""
    import anionpy_b200 as ap
    from . import workloads
    calls, _ = workloads.mixed_stream(ncalls=ncalls, seed=seed)
    pools = workloads.DevicePools(ap, pool_elems=1 << 22, seed=seed + 17)
    b, _ = workloads.build_batch(ap, calls, pools)
    n = len(b)
    F = features(b)
    groups = {}
    for i, k in enumerate(class_keys(F)):
        groups.setdefault(k, []).append(i)
    timed = _stream_timer()
    t0 = time.time()
    uni = [timed(b, np.full(n, sch), reps=reps) for sch in range(NUM_SCHEDULES)]
    cur = np.full(n, int(np.argmin(uni)))
    best_t = min(uni)
    work = {k: float(np.sum(10.0 ** (F[idx, 20] * 20 * np.log10(2)))) for k, idx in groups.items()}
    for gi, k in enumerate(sorted(groups, key=lambda k: -work[k])):
        idx = np.array(groups[k])
        trial = cur.copy()
        ts = []
        for sch in range(NUM_SCHEDULES):
            trial[idx] = sch
            ts.append(timed(b, trial, reps=reps))
        base = timed(b, cur, reps=reps)
        sbest = int(np.argmin(ts))
        if ts[sbest] < base * (1.0 - accept):
            cur[idx] = sbest
            best_t = ts[sbest]
        if log and (gi + 1) % 10 == 0:
            log(f"stream {seed}: class {gi + 1}/{len(groups)}, stream {best_t:.3f} ms, {time.time() - t0:.0f} s")
    Y = np.ones((n, NUM_SCHEDULES), np.float32)
    Y[np.arange(n), cur] = 0.0
    return F, Y, {"classes": len(groups), "default_ms": round(uni[DEFAULT_INDEX], 3),
                  "best_uniform_ms": round(min(uni), 3), "tuned_ms": round(timed(b, cur, reps=reps), 3)}


class StreamPicker(SchedulePicker):
    """The picker trained on in-stream labels: the network scores each
    schedule for a call (0 = the schedule the measured stream assigned to
    calls like it, 1 = any other) and the call takes the lowest score."""

    def __init__(self, path=STREAM_WEIGHTS):
        super().__init__(path)

    def pick(self, batch: Batch, fallback=False, reps=3, allowed=None) -> np.ndarray:
        self.fallbacks = 0
        return np.argmin(self.predict(features(batch)), axis=1)


def stream_evaluate(picker_, ncalls, seed, reps=4):
    """Device ms of a fresh mixed stream under the default schedule, under
    the best single schedule, and (picker_ given) under its per-call picks."""
    import anionpy_b200 as ap
    from . import workloads
    calls, _ = workloads.mixed_stream(ncalls=ncalls, seed=seed)
    pools = workloads.DevicePools(ap, pool_elems=1 << 22, seed=seed + 17)
    b, _ = workloads.build_batch(ap, calls, pools)
    timed = _stream_timer()
    n = len(b)
    uniform = {s: timed(b, np.full(n, s), reps=reps) for s in range(NUM_SCHEDULES)}
    default = timed(b, np.full(n, DEFAULT_INDEX), reps=reps)
    best_s = min(uniform, key=uniform.get)
    res = {"calls": n, "seed": seed, "default_ms": round(default, 3),
           "best_uniform_schedule": int(best_s), "best_uniform_ms": round(uniform[best_s], 3)}
    if picker_ is not None:
        picks = picker_.pick(b)
        res.update({"learned_ms": round(timed(b, picks, reps=reps), 3),
                    "calls_off_default": int(np.sum(picks != DEFAULT_INDEX)),
                    "distinct_schedules": int(len(set(picks.tolist())))})
    return res


def stream_study(ncalls=10000, train_seeds=(101, 102), eval_seeds=(7, 9, 13), reps=3, epochs=60,
                 out=STREAM_WEIGHTS, log=print):
    Xs, Ys, ncls = [], [], []
    for sd in train_seeds:
        X, Y, info = stream_collect(ncalls, sd, reps=reps, log=log)
        Xs.append(X); Ys.append(Y); ncls.append(info)
    X, Y = np.concatenate(Xs), np.concatenate(Ys)
    mlp = Mlp(seed=3)
    losses = mlp.fit(X, Y, epochs=epochs, log=log)
    lo, hi = X.min(axis=0), X.max(axis=0)
    os.makedirs(os.path.dirname(out), exist_ok=True)
    np.savez_compressed(out, params=mlp.params(), nin=NFEAT, hidden=HIDDEN, nout=NUM_SCHEDULES, feat_lo=lo, feat_hi=hi)
    sp = StreamPicker(out)
    res = {"train_streams": list(train_seeds), "calls_per_stream": ncalls, "training": ncls,
           "final_train_loss": losses[-1],
           "eval": [stream_evaluate(sp, ncalls, sd) for sd in eval_seeds]}
    return res


def main():
    ap_ = argparse.ArgumentParser()
    sub = ap_.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("stream", help="time the mixed stream under every schedule")
    t.add_argument("--calls", type=int, default=10000)
    ss = sub.add_parser("stream-study", help="train the picker on in-stream labels")
    ss.add_argument("--calls", type=int, default=10000)
    ss.add_argument("--epochs", type=int, default=60)
    ss.add_argument("--out", default=STREAM_WEIGHTS)
    ss.add_argument("--report", default=None)
    s = sub.add_parser("study")
    s.add_argument("--train", type=int, default=50000)
    s.add_argument("--test", type=int, default=5000)
    s.add_argument("--reps", type=int, default=3)
    s.add_argument("--epochs", type=int, default=60)
    s.add_argument("--out", default=DEFAULT_WEIGHTS)
    s.add_argument("--report", default=None, help="write the regret summary (JSON) here")
    s.add_argument("--dump", default=None, help="save the timing dataset (npz) here")
    args = ap_.parse_args()
    if args.cmd == "stream":
        print(json.dumps(stream_sweep(args.calls), indent=1))
        return
    if args.cmd == "stream-study":
        res = stream_study(args.calls, epochs=args.epochs, out=args.out)
        print(json.dumps(res, indent=1))
        if args.report:
            with open(args.report, "w") as f:
                json.dump(res, f, indent=1)
        return
    res, data = study(args.train, args.test, reps=args.reps, epochs=args.epochs, out=args.out)
    print(json.dumps(res, indent=1))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(res, f, indent=1)
    if args.dump:
        np.savez_compressed(args.dump, Xtr=data[0], Ttr=data[1], Xte=data[2], Tte=data[3])


if __name__ == "__main__":
    main()
