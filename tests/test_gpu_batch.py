"""GPU parity of the batched mixed stream: one persistent kernel (and its CUDA
graph replay) against one ionp_binary / ionp_reduce launch per call and
against the oracle, bit for bit, under the default schedule and under random
schedules from the 48-point space (a schedule must never change a bit)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests._util import assert_bits_equal

ap = pytest.importorskip("anionpy_b200")
pytestmark = pytest.mark.gpu

from anionpy_b200 import _lib, workloads  # noqa: E402
from anionpy_b200._batch import NUM_SCHEDULES, Batch, schedule  # noqa: E402


def _scramble(outs):
    """Overwrite every output with a byte pattern so a later run must write
    every element."""
    L = _lib.lib()
    for o in outs:
        if o.size:
            junk = np.full(o.nbytes, 0xA5, np.uint8)
            _lib.check(L.ionp_memcpy(o.data_ptr, junk.ctypes.data, o.nbytes, 0, None))
    _lib.check(L.ionp_device_synchronize())


def _gets(outs):
    return [o.get() for o in outs]


@pytest.fixture(scope="module")
def pools():
    return workloads.DevicePools(ap, pool_elems=1 << 20, seed=4)


@pytest.fixture(scope="module")
def stream_calls():
    calls, skipped = workloads.mixed_stream(ncalls=300, seed=3, n_max=60000)
    return calls


def test_batch_equals_per_call_and_oracle(pools, stream_calls):
    b, hosts = workloads.build_batch(ap, stream_calls, pools, keep_host=True)
    b.run_per_call()
    want = _gets(b.outputs)
    # the oracle on the host copies of the same operands
    for i, (c, h) in enumerate(zip(stream_calls, hosts)):
        if c.kind == "binary":
            ref = O.binary(c.op, h[0], h[1])[0]
        else:
            ref = np.asarray(O.reduce(c.op, h[0], axis=c.axis))
        assert_bits_equal(want[i], ref.reshape(want[i].shape), f"per-call {i} {c}")
    for graph in (False, True, True):
        _scramble(b.outputs)
        b.run(graph=graph)
        got = _gets(b.outputs)
        for i, c in enumerate(stream_calls):
            assert_bits_equal(got[i], want[i], f"batch (graph={graph}) call {i} {c}")


def test_schedules_never_change_results(pools, stream_calls):
    b, _ = workloads.build_batch(ap, stream_calls, pools)
    b.run(graph=False)
    want = _gets(b.outputs)
    rng = np.random.default_rng(9)
    for trial in range(3):
        b.set_schedules(rng.integers(0, NUM_SCHEDULES, len(b)))
        _scramble(b.outputs)
        b.run(graph=False)
        got = _gets(b.outputs)
        for i, c in enumerate(stream_calls):
            assert_bits_equal(got[i], want[i], f"trial {trial} call {i} {c}")


@pytest.mark.parametrize("sched", [0, 1, 13, 47])
def test_split_and_long_reductions(pools, sched):
    """Runs long enough for one CTA per output (and the two-half split),
    narrow axes with the associative split, float16 widening."""
    b = Batch()
    cases = [("add", "float32", (3, 250000), 1), ("add", "float64", (2, 70001), 1), ("maximum", "float32", (5, 9000), 1),
             ("add", "int32", (4, 100000), 1), ("maximum", "int64", (3000, 40), 0), ("add", "int16", (700, 300), 0),
             ("add", "float16", (6, 30001), 1), ("add", "float64", (257, 129), 0), ("maximum", "float16", (9, 999), 0),
             ("add", "bool", (5, 4097), 1)]
    hosts = []
    for op, dt, shape, axis in cases:
        x, hx = pools.array(shape, dt)
        b.add_reduce(op, x, axis, sched=sched)
        hosts.append(hx)
    _scramble(b.outputs)
    b.run(graph=True)
    for (op, dt, shape, axis), h, o in zip(cases, hosts, b.outputs):
        ref = np.asarray(O.reduce(op, h, axis=axis))
        assert_bits_equal(o.get(), ref, f"{op}.reduce {dt}{shape} axis={axis} sched={sched}")


def test_broadcast_and_mixed_dtypes(pools):
    b = Batch()
    cases = [("add", ((3, 1, 5), "int8"), ((1, 4, 5), "float16")), ("less", ((7, 1), "int16"), ((1, 9), "float32")),
             ("multiply", ((2, 3, 1, 4), "float32"), ((2, 1, 6, 1), "float64")), ("logical_and", ((10,), "float64"), ((10,), "int8")),
             ("maximum", ((33, 1), "bool"), ((1, 65), "int64")), ("subtract", ((5,), "bool"), ((1,), "int32"))]
    hosts = []
    for op, (sa, da), (sb, db) in cases:
        x, hx = pools.array(sa, da)
        y, hy = pools.array(sb, db)
        b.add_binary(op, x, y)
        hosts.append((hx, hy))
    b.run(graph=False)
    for (op, _, _), (hx, hy), o in zip(cases, hosts, b.outputs):
        ref = O.binary(op, hx, hy)[0]
        assert_bits_equal(o.get(), ref, f"{op} {hx.dtype}{hx.shape} {hy.dtype}{hy.shape}")


def test_batch_errors_match_the_reference():
    b = Batch()
    x = ap.from_numpy(np.ones(4, np.bool_))
    with pytest.raises(TypeError, match="boolean subtract"):
        b.add_binary("subtract", x, x)
    with pytest.raises(ValueError, match="could not be broadcast"):
        b.add_binary("add", ap.from_numpy(np.ones(3)), ap.from_numpy(np.ones(4)), out=ap.empty((3,), np.float64))


def test_fpe_words():
    b = Batch()
    big = ap.from_numpy(np.array([1e30, 2.0, 3.0], np.float32))
    tiny = ap.from_numpy(np.array([1e-30, 1.0, 1.0], np.float32))
    b.add_binary("multiply", big, big)     # overflow
    b.add_binary("multiply", tiny, tiny)   # underflow
    b.add_binary("add", big, big)          # add has no detector in the reference
    b.run(graph=False)
    w = b.fpe()
    assert w[0] & _lib.FPE_OVER and w[1] & _lib.FPE_UNDER and w[2] == 0


def test_time_call_reports_every_schedule(pools):
    b = Batch()
    x, _ = pools.array((1000, 300), "float32")
    y, _ = pools.array((1000, 300), "float32")
    b.add_binary("add", x, y)
    b.add_reduce("add", x, 1)
    for call in range(2):
        t = b.time_call(call, reps=2)
        assert t.shape == (NUM_SCHEDULES,) and np.all(t > 0) and np.all(np.isfinite(t))
    assert schedule(47).block_tile == 1024 and schedule(47).red_split == 2


def test_schedule_knob_applies_and_keeps_results(pools, stream_calls, monkeypatch):
    """IONP_BATCH_SCHEDULE puts every call queued without a schedule of its
    own on that schedule at the first run (the tile count matches a batch set
    to it explicitly), and each result stays that of the same call launched
    on its own."""
    ref, _ = workloads.build_batch(ap, stream_calls, pools)
    ref.run(graph=False)
    explicit, _ = workloads.build_batch(ap, stream_calls, pools)
    explicit.set_schedules(np.full(len(explicit), 0))
    explicit.run(graph=False)
    monkeypatch.setenv("IONP_BATCH_SCHEDULE", "0")
    b, _ = workloads.build_batch(ap, stream_calls, pools)
    b.run(graph=True)
    assert b.info()["tiles"] == explicit.info()["tiles"] != ref.info()["tiles"]
    got = _gets(b.outputs)
    b.run_per_call()
    want = _gets(b.outputs)
    for i, c in enumerate(stream_calls):
        assert_bits_equal(got[i], want[i], f"knob schedule call {i} {c}")
