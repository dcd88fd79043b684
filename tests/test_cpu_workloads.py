"""CPU checks of the mixed-stream generator and the schedule space (no kernel
launches)."""
import numpy as np

from anionpy_b200 import _lib, workloads
from anionpy_b200._batch import BLOCK_TILES, ELEMS_PER_THREAD, NUM_SCHEDULES, RED_SPLITS, VEC_WIDTHS, schedule_index


def test_stream_is_seeded_and_shaped_like_the_workload():
    a, sa = workloads.mixed_stream(ncalls=2000, seed=7)
    b, sb = workloads.mixed_stream(ncalls=2000, seed=7)
    assert sa == sb and [(c.kind, c.op, c.shapes, c.dtypes, c.axis) for c in a] == \
        [(c.kind, c.op, c.shapes, c.dtypes, c.axis) for c in b]
    kinds = np.array([c.kind == "binary" for c in a])
    assert 0.66 < kinds.mean() < 0.74
    ranks = [len(c.shapes[0]) for c in a]
    assert set(ranks) == {1, 2, 3, 4}
    for c in a:
        if c.kind == "binary":
            assert c.op in workloads.BINARY6
            assert not (c.op == "subtract" and np.promote_types(*c.dtypes) == np.bool_)
            np.broadcast_shapes(*c.shapes)
        else:
            assert c.op in workloads.REDUCE2 and 0 <= c.axis < len(c.shapes[0])
    sizes = [int(np.prod(c.shapes[0])) for c in a if c.kind == "reduce"]
    assert min(sizes) >= 1 and max(sizes) < 3 * 10 ** 6


def test_schedule_space_matches_the_library():
    L = _lib.load_library()
    seen = set()
    for k in range(NUM_SCHEDULES):
        s = _lib.IonpSchedule()
        assert L.ionp_schedule_from_index(k, s) == 0
        t = (s.block_tile, s.vec_width, s.elems_per_thread, s.red_split)
        assert t[0] in BLOCK_TILES and t[1] in VEC_WIDTHS and t[2] in ELEMS_PER_THREAD and t[3] in RED_SPLITS
        assert schedule_index(*t) == k
        seen.add(t)
    assert len(seen) == 48
    assert L.ionp_schedule_from_index(48, _lib.IonpSchedule()) != 0


def test_stream_schedule_set():
    from anionpy_b200 import picker
    from anionpy_b200._batch import BLOCK_TILES, ELEMS_PER_THREAD, RED_SPLITS, VEC_WIDTHS
    allowed = picker.stream_schedules()
    assert len(allowed) == 7 and len(set(allowed.tolist())) == 7
    default = schedule_index(256, 1, 4, 1)
    assert default in allowed
    for k in allowed:
        bt, rest = BLOCK_TILES[k // 12], k % 12
        vw, ept, sp = VEC_WIDTHS[rest // 4], ELEMS_PER_THREAD[(rest % 4) // 2], RED_SPLITS[rest % 2]
        assert bt >= 256 and bt * vw * ept <= 1024 and sp == 1
