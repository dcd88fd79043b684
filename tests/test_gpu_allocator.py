"""The caching device allocator (ionp_alloc / ionp_free): reuse on the same
stream, reuse from another stream after the freeing stream's event, the
out-of-memory path (an impossible request fails on the host after the
device's cached blocks are released, with no device fault), and the
per-device statistics."""
import ctypes

import numpy as np
import pytest

from anionpy_b200 import _lib

ap = pytest.importorskip("anionpy_b200")
pytestmark = pytest.mark.gpu


def stats():
    s = (ctypes.c_uint64 * 4)()
    _lib.check(_lib.lib().ionp_alloc_stats(s))
    return list(s)


def alloc(n, stream=None):
    p = ctypes.c_void_p()
    st = _lib.lib().ionp_alloc(ctypes.byref(p), n, stream)
    return st, p.value


def test_same_stream_reuse():
    L = _lib.lib()
    _lib.check(L.ionp_device_synchronize())
    L.ionp_alloc_trim()   # no other cached block of the size class can be handed out first
    st, p = alloc(3 << 20)
    assert st == 0 and p
    m0 = stats()[3]
    _lib.check(L.ionp_free(p, None))
    st, q = alloc(3 << 20)
    assert st == 0 and q == p, "a freed block of the same size class is reused"
    assert stats()[3] == m0, "reuse makes no cudaMalloc call"
    _lib.check(L.ionp_free(q, None))


def test_cross_stream_reuse_waits_for_the_free():
    """A block written on stream A and freed there is reused on stream B;
    B's next write must land after A's work, so B's result is B's."""
    L = _lib.lib()
    sa, sb = ctypes.c_void_p(), ctypes.c_void_p()
    _lib.check(L.ionp_stream_create(ctypes.byref(sa)))
    _lib.check(L.ionp_stream_create(ctypes.byref(sb)))
    n = 1 << 22
    _lib.check(L.ionp_device_synchronize())
    L.ionp_alloc_trim()
    host_a = np.full(n, 1.0)
    host_b = np.full(n, 2.0)
    st, p = alloc(n * 8, sa)
    assert st == 0
    _lib.check(L.ionp_memcpy(p, host_a.ctypes.data, n * 8, 0, sa))
    _lib.check(L.ionp_free(p, sa))
    st, q = alloc(n * 8, sb)
    assert st == 0 and q == p
    _lib.check(L.ionp_memcpy(q, host_b.ctypes.data, n * 8, 0, sb))
    back = np.empty(n)
    _lib.check(L.ionp_memcpy(back.ctypes.data, q, n * 8, 1, sb))
    _lib.check(L.ionp_stream_synchronize(sb))
    assert (back == 2.0).all()
    _lib.check(L.ionp_free(q, sb))
    _lib.check(L.ionp_device_synchronize())
    L.ionp_stream_destroy(sa)
    L.ionp_stream_destroy(sb)


def test_out_of_memory_trims_and_fails_cleanly():
    L = _lib.lib()
    st, p = alloc(8 << 20)
    assert st == 0
    _lib.check(L.ionp_free(p, None))
    assert stats()[1] >= 8 << 20, "the freed block is cached"
    st, _ = alloc(1 << 50)   # far beyond any GPU: cudaMalloc refuses on the host
    assert st == _lib.ERR_OOM
    assert "failed" in _lib.last_error()
    assert stats()[1] == 0, "the cache was released before the retry"
    # the device is still usable
    d = ap.from_numpy(np.arange(10.0))
    assert float(ap.add.reduce(d)) == 45.0


def test_invalid_free_and_stats():
    L = _lib.lib()
    assert L.ionp_free(0x1234, None) == _lib.ERR_INVALID
    assert "not from ionp_alloc" in _lib.last_error()
    s = stats()
    assert s[2] >= s[0] >= 0
    _lib.check(L.ionp_alloc_trim())
    assert stats()[1] == 0
