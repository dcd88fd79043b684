"""CPU check of the NaN-chain shortcut in the float32 row-sum kernel
(`k_red_pw32` in anionpy_b200/csrc/ionp_reduce_rowst.cuh): one of a leaf's
eight 16-element chains that sums to NaN is the engine's sequential add
(x86 NaN rules: the first NaN operand, quieted; inf - inf the default NaN)
of its elements, and the kernel finds that value without replaying the adds:
the first NaN element quieted, unless the plain sum of the elements before
it is already NaN (an inf - inf), and the default NaN when no element is a
NaN. Checked against the sequential rule on seeded chains."""
import numpy as np

DNAN = np.uint32(0xFFC00000)


def bits(v):
    return np.float32(v).view(np.uint32)


def quiet(v):
    return (bits(v) | np.uint32(0x00400000)).view(np.float32)


def x86_add(a, b):
    """float32 add with x86 SSE NaN results"""
    if np.isnan(a):
        return quiet(a)
    if np.isnan(b):
        return quiet(b)
    with np.errstate(invalid="ignore", over="ignore"):
        r = np.float32(a) + np.float32(b)
    return DNAN.view(np.float32) if np.isnan(r) else r


def shortcut(xc):
    """the kernel's value for a chain whose plain sum is NaN"""
    nan = np.isnan(xc)
    i0 = int(np.argmax(nan)) if nan.any() else len(xc)
    pre = xc[0]
    with np.errstate(invalid="ignore", over="ignore"):
        for i in range(1, min(i0, len(xc))):
            pre = np.float32(pre + xc[i])
    if i0 == len(xc) or (i0 > 0 and np.isnan(pre)):
        return DNAN.view(np.float32)
    return quiet(xc[i0])


def test_shortcut_equals_sequential_nan_rule():
    rng = np.random.default_rng(11)
    specials = np.array([np.inf, -np.inf, 3e38, -3e38], np.float32)
    payloads = np.array([0x7FC00001, 0xFFC12345, 0x7F800001, 0xFF900000, 0x7FFFFFFF], np.uint32).view(np.float32)
    checked = 0
    for _ in range(20000):
        xc = rng.standard_normal(16).astype(np.float32)
        k = rng.integers(0, 4)
        if k >= 1:                                   # infinities / overflow
            idx = rng.choice(16, rng.integers(1, 4), replace=False)
            xc[idx] = rng.choice(specials, idx.size)
        if k != 1:                                   # NaN payloads, signaling ones included
            idx = rng.choice(16, rng.integers(1, 4), replace=False)
            xc[idx] = rng.choice(payloads, idx.size)
        with np.errstate(invalid="ignore", over="ignore"):
            plain = xc[0]
            for v in xc[1:]:
                plain = np.float32(plain + v)
        if not np.isnan(plain):
            continue                                 # the kernel keeps the plain sum
        seq = xc[0] if not np.isnan(xc[0]) else quiet(xc[0])
        for v in xc[1:]:
            seq = x86_add(seq, v)
        assert bits(shortcut(xc)) == bits(seq), [hex(b) for b in xc.view(np.uint32)]
        checked += 1
    assert checked > 10000
