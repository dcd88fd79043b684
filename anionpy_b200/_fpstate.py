"""Floating-point error state: seterr / geterr / errstate / seterrcall.

Host-side restatement of ionp-py/src/fpstate.rs:39-402. The device only
produces the OR of FPE bits per call; which category is reported and how
(ignore / warn / raise / print / call / log) is decided here, per thread.
"""
from __future__ import annotations

import functools
import sys
import threading
import warnings

_MODES = ("ignore", "warn", "raise", "print", "call", "log")
_CATS = ("divide", "over", "under", "invalid")
_DEFAULT = {"divide": "warn", "over": "warn", "under": "ignore", "invalid": "warn"}
_PHRASE = {"divide": "divide by zero", "over": "overflow", "under": "underflow", "invalid": "invalid value"}
_BIT = {"divide": 1, "over": 2, "under": 4, "invalid": 8}

_tls = threading.local()


def _state():
    st = getattr(_tls, "state", None)
    if st is None:
        st = dict(_DEFAULT)
        _tls.state = st
    return st


def _parse(name, val):
    if not isinstance(val, str):
        raise TypeError(f"seterr() argument '{name}' must be str")
    if val not in _MODES:
        raise ValueError(f'invalid error mode "{val}"')
    return val


def seterr(all=None, divide=None, over=None, under=None, invalid=None):
    st = _state()
    prev = dict(st)
    new = dict(st)
    if all is not None:
        m = _parse("all", all)
        for c in _CATS:
            new[c] = m
    for c, v in (("divide", divide), ("over", over), ("under", under), ("invalid", invalid)):
        if v is not None:
            new[c] = _parse(c, v)
    _tls.state = new
    return prev


def geterr():
    return dict(_state())


def seterrcall(func):
    prev = getattr(_tls, "callback", None)
    _tls.callback = func
    return prev


def geterrcall():
    return getattr(_tls, "callback", None)


class errstate:
    """Context manager / decorator that sets the error state for a block."""

    def __init__(self, *, call=None, all=None, divide=None, over=None, under=None, invalid=None):
        am = _parse("all", all) if all is not None else None
        self._set = {}
        for c, v in (("divide", divide), ("over", over), ("under", under), ("invalid", invalid)):
            m = _parse(c, v) if v is not None else am
            if m is not None:
                self._set[c] = m
        self._call = call
        self._saved = None

    def __enter__(self):
        self._saved = (dict(_state()), getattr(_tls, "callback", None))
        new = dict(_state())
        new.update(self._set)
        _tls.state = new
        if self._call is not None:
            _tls.callback = self._call
        return self

    def __exit__(self, *exc):
        if self._saved is not None:
            _tls.state, _tls.callback = self._saved
            self._saved = None
        return False

    def __call__(self, func):
        @functools.wraps(func)
        def wrapper(*a, **k):
            with self:
                return func(*a, **k)
        return wrapper


def signal(cat: str, ufunc_name: str, stacklevel: int = 3):
    """fpstate::signal (fpstate.rs:212-285)."""
    mode = _state()[cat]
    msg = f"{_PHRASE[cat]} encountered in {ufunc_name}"
    if mode == "ignore":
        return
    if mode == "warn":
        warnings.warn(msg, RuntimeWarning, stacklevel=stacklevel)
    elif mode == "raise":
        raise FloatingPointError(msg)
    elif mode == "print":
        print(f"Warning: {msg}", file=sys.stderr)
    elif mode == "call":
        cb = getattr(_tls, "callback", None)
        if cb is None:
            raise NameError(f"call specified for {_PHRASE[cat]} (in {ufunc_name}) but no callable function found")
        cb(_PHRASE[cat], _BIT[cat])
    elif mode == "log":
        cb = getattr(_tls, "callback", None)
        if cb is None:
            raise NameError(f"log specified for {_PHRASE[cat]} (in {ufunc_name}) but no object with write method found.")
        cb.write(f"Warning: {msg}\n")


def category_of(op_kind: str, bits: int):
    """The one category the reference reports for a call (fpe.rs:162-168):
    divide family / sqrt / log: invalid beats divide; multiply: over beats
    under."""
    if not bits:
        return None
    if op_kind == "multiply":
        return "over" if bits & 2 else ("under" if bits & 4 else None)
    if bits & 8:
        return "invalid"
    if bits & 1:
        return "divide"
    return None
