"""Run-time knobs of the batched path. All are off by default, which keeps the
fixed heuristic schedule for every call.

* ``IONP_BATCH_SCHEDULE=<0..47>``: every call of a batch that was queued
  without an explicit schedule runs on this schedule number.
* ``IONP_BATCH_PICKER=stream|autotune|off``: choose such calls' schedules
  when the batch first runs -- ``stream``: the picker trained on in-stream
  labels (``anionpy_b200/data/picker_stream.npz``); ``autotune``: each call
  timed under all 48 schedules (exact, slow); ``off``: the default.
* ``IONP_CONFIG=<file.json>``: the same settings as a JSON object,
  ``{"batch_schedule": 24, "batch_picker": "stream"}``; an environment
  variable wins over the file.
* ``IONP_NVTX=1``: NVTX ranges around every C-ABI call and batch run, read by
  the native library itself.

A schedule only changes how a call's work is tiled, never its result.
"""
from __future__ import annotations

import json
import os

PICKERS = ("off", "stream", "autotune")


def settings(environ=None) -> dict:
    """{"batch_schedule": int | None, "batch_picker": str} from IONP_CONFIG
    and the environment. Raises ValueError on a malformed value."""
    env = os.environ if environ is None else environ
    cfg = {}
    path = env.get("IONP_CONFIG")
    if path:
        with open(path) as f:
            cfg = json.load(f)
        if not isinstance(cfg, dict):
            raise ValueError(f"IONP_CONFIG {path}: expected a JSON object")
    sched = env.get("IONP_BATCH_SCHEDULE", cfg.get("batch_schedule"))
    picker = env.get("IONP_BATCH_PICKER", cfg.get("batch_picker", "off"))
    if sched is not None and sched != "":
        try:
            sched = int(sched)
        except (TypeError, ValueError):
            raise ValueError(f"batch schedule must be an integer 0..47, got {sched!r}") from None
        if not 0 <= sched < 48:
            raise ValueError(f"batch schedule must be in 0..47, got {sched}")
    else:
        sched = None
    picker = str(picker).lower()
    if picker not in PICKERS:
        raise ValueError(f"batch picker must be one of {PICKERS}, got {picker!r}")
    return {"batch_schedule": sched, "batch_picker": picker}
