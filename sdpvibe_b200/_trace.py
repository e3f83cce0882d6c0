"""Lightweight tracing of library calls (the B200 counterpart of the reference's SDPB_GPU_TIMING
phase timers, sdpvibe/solver.py:119-143).

While a `Trace` is active, every kernel-launching C-ABI call is counted per entry point, and the
entry points listed in `timed` are bracketed with CUDA events on the launching stream, so per-kernel
device time can be read back after a synchronize.  Inactive tracing costs one attribute test per call.
"""
import collections

import torch

_active = None

# Entry points that configure or query rather than launch a kernel.
NON_LAUNCH = {"sdpv_version", "sdpv_last_error", "sdpv_ctx_create", "sdpv_ctx_destroy", "sdpv_ctx_query",
              "sdpv_ctx_moduli", "sdpv_get_error", "sdpv_bigfloat_index", "sdpv_tune_set", "sdpv_tune_get"}


class Trace:
    def __init__(self, timed=()):
        self.timed = set(timed)
        self.launches = collections.Counter()
        self.events = collections.defaultdict(list)

    def __enter__(self):
        global _active
        self._prev, _active = _active, self
        return self

    def __exit__(self, *exc):
        global _active
        _active = self._prev

    @property
    def total_launches(self):
        return sum(self.launches.values())

    def kernel_ms(self, name):
        """Device milliseconds of every traced launch of `name` (synchronises)."""
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in self.events[name]]


def before(name):
    t = _active
    if t is None or name in NON_LAUNCH:
        return None
    t.launches[name] += 1
    if name in t.timed and not torch.cuda.is_current_stream_capturing():
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        t.events[name].append((a, b))
        return b
    return None


def replay(launches, label="graph_replay"):
    """A CUDA graph of recorded library launches is about to be replayed: count them, and time the replay
    under `label` when the active trace times anything.  Returns the end event to record, or None."""
    t = _active
    if t is None:
        return None
    t.launches.update(launches)
    if not t.timed:
        return None
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    t.events[label].append((a, b))
    return b
