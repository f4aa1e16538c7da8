"""Device plumbing: current stream handle and grow-only workspaces.

Workspaces are plain uint8 device tensors owned by the host layer and
passed to the C ABI, so the kernels themselves never allocate.
"""
from __future__ import annotations

import torch

_ws = {}


def stream_handle(device=None):
    return torch.cuda.current_stream(device).cuda_stream


def workspace(nbytes, device, slot="default"):
    """Return a uint8 device buffer of at least nbytes for the given slot."""
    key = (str(device), slot)
    buf = _ws.get(key)
    if buf is None or buf.numel() < nbytes:
        _ws.pop(key, None)
        buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
        _ws[key] = buf
    return buf


def workspace_refs():
    """References to every current workspace buffer (a captured CUDA graph
    holds these so that its baked-in pointers outlive slot growth)."""
    return list(_ws.values())


def release_workspaces():
    _ws.clear()


class StageTimer:
    """Records CUDA events between pipeline stages on the launching stream.

    While a timer is active (``with StageTimer() as t``) the force and force
    adjoint run as separate C-ABI stage calls with an event after each; the
    kernels launched are the same as the fused entry points'.  ``totals()``
    returns milliseconds per stage summed over all recorded launches."""

    active = None

    def __init__(self):
        self.events = []  # (name, start_event, end_event)
        self.counts = {}

    def __enter__(self):
        StageTimer.active = self
        return self

    def __exit__(self, *exc):
        StageTimer.active = None

    def mark(self, name, start):
        end = torch.cuda.Event(enable_timing=True)
        end.record()
        self.events.append((name, start, end))
        self.counts[name] = self.counts.get(name, 0) + 1
        return end

    def start(self):
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        return e

    def tag(self, name):
        """Count a variant of the last stage (no event): e.g. gathers that also kick."""
        self.counts[name] = self.counts.get(name, 0) + 1

    def totals(self):
        torch.cuda.synchronize()
        out = {}
        for name, s, e in self.events:
            out[name] = out.get(name, 0.0) + s.elapsed_time(e)
        return out


def ptr(t):
    return None if t is None else t.data_ptr()


def require_cuda(*tensors):
    for t in tensors:
        if t is not None and (not t.is_cuda):
            raise ValueError("pmpp_b200 kernels need CUDA tensors")
        if t is not None and not t.is_contiguous():
            raise ValueError("pmpp_b200 kernels need contiguous tensors")
