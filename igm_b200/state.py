"""The shared state bag and its residency.

``State`` mirrors igm.common.State (igm/common/core/src.py:19-20): a plain
attribute bag.  The processes accept two residencies:

* device-resident (the fast path): 2-D/3-D fields are torch CUDA tensors;
  processes rebind attributes to new tensors, as the reference rebinds TF
  tensors;
* host-resident: ``state.thk`` is a numpy array.  A process reads a host
  field through a device copy and writes the fields it produces back into
  pinned numpy arrays on the state:

  - a host array the processes did not produce is replaced, on its first
    use, by a pinned array of the same values, so every copy is a DMA from
    pinned memory;
  - the state keeps the device copy of every host field it copied or
    produced, and copies a field to the device again only when the caller
    has rebound it (as the reference's tensors change: by rebinding) or
    declared it changed in place with ``invalidate``;
  - results go back to the host on a side stream, issued when the process
    update ends and overlapping the processes that follow; the host arrays
    hold the results once ``sync_host`` has returned (the processes do not
    wait for the copies themselves).  A device tensor bound by put() is not
    written in place afterwards, except through get(..., writable=True).

  ``transfer_counts`` gives the bytes copied each way.
"""

from __future__ import annotations

import numpy as np
import torch


class State:
    pass


def is_host(state) -> bool:
    return isinstance(getattr(state, "thk", None), np.ndarray)


def device(state):
    d = getattr(state, "device", None)
    if d is not None:
        return torch.device(d)
    t = getattr(state, "thk", None)
    if isinstance(t, torch.Tensor) and t.is_cuda:
        return t.device
    return torch.device("cuda", torch.cuda.current_device())


def _pinned(state, name, shape, dtype):
    cache = state.__dict__.setdefault("_igm_pinned", {})
    key = (name, tuple(shape), dtype)
    buf = cache.get(key)
    if buf is None:
        buf = torch.empty(shape, dtype=dtype, pin_memory=True)
        cache[key] = buf
    return buf


class update_scope:
    """One process update: inside it, get() returns one device tensor per
    field and dtype (a converted copy is made once) until put() rebinds the
    field, and the device->host copies of the fields put() binds are issued
    together when the scope ends.  Scopes nest (the outermost one owns the
    copies)."""

    def __init__(self, state):
        self.state = state
        self.outer = False

    def __enter__(self):
        if "_igm_fetched" not in self.state.__dict__:
            self.state.__dict__["_igm_fetched"] = {}
            self.state.__dict__["_igm_pending"] = []
            self.outer = True
        return self

    def __exit__(self, *exc):
        if self.outer:
            self.state.__dict__.pop("_igm_fetched", None)
            _issue_copies(self.state.__dict__.pop("_igm_pending", []))
        return False


def transfer_counts(state):
    """(host->device bytes, device->host bytes) the state's fields have been
    copied since the state was created or reset_transfer_counts() was called."""
    return int(state.__dict__.get("_igm_h2d_bytes", 0)), int(state.__dict__.get("_igm_d2h_bytes", 0))


def reset_transfer_counts(state):
    state.__dict__["_igm_h2d_bytes"] = 0
    state.__dict__["_igm_d2h_bytes"] = 0


def _stream_index(dev) -> int:
    return dev.index if dev.index is not None else torch.cuda.current_device()


_COPY_STREAMS: dict = {}


def _copy_stream(dev):
    """The side stream that carries a device's device->host result copies."""
    i = _stream_index(dev)
    s = _COPY_STREAMS.get(i)
    if s is None:
        s = _COPY_STREAMS[i] = torch.cuda.Stream(device=i)
    return s


def _issue_copies(pairs):
    """Copies (pinned host buffer, device tensor) pairs device->host on the
    side stream, after the work the current stream has queued so far; the
    copy stream holds on to each tensor's memory until its copy is done."""
    if not pairs:
        return
    dev = pairs[0][1].device
    cs = _copy_stream(dev)
    cs.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(cs):
        for host, t in pairs:
            host.copy_(t, non_blocking=True)
    for _, t in pairs:
        t.record_stream(cs)
    pairs.clear()


def invalidate(state, *names):
    """Declares host fields changed in place by the caller (all fields when no
    name is given): their next use copies them to the device again.  A field
    rebound to another array needs no call."""
    mirror = state.__dict__.get("_igm_mirror", {})
    fetched = state.__dict__.get("_igm_fetched")
    for n in (names or list(mirror)):
        mirror.pop(n, None)
        if fetched is not None:
            for key in [k for k in fetched if k[0] == n]:
                del fetched[key]


def get(state, name, dtype=torch.float32, writable=False):
    """Field ``name`` as a device tensor of ``dtype``.  A caller that writes
    into it in place (and then binds it with put()) passes writable=True: its
    writes then follow the device->host copies of the field still running."""
    v = getattr(state, name)
    if isinstance(v, torch.Tensor) and v.is_cuda:
        return v if v.dtype == dtype else v.to(dtype)
    dev = device(state)
    if writable:
        _issue_copies(state.__dict__.get("_igm_pending", []))
        cs = _COPY_STREAMS.get(_stream_index(dev))
        if cs is not None:
            torch.cuda.current_stream(dev).wait_stream(cs)
    fetched = state.__dict__.get("_igm_fetched")
    if fetched is not None and (name, dtype) in fetched:
        return fetched[(name, dtype)]
    mirror = state.__dict__.setdefault("_igm_mirror", {})
    m = mirror.get(name)
    if m is not None and m[0] is v:
        out = m[1]  # the device copy of this very host array
    else:
        if isinstance(v, torch.Tensor):
            src = v
        else:
            arr = np.asarray(v)
            pv = state.__dict__.get("_igm_pinned_views", {}).get(name)
            src = pv[1] if pv is not None and pv[0] is v else None  # an array the state bound: pinned
            if src is None:
                # a host array the processes did not produce: copy it once into a pinned buffer and bind
                # that in its place (same values), so that every later copy to the device is a DMA from
                # pinned memory, without a host-side staging copy
                key = ("in:" + name, tuple(arr.shape), torch.from_numpy(np.empty(0, arr.dtype)).dtype)
                if key in state.__dict__.get("_igm_pinned", {}):
                    # the buffer held an earlier array of this field: its copies to the device are done first
                    torch.cuda.current_stream(dev).synchronize()
                src = _pinned(state, *key)
                src.numpy()[...] = arr
                view = src.numpy()
                state.__dict__.setdefault("_igm_pinned_views", {})[name] = (view, src)
                setattr(state, name, view)
        cs = _COPY_STREAMS.get(_stream_index(dev))
        if cs is not None:
            # a result copy into this pinned buffer may still be running on the side stream
            torch.cuda.current_stream(dev).wait_stream(cs)
        out = src.to(dev, non_blocking=True)
        state.__dict__["_igm_h2d_bytes"] = state.__dict__.get("_igm_h2d_bytes", 0) + src.numel() * src.element_size()
        mirror[name] = (getattr(state, name), out)
    if out.dtype != dtype:
        out = out.to(dtype)
    if fetched is not None:
        fetched[(name, dtype)] = out
    return out


def put(state, name, tensor):
    """Bind ``tensor`` (device) to ``state.name`` in the state's residency."""
    if not is_host(state):
        setattr(state, name, tensor)
        return
    fetched = state.__dict__.get("_igm_fetched")
    if fetched is not None:
        for key in [k for k in fetched if k[0] == name]:
            del fetched[key]
    host = _pinned(state, "out:" + name, tensor.shape, tensor.dtype)
    pending = state.__dict__.get("_igm_pending")
    if pending is not None:
        pending.append((host, tensor))  # issued with the update's other results when its scope ends
    else:
        _issue_copies([(host, tensor)])
    state.__dict__["_igm_d2h_bytes"] = state.__dict__.get("_igm_d2h_bytes", 0) + tensor.numel() * tensor.element_size()
    arr = host.numpy()
    state.__dict__.setdefault("_igm_pinned_views", {})[name] = (arr, host)
    setattr(state, name, arr)
    state.__dict__.setdefault("_igm_mirror", {})[name] = (arr, tensor)


def sync_host(state):
    """Waits for the device->host copies of a host-resident state: its host
    arrays then hold the processes' results."""
    if is_host(state) and torch.cuda.is_initialized():
        _issue_copies(state.__dict__.get("_igm_pending", []))
        dev = device(state)
        torch.cuda.current_stream(dev).synchronize()
        cs = _COPY_STREAMS.get(_stream_index(dev))
        if cs is not None:
            cs.synchronize()
