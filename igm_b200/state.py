"""The shared state bag and its residency.

``State`` mirrors igm.common.State (igm/common/core/src.py:19-20): a plain
attribute bag.  The processes accept two residencies:

* device-resident (the fast path): 2-D/3-D fields are torch CUDA tensors;
  processes rebind attributes to new tensors, as the reference rebinds TF
  tensors;
* host-resident: ``state.thk`` is a numpy array.  Each process then copies
  the fields it reads to the device and writes the fields it produces back
  into pinned numpy arrays on the state; a host array the processes did not
  produce is replaced, on its first use, by a pinned array of the same values,
  so every copy is a DMA from pinned memory; within one process update
  (``update_scope``) a field is copied to the device once.  This is what a
  host-side caller of the plugin pays per step (``transfer_counts``).
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
    """One process update: inside it, each host field is copied to the device
    once -- further get() calls of the same field reuse that copy until the
    field is rebound by put() -- since no one else can change the host array
    while the update runs.  Scopes nest (the outermost one owns the copies)."""

    def __init__(self, state):
        self.state = state
        self.outer = False

    def __enter__(self):
        if "_igm_fetched" not in self.state.__dict__:
            self.state.__dict__["_igm_fetched"] = {}
            self.outer = True
        return self

    def __exit__(self, *exc):
        if self.outer:
            self.state.__dict__.pop("_igm_fetched", None)
        return False


def transfer_counts(state):
    """(host->device bytes, device->host bytes) the state's fields have been
    copied since the state was created or reset_transfer_counts() was called."""
    return int(state.__dict__.get("_igm_h2d_bytes", 0)), int(state.__dict__.get("_igm_d2h_bytes", 0))


def reset_transfer_counts(state):
    state.__dict__["_igm_h2d_bytes"] = 0
    state.__dict__["_igm_d2h_bytes"] = 0


def get(state, name, dtype=torch.float32):
    """Field ``name`` as a device tensor of ``dtype``."""
    v = getattr(state, name)
    dev = device(state)
    if isinstance(v, torch.Tensor):
        if v.is_cuda:
            return v if v.dtype == dtype else v.to(dtype)
        src = v
    else:
        src = None
        arr = np.asarray(v)
        pins = state.__dict__.get("_igm_pinned_views", {})
        t = pins.get(id(v))
        if t is not None and t.numpy() is not None and t.data_ptr() == arr.__array_interface__["data"][0]:
            src = t
        if src is None:
            # a host array the processes did not produce: copy it once into a pinned buffer and bind that
            # in its place (same values), so that every later step copies it to the device by DMA from
            # pinned memory, without a host-side staging copy
            src = _pinned(state, "in:" + name, arr.shape, torch.from_numpy(np.empty(0, arr.dtype)).dtype)
            src.numpy()[...] = arr
            view = src.numpy()
            state.__dict__.setdefault("_igm_pinned_views", {})[id(view)] = src
            setattr(state, name, view)
    fetched = state.__dict__.get("_igm_fetched")
    if fetched is not None and (name, dtype) in fetched:
        return fetched[(name, dtype)]
    out = src.to(dev, non_blocking=True).to(dtype)
    state.__dict__["_igm_h2d_bytes"] = state.__dict__.get("_igm_h2d_bytes", 0) + src.numel() * src.element_size()
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
    host.copy_(tensor, non_blocking=True)
    state.__dict__["_igm_d2h_bytes"] = state.__dict__.get("_igm_d2h_bytes", 0) + tensor.numel() * tensor.element_size()
    arr = host.numpy()
    state.__dict__.setdefault("_igm_pinned_views", {})[id(arr)] = host
    setattr(state, name, arr)


def sync_host(state):
    """Completes the device->host copies of a host-resident state."""
    if is_host(state):
        torch.cuda.current_stream().synchronize()
