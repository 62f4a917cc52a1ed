"""A minimal TensorFlow-API shim over torch, used only by ``make_golden.py``.

TensorFlow 2.15 (the reference's backend) cannot be installed in this
environment, so the reference's own source files for the hot path are
executed against this shim instead: every ``tf.*`` call they make is mapped
to the torch op with the same semantics, ``tf.GradientTape`` to torch
autograd, and ``tf.keras.optimizers.legacy.Adam`` to the published Adam
update in the form TF's ``ApplyAdam`` kernel evaluates it.  Only the subset
of the API that those files use is provided.
"""

from __future__ import annotations

import sys
import types

import numpy as np
import torch

__version__ = "2.15.1"

float32 = torch.float32
float64 = torch.float64
int32 = torch.int32

_DT = {"float32": torch.float32, "float64": torch.float64, "int32": torch.int32,
       torch.float32: torch.float32, torch.float64: torch.float64, torch.int32: torch.int32,
       None: None}


def _dt(d):
    return _DT[d] if d in _DT else d


def _as(x, like=None):
    if isinstance(x, torch.Tensor):
        return x
    if like is not None and isinstance(like, torch.Tensor):
        return torch.as_tensor(x, dtype=like.dtype)
    a = np.asarray(x)
    if a.dtype == np.float64 and like is None:
        return torch.as_tensor(a, dtype=torch.float32)
    return torch.as_tensor(a)


def function(*args, **kwargs):
    if len(args) == 1 and callable(args[0]) and not kwargs:
        return args[0]
    return lambda f: f


def _assign(t):
    def assign(v):
        with torch.no_grad():
            t.copy_(_as(v, t))
        return t
    t.assign = assign
    return t


def Variable(x, dtype=None, trainable=True, **kw):
    t = _as(x).detach().clone()
    if dtype is not None:
        t = t.to(_dt(dtype))
    if t.dtype in (torch.float32, torch.float64) and trainable:
        t.requires_grad_(True)
    return _assign(t)


def constant(x, dtype=None):
    t = _as(x)
    return t.to(_dt(dtype)) if dtype is not None else t


def convert_to_tensor(x, dtype=None):
    return constant(x, dtype)


def cast(x, dtype):
    return _as(x).to(_dt(dtype))


def range(n, *a, dtype=None):
    return torch.arange(n, *a, dtype=torch.float64 if dtype is None else _dt(dtype))


def zeros(shape, dtype=torch.float32):
    return torch.zeros(shape, dtype=_dt(dtype))


def ones(shape, dtype=torch.float32):
    return torch.ones(shape, dtype=_dt(dtype))


def zeros_like(x):
    return torch.zeros_like(x)


def ones_like(x):
    return torch.ones_like(x)


def maximum(a, b):
    a = _as(a, b if isinstance(b, torch.Tensor) else None)
    return torch.maximum(a, _as(b, a))


def minimum(a, b):
    a = _as(a, b if isinstance(b, torch.Tensor) else None)
    return torch.minimum(a, _as(b, a))


def where(c, a, b):
    like = a if isinstance(a, torch.Tensor) else b
    return torch.where(c, _as(a, like), _as(b, like))


def clip_by_value(x, lo, hi):
    x = _as(x)
    npdt = np.float32 if x.dtype == torch.float32 else np.float64
    with np.errstate(over="ignore"):
        lo_t = torch.as_tensor(npdt(lo), dtype=x.dtype)
        hi_t = torch.as_tensor(npdt(hi), dtype=x.dtype)
    return torch.clamp(x, min=lo_t, max=hi_t)


def reduce_sum(x, axis=None):
    return torch.sum(x) if axis is None else torch.sum(x, dim=axis)


def reduce_mean(x, axis=None):
    return torch.mean(x) if axis is None else torch.mean(x, dim=axis)


def reduce_max(x, axis=None):
    return torch.max(x) if axis is None else torch.amax(x, dim=axis)


def reduce_min(x, axis=None):
    return torch.min(x) if axis is None else torch.amin(x, dim=axis)


def add_n(xs):
    out = xs[0]
    for x in xs[1:]:
        out = out + x
    return out


def abs(x):  # noqa: A001
    return torch.abs(x)


def sqrt(x):
    return torch.sqrt(x)


def less(a, b):
    return a < b


def concat(xs, axis):
    like = next(x for x in xs if isinstance(x, torch.Tensor))
    return torch.cat([_as(x, like) for x in xs], dim=axis)


def cumsum(x, axis=0):
    """Inclusive scan accumulated in the tensor's own dtype, one slice after
    the other along ``axis`` (TF's kernel; torch.cumsum on CPU accumulates
    float32 in double)."""
    import builtins
    x = _as(x)
    parts = [x.narrow(axis, 0, 1)]
    for i in builtins.range(1, x.shape[axis]):
        parts.append(parts[-1] + x.narrow(axis, i, 1))
    return torch.cat(parts, dim=axis)


def stack(xs, axis=0):
    return torch.stack([_as(x) for x in xs], dim=axis)


def expand_dims(x, axis):
    return torch.unsqueeze(x, axis)


def einsum(eq, *xs):
    return torch.einsum(eq, *xs)


def norm(x, axis=None):
    return torch.linalg.vector_norm(x, dim=axis)


def pad(x, paddings, mode="CONSTANT", constant_values=0):
    flat = []
    for p in reversed(paddings):
        flat += [int(p[0]), int(p[1])]
    if mode.upper() == "CONSTANT":
        return torch.nn.functional.pad(x, flat, value=constant_values)
    if mode.upper() == "SYMMETRIC":
        out = x
        for dim, (lo, hi) in enumerate(paddings):
            lo, hi = int(lo), int(hi)
            if lo == 0 and hi == 0:
                continue
            parts = []
            if lo:
                parts.append(torch.flip(out.narrow(dim, 0, lo), [dim]))
            parts.append(out)
            if hi:
                parts.append(torch.flip(out.narrow(dim, out.shape[dim] - hi, hi), [dim]))
            out = torch.cat(parts, dim=dim)
        return out
    raise NotImplementedError(mode)


def _conv2d(x, k, strides=None, padding="SAME"):
    """tf.nn.conv2d, NHWC input and HWIO filter, stride 1, SAME or VALID padding."""
    xt = x.permute(0, 3, 1, 2)
    kt = k.permute(3, 2, 0, 1).to(xt.dtype)
    pad = (k.shape[0] // 2) if padding == "SAME" else 0
    y = torch.nn.functional.conv2d(xt, kt, padding=pad)
    return y.permute(0, 2, 3, 1)


math = types.SimpleNamespace(is_nan=torch.isnan, reduce_mean=lambda x, axis=None: reduce_mean(x, axis),
                             reduce_sum=lambda x, axis=None: reduce_sum(x, axis), log=torch.log)
nn = types.SimpleNamespace(l2_loss=lambda x: torch.sum(x * x) / 2, conv2d=_conv2d)


def squeeze(x, axis=None):
    return torch.squeeze(x) if axis is None else torch.squeeze(x, axis)


experimental = types.SimpleNamespace(numpy=types.SimpleNamespace(
    moveaxis=lambda x, src, dst: torch.movedim(x, src, dst)))

linalg = types.SimpleNamespace(
    global_norm=lambda gs: torch.sqrt(sum(torch.sum(g.detach().to(torch.float64) ** 2) for g in gs)))


class GradientTape:
    def __init__(self, persistent=False):
        self.persistent = persistent

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False

    def watch(self, x):
        pass

    def gradient(self, target, sources, output_gradients=None):
        gs = torch.autograd.grad(target, list(sources), grad_outputs=output_gradients,
                                 retain_graph=True, allow_unused=True)
        return [torch.zeros_like(s) if g is None else g for g, s in zip(gs, sources)]


class _LegacyAdam:
    """TF ApplyAdam semantics with OptimizerV2's per-variable clipnorm."""

    def __init__(self, learning_rate=0.001, beta_1=0.9, beta_2=0.999, epsilon=1e-7, clipnorm=None, **kw):
        self.lr = learning_rate
        self.beta_1, self.beta_2, self.epsilon, self.clipnorm = beta_1, beta_2, epsilon, clipnorm
        self.iterations = 0
        self._slots = {}

    def apply_gradients(self, grads_and_vars):
        grads_and_vars = list(grads_and_vars)
        t = self.iterations + 1
        with torch.no_grad():
            for g, x in grads_and_vars:
                dt = x.dtype
                if self.clipnorm is not None:
                    n = torch.sqrt(torch.sum(g.to(torch.float64) ** 2)).to(dt)
                    g = g * self.clipnorm / torch.maximum(n, torch.tensor(self.clipnorm, dtype=dt))
                # keyed by the variable object (held in the slot so its id is never reused)
                if id(x) not in self._slots or self._slots[id(x)][0] is not x:
                    self._slots[id(x)] = (x, torch.zeros_like(x), torch.zeros_like(x))
                _, m, v = self._slots[id(x)]
                one = torch.tensor(1.0, dtype=dt)
                alpha = float(self.lr) * torch.sqrt(one - torch.tensor(self.beta_2, dtype=dt) ** t) / (
                    one - torch.tensor(self.beta_1, dtype=dt) ** t)
                m += (g - m) * (1 - self.beta_1)
                v += (g * g - v) * (1 - self.beta_2)
                x -= (m * alpha) / (torch.sqrt(v) + self.epsilon)
        self.iterations += 1


keras = types.SimpleNamespace(optimizers=types.SimpleNamespace(
    Adam=_LegacyAdam, legacy=types.SimpleNamespace(Adam=_LegacyAdam)))

newaxis = None


def install():
    """Register this module as ``tensorflow`` and stub the plotting imports."""
    sys.modules["tensorflow"] = sys.modules[__name__]
    mpl = types.ModuleType("matplotlib")
    mpl.colors = types.SimpleNamespace(LogNorm=lambda **k: None)
    plt = types.ModuleType("matplotlib.pyplot")
    mpl.pyplot = plt
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", plt)
    sys.modules.setdefault("importlib_resources", types.ModuleType("importlib_resources"))
    # TF tensors expose .numpy() whether or not they are watched by a tape.
    if not getattr(torch.Tensor, "_shim_numpy", False):
        orig = torch.Tensor.numpy
        torch.Tensor.numpy = lambda self, *a, **k: orig(self.detach(), *a, **k)
        torch.Tensor._shim_numpy = True
