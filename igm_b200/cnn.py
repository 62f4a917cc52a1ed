"""The CNN velocity emulator on the device (neural_network.py:9-66).

All arithmetic runs in libigmb200: tensor-core 3x3 convolutions (BF16 in,
FP32 accumulate), the 1x1 head, the energy and its adjoint, and Adam.  Torch
tensors are only the device buffers.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib as L

F = 32  # filters of the hidden layers


def _p(t):
    return None if t is None else t.data_ptr()


class CNN:
    """nb_layers x [Conv2D 3x3 same (32) + LeakyReLU(alpha)] + Conv2D 1x1 -> nout.

    ``params`` is one fp32 vector in Keras order (kernel [3,3,cin,32], bias
    [32] per layer; head kernel [1,1,32,nout], bias [nout])."""

    def __init__(self, nb_layers=16, cin=5, nout=20, alpha=0.01, init="glorot_uniform", seed=0,
                 scales=(1.0, 1.0, 1.0, 1.0, 1.0), device="cuda", nb_out_filter=32, out_scale=1.0):
        if nb_out_filter != F:
            raise NotImplementedError(f"nb_out_filter={nb_out_filter}: only 32 filters are supported")
        if cin > 8:
            raise NotImplementedError("at most 8 input fields")
        self.L, self.cin, self.nout, self.alpha = int(nb_layers), int(cin), int(nout), float(alpha)
        self.out_scale = float(out_scale)  # the head's outputs are multiplied by this fixed factor
        self.nz = self.nout // 2
        self.device = torch.device(device)
        self.scales = np.asarray(list(scales) + [1.0] * (5 - len(scales)), dtype=np.float32)[:5]
        lib = L.lib()
        self.n_params = int(lib.igm_cnn_param_count(self.L, self.cin, self.nout))
        self.shapes = []  # Keras-ordered variable shapes
        for l in range(self.L):
            self.shapes += [(3, 3, self.cin if l == 0 else F, F), (F,)]
        self.shapes += [(1, 1, F, self.nout), (self.nout,)]
        offs = [0]
        for s in self.shapes:
            offs.append(offs[-1] + int(np.prod(s)))
        assert offs[-1] == self.n_params
        self.offsets = offs
        self.params = torch.zeros(self.n_params, dtype=torch.float32, device=self.device)
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        offs = (C.c_size_t * len(self.offsets))(*self.offsets)
        self.norms = torch.zeros(int(L.lib().igm_adam_norms_len(len(self.shapes), offs)), dtype=torch.float64,
                                 device=self.device)
        self.opt_iterations = 0
        self.wpack_f = torch.zeros(9 * 2 * F * 8 + (self.L - 1) * 9 * 4 * F * 8, dtype=torch.bfloat16,
                                   device=self.device)
        self.wpack_b = torch.zeros(max(self.L - 1, 1) * 9 * 4 * F * 8, dtype=torch.bfloat16, device=self.device)
        self.init_weights(init, seed)
        self._bufs = {}
        self.event_hook = None  # list: (start, end) CUDA events of each inference's 32-channel conv stack
        self._epoch = 0  # tile-flag epoch of the conv stack launches
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.n_sm = int(lib.igm_conv_sm_count())

    # ---- parameters ------------------------------------------------------
    def init_weights(self, init="glorot_uniform", seed=0, head_gain=1.0):
        """Keras initialisers: glorot_uniform (the reference default,
        iceflow.yaml weight_initialization) or he_normal / he_uniform; biases
        zero.  ``head_gain`` multiplies the head kernel's initial values."""
        rng = np.random.default_rng(seed)
        host = np.zeros(self.n_params, dtype=np.float32)
        for i, s in enumerate(self.shapes):
            if len(s) == 1:
                continue
            fan_in = s[0] * s[1] * s[2]
            fan_out = s[0] * s[1] * s[3]
            if init == "glorot_uniform":
                lim = math.sqrt(6.0 / (fan_in + fan_out))
                w = rng.uniform(-lim, lim, size=s)
            elif init == "he_normal":
                std = math.sqrt(2.0 / fan_in)
                w = np.clip(rng.normal(0, std, size=s), -2 * std, 2 * std)  # truncated normal
            elif init == "he_uniform":
                lim = math.sqrt(6.0 / fan_in)
                w = rng.uniform(-lim, lim, size=s)
            else:
                raise NotImplementedError(f"weight_initialization={init!r}")
            if i == len(self.shapes) - 2:
                w = w * head_gain
            host[self.offsets[i]:self.offsets[i + 1]] = w.astype(np.float32).ravel()
        self.set_params(host)

    def set_params(self, host):
        self.params.copy_(torch.as_tensor(np.asarray(host, dtype=np.float32)).to(self.device))
        self.pack()

    def get_variables(self):
        """Keras-ordered list of numpy arrays (kernel, bias, ...)."""
        h = self.params.cpu().numpy()
        return [h[self.offsets[i]:self.offsets[i + 1]].reshape(s) for i, s in enumerate(self.shapes)]

    def pack(self):
        L.check(L.lib().igm_cnn_pack_weights(self.L, self.cin, self.nout, _p(self.params), _p(self.wpack_f),
                                             _p(self.wpack_b), L.stream_ptr()), "igm_cnn_pack_weights")

    def _wf(self, l):
        off = 0 if l == 0 else 9 * 2 * F * 8 + (l - 1) * 9 * 4 * F * 8
        return self.wpack_f.data_ptr() + 2 * off

    def _wb(self, l):
        return self.wpack_b.data_ptr() + 2 * (l - 1) * 9 * 4 * F * 8

    def _b(self, l):
        return self.params.data_ptr() + 4 * self.offsets[2 * l + 1]

    def _w_off(self, l):
        return self.offsets[2 * l]

    # ---- buffers -----------------------------------------------------------
    def buffers(self, B, h, w, train):
        key = (B, h, w, train)
        b = self._bufs.get(key)
        if b is None:
            d = self.device
            act = lambda c: torch.empty((B, h, c // 8, w, 8), dtype=torch.bfloat16, device=d)
            b = {"acts": [act(F) for _ in range(self.L if train else 2)]}
            b["U"] = torch.empty((B, self.nz, h, w), dtype=torch.float32, device=d)
            b["V"] = torch.empty_like(b["U"])
            b["fields"] = [torch.empty((B, h, w), dtype=torch.float32, device=d) for _ in range(4)]
            b["X"] = act(16)  # split first-layer input (igm_cnn_input)
            if train:
                b["g"] = [act(F), act(F)]
                b["dyb"] = act(F)  # head output gradient in bf16 (head backward on the tensor cores)
                npart = self.n_sm
                b["npart"] = npart          # persistent tensor-core kernels: one CTA per SM
                b["npart2"] = 2 * npart     # head / first-layer reductions: two CTAs per SM
                wlen = max(int(L.lib().igm_conv3x3_wgrad_partial_len(F)), int(L.lib().igm_conv3x3_wgrad_partial_len(16)))
                b["wpart"] = torch.empty(npart * wlen, dtype=torch.float32, device=d)
                # the hidden layers' fused backward alternates between two partial buffers: each call
                # finishes the previous call's partials while it writes its own
                plen = int(L.lib().igm_conv3x3_wgrad_partial_len(F))
                b["wpart2"] = [torch.empty(npart * plen, dtype=torch.float32, device=d) for _ in range(2)]
                b["dbpart2"] = [torch.zeros((npart, F), dtype=torch.float32, device=d) for _ in range(2)]
                hl = int(L.lib().igm_cnn_head_partial_len(self.nz))
                b["hpart"] = torch.empty((2 * npart, hl), dtype=torch.float32, device=d)
            nst = max(self.L - 1, 1)
            b["flags"] = torch.zeros(int(L.lib().igm_conv3x3_stack_flags_len(B, h, w, nst)), dtype=torch.int32, device=d)
            self._bufs[key] = b
        return b

    # ---- forward -----------------------------------------------------------
    def prepare_input(self, fields_full, dx, windows, h, w, buf):
        """fields_full: [thk, usurf, arrhenius, slidingco] device [Ny, Nx]."""
        ny, nx = fields_full[0].shape
        B = len(windows)
        y0 = (C.c_int * B)(*[int(a) for a, _ in windows])
        x0 = (C.c_int * B)(*[int(b) for _, b in windows])
        sc = (C.c_float * 5)(*[float(s) for s in self.scales])
        rc = L.lib().igm_cnn_input(B, h, w, ny, nx, *[_p(f) for f in fields_full], float(dx), sc, y0, x0,
                                   _p(buf["X"]), *[_p(f) for f in buf["fields"]], L.stream_ptr())
        L.check(rc, "igm_cnn_input")
        buf["dx"] = float(dx)

    def _scales(self):
        return (C.c_float * 5)(*[float(s) for s in self.scales])

    def forward(self, buf, B, h, w, thk_mask=None, keep_acts=False):
        """Runs the network on the windowed fields of ``buf`` (prepare_input):
        the first layer on the split (x_h, x_l, x_h) input, the 3x3 layers, the
        head -- all convolutions on the tensor cores; U, V into buf."""
        lib, st = L.lib(), L.stream_ptr()
        acts = buf["acts"]
        rc = lib.igm_conv3x3(0, B, h, w, 16, _p(buf["X"]), self._wf(0), self._b(0), None, _p(acts[0]), None, 0,
                             self.alpha, _p(self.err), st)
        L.check(rc, "igm_conv3x3 layer 0")
        x = acts[0]
        if self.L > 1:
            # the 32-channel layers 1 .. L-1 in one launch (igm_conv3x3_stack)
            n = self.L - 1
            ys = [acts[l] if keep_acts else acts[l % 2] for l in range(1, self.L)]
            outs = (C.c_void_p * n)(*[_p(y) for y in ys])
            wps = (C.c_void_p * n)(*[self._wf(l) for l in range(1, self.L)])
            bs = (C.c_void_p * n)(*[self._b(l) for l in range(1, self.L)])
            self._epoch = self._epoch % 2147483646 + 1
            hook = self.event_hook if (self.event_hook is not None and not keep_acts) else None
            if hook is not None:
                ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                ev[0].record()
            rc = lib.igm_conv3x3_stack(B, h, w, n, _p(x), outs, wps, bs, _p(buf["flags"]), self._epoch, self.alpha,
                                       _p(self.err), st)
            L.check(rc, "igm_conv3x3_stack")
            if hook is not None:
                ev[1].record()
                hook.append(ev)
            x = ys[-1]
        hw = self.params.data_ptr() + 4 * self.offsets[2 * self.L]
        hb = self.params.data_ptr() + 4 * self.offsets[2 * self.L + 1]
        rc = lib.igm_cnn_head_forward(B, h, w, self.nz, _p(x), hw, hb, self.out_scale, _p(buf["U"]), _p(buf["V"]),
                                      _p(thk_mask), st)
        L.check(rc, "igm_cnn_head_forward")
        return buf["U"], buf["V"]

    # ---- backward ----------------------------------------------------------
    def backward(self, buf, B, h, w, dU, dV, field_grad=None, param_grads=True):
        """Gradients of the parameters into self.grads, given dE/dU, dE/dV
        (planar [B, nz, h, w]); requires forward(keep_acts=True).  With
        ``field_grad`` (float32 [B, n, h, w], n <= cin) also the gradient with
        respect to the first n raw input fields (igm_cnn_input_gradient); ``param_grads=False``
        runs only the data-gradient chain (self.grads is then not written)."""
        lib, st = L.lib(), L.stream_ptr()
        acts = buf["acts"]
        npart, npart2 = buf["npart"], buf["npart2"]
        hw = self.params.data_ptr() + 4 * self.offsets[2 * self.L]
        hl = buf["hpart"].shape[1]
        g = buf["g"]
        gp = self.grads.data_ptr()
        nh = F * self.nout
        if self.nout <= F:
            # pixel part on CUDA cores, the head kernel gradient A16^T dY on the tensor cores
            # data-only backward: no bf16 dY for the head's weight gradient, no partial sums
            rc = lib.igm_cnn_head_backward_tc(B, h, w, self.nz, _p(acts[self.L - 1]), hw, _p(dU), _p(dV),
                                              self.out_scale, self.alpha, _p(g[0]),
                                              _p(buf["dyb"]) if param_grads else None,
                                              _p(buf["hpart"]) if param_grads else None, npart2, st)
            L.check(rc, "igm_cnn_head_backward_tc")
        if self.nout <= F and param_grads:
            stride = self.nout + F
            L.check(lib.igm_reduce_partials(_p(buf["hpart"]), npart2, self.nout, stride,
                                            gp + 4 * self.offsets[2 * self.L + 1], 0, st), "reduce head bias")
            L.check(lib.igm_reduce_partials(buf["hpart"].data_ptr() + 4 * self.nout, npart2, F, stride,
                                            gp + 4 * self.offsets[2 * (self.L - 1) + 1], 0, st), "reduce db")
            rc = lib.igm_conv1x1_wgrad(B, h, w, _p(acts[self.L - 1]), _p(buf["dyb"]), _p(buf["wpart"]), npart,
                                       _p(self.err), st)
            L.check(rc, "igm_conv1x1_wgrad head")
            L.check(lib.igm_cnn_head_wgrad_finish(_p(buf["wpart"]), npart, self.nout, gp + 4 * self.offsets[2 * self.L],
                                                  st), "igm_cnn_head_wgrad_finish")
        elif self.nout > F:
            rc = lib.igm_cnn_head_backward(B, h, w, self.nz, _p(acts[self.L - 1]), hw, _p(dU), _p(dV),
                                           self.out_scale, self.alpha, _p(g[0]), _p(buf["hpart"]), npart2, st)
            L.check(rc, "igm_cnn_head_backward")
            if param_grads:
                # head kernel + bias gradients, last conv layer's bias gradient
                L.check(lib.igm_reduce_partials(_p(buf["hpart"]), npart2, nh + self.nout, hl,
                                                gp + 4 * self.offsets[2 * self.L], 0, st), "reduce head")
                L.check(lib.igm_reduce_partials(buf["hpart"].data_ptr() + 4 * (nh + self.nout), npart2, F, hl,
                                                gp + 4 * self.offsets[2 * (self.L - 1) + 1], 0, st), "reduce db")
        cur = 0
        prev = None  # the hidden layer whose partials the next fused call finishes
        for l in range(self.L - 1, -1, -1):
            gl = g[cur]
            if l > 0 and param_grads:
                # both gradients of the layer in one pass (igm_conv3x3_backward), which also finishes
                # the layer above's weight and bias gradients from the previous call's partials
                nxt = g[1 - cur]
                wp, dbp = buf["wpart2"][l % 2], buf["dbpart2"][l % 2]
                if prev is None:
                    fin = (None, None, None, None)
                else:
                    fin = (_p(buf["wpart2"][prev % 2]), _p(buf["dbpart2"][prev % 2]), gp + 4 * self.offsets[2 * prev],
                           gp + 4 * self.offsets[2 * (prev - 1) + 1])
                rc = lib.igm_conv3x3_backward(B, h, w, _p(gl), self._wb(l), _p(acts[l - 1]), _p(nxt), _p(dbp), _p(wp),
                                              npart, self.alpha, _p(self.err), *fin, st)
                L.check(rc, f"igm_conv3x3_backward layer {l}")
                prev = l
                cur = 1 - cur
                continue
            if prev is not None and param_grads:
                # the last fused call's partials (layer 1)
                L.check(lib.igm_cnn_wgrad_finish(_p(buf["wpart2"][prev % 2]), npart, F, F,
                                                 gp + 4 * self.offsets[2 * prev], st), "igm_cnn_wgrad_finish")
                L.check(lib.igm_reduce_partials(_p(buf["dbpart2"][prev % 2]), npart, F, F,
                                                gp + 4 * self.offsets[2 * (prev - 1) + 1], 0, st), "reduce db")
                prev = None
            if l == 0:
                if field_grad is not None:
                    ng = int(field_grad.shape[1])
                    if field_grad.shape != (B, ng, h, w) or not field_grad.is_contiguous() or ng > self.cin:
                        raise ValueError("field_grad must be contiguous float32 [B, n <= cin, h, w]")
                    sc = (C.c_double * ng)(*[float(x) for x in self.scales[:ng]])
                    rc = lib.igm_cnn_input_gradient(B, h, w, self.cin, ng, _p(gl), self.params.data_ptr(), sc,
                                                    _p(field_grad), st)
                    L.check(rc, "igm_cnn_input_gradient")
                if param_grads:
                    rc = lib.igm_conv3x3_wgrad(B, h, w, 16, _p(buf["X"]), _p(gl), _p(buf["wpart"]), npart,
                                               _p(self.err), st)
                    L.check(rc, "igm_conv3x3_wgrad layer 0")
                    rc = lib.igm_cnn_wgrad_finish_split(_p(buf["wpart"]), npart, self.cin, gp + 4 * self.offsets[0],
                                                        st)
                    L.check(rc, "igm_cnn_wgrad_finish_split")
            if l > 0:
                # the data gradient alone (no parameter gradients wanted)
                nxt = g[1 - cur]
                rc = lib.igm_conv3x3(1, B, h, w, F, _p(gl), self._wb(l), None, _p(acts[l - 1]), _p(nxt), None, npart,
                                     self.alpha, _p(self.err), st)
                L.check(rc, f"igm_conv3x3 dgrad layer {l}")
                cur = 1 - cur

    def adam_step(self, lr, beta_1=0.9, beta_2=0.999, epsilon=1e-7, clipnorm=1.0):
        """Keras legacy Adam with per-variable clipnorm; repacks the weights."""
        self.opt_iterations += 1
        offs = (C.c_size_t * len(self.offsets))(*self.offsets)
        rc = L.lib().igm_adam_clipnorm(len(self.shapes), offs, _p(self.params), _p(self.grads), _p(self.m),
                                       _p(self.v), _p(self.norms), float(lr), float(beta_1), float(beta_2),
                                       float(epsilon), float(clipnorm if clipnorm else 0.0),
                                       int(self.opt_iterations), L.stream_ptr())
        L.check(rc, "igm_adam_clipnorm")
        self.pack()

    def check_errors(self):
        e = int(self.err.item())
        if e != 0:
            self.err.zero_()
            raise L.IgmError(5, f"tensor-core pipeline wait timed out (code {e})")
