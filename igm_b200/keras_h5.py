"""Loader and writer for the Keras HDF5 model files the reference ships and
saves (``tf.keras.models.load_model(".../model.h5")``, emulate.py:64-93, and
``save_iceflow_model``, emulate.py:331-359), without h5py or TensorFlow.

It implements the part of the HDF5 file format (superblock version 0/1,
version-1 object headers, symbol-table groups with version-1 B-trees and local
heaps, compact and contiguous dataset storage, fixed-length and variable-length
(global heap) string attributes, IEEE float and integer datasets) that h5py writes for a Keras model with the
library's default settings, and walks the Keras layout: the group
``model_weights`` (or the root of a weights-only file) lists its layers in the
attribute ``layer_names``, each layer group lists its tensors in
``weight_names``.  Anything outside that subset (chunked or filtered storage,
other variable-length data, version-2 object headers) raises ``NotImplementedError``
naming what was found.

Host-side file parsing only: the weights are then packed for the tensor-core
kernels by ``igm_b200.cnn.CNN.set_params``.
"""

from __future__ import annotations

import numpy as np

_SIG = b"\x89HDF\r\n\x1a\n"


class H5Error(ValueError):
    pass


class _File:
    def __init__(self, path: str):
        with open(path, "rb") as f:
            self.b = f.read()
        b = self.b
        if b[:8] != _SIG:
            raise H5Error(f"{path}: not an HDF5 file")
        ver = b[8]
        if ver not in (0, 1):
            raise NotImplementedError(f"{path}: HDF5 superblock version {ver} (only 0 and 1 are read)")
        self.so, self.sl = b[13], b[14]
        p = 24 + (4 if ver == 1 else 0)
        self.base = self.off(p)
        p += 4 * self.so  # base, free-space, end-of-file and driver addresses
        # root group symbol table entry: link name offset, object header address
        self.root = self.off(p + self.so)

    # ---- primitive readers
    def u(self, p, n):
        return int.from_bytes(self.b[p:p + n], "little")

    def off(self, p):
        return self.u(p, self.so)

    def undefined(self, a):
        return a == (1 << (8 * self.so)) - 1

    # ---- object headers
    def messages(self, addr):
        """(type, data offset, data size) of every message of a version-1 object header."""
        b = self.b
        if b[addr] != 1:
            raise NotImplementedError(f"object header version {b[addr]} at {addr} (only version 1 is read)")
        nmsg = self.u(addr + 2, 2)
        size = self.u(addr + 8, 4)
        blocks = [(addr + 16, size)]
        out = []
        while blocks and len(out) < nmsg:
            p, n = blocks.pop(0)
            end = p + n
            while p + 8 <= end and len(out) < nmsg:
                mtype, msize = self.u(p, 2), self.u(p + 2, 2)
                data = p + 8
                if mtype == 0x10:  # continuation
                    blocks.append((self.off(data), self.u(data + self.so, self.sl)))
                out.append((mtype, data, msize))
                p = data + msize
        return out

    # ---- datatype / dataspace
    def datatype(self, p):
        cls = self.b[p] & 0x0F
        bits = self.b[p + 1:p + 4]
        size = self.u(p + 4, 4)
        if cls == 1:  # IEEE float
            if bits[0] & 1:
                raise NotImplementedError("big-endian floating point data")
            return np.dtype({4: "<f4", 8: "<f8", 2: "<f2"}[size])
        if cls == 0:  # fixed point
            signed = bool(bits[0] & 0x08)
            big = bool(bits[0] & 1)
            return np.dtype(("%s%s%d" % (">" if big else "<", "i" if signed else "u", size)))
        if cls == 3:  # fixed-length string
            return np.dtype("S%d" % size)
        raise NotImplementedError(f"HDF5 datatype class {cls}")

    def _datatype_or_none(self, p):
        try:
            return self.datatype(p)
        except NotImplementedError:
            return None

    def dataspace(self, p):
        ver, nd, flags = self.b[p], self.b[p + 1], self.b[p + 2]
        q = p + (8 if ver == 1 else 4)
        if ver == 2 and self.b[p + 3] == 0:  # scalar
            return ()
        return tuple(self.u(q + i * self.sl, self.sl) for i in range(nd))

    # ---- attributes
    def attributes(self, addr):
        out = {}
        for mtype, p, _ in self.messages(addr):
            if mtype != 0x0C:
                continue
            ver = self.b[p]
            nlen, tlen, slen = self.u(p + 2, 2), self.u(p + 4, 2), self.u(p + 6, 2)
            if ver == 1:
                q = p + 8
                pad = lambda n: (n + 7) // 8 * 8  # noqa: E731
                name = self.b[q:q + nlen].rstrip(b"\x00").decode()
                q += pad(nlen)
                q_dt = q
                dt = self._datatype_or_none(q)
                q += pad(tlen)
                shape = self.dataspace(q)
                q += pad(slen)
            elif ver in (2, 3):
                q = p + (9 if ver == 3 else 8)
                name = self.b[q:q + nlen].rstrip(b"\x00").decode()
                q += nlen
                q_dt = q
                dt = self._datatype_or_none(q)
                q += tlen
                shape = self.dataspace(q)
                q += slen
            else:
                raise NotImplementedError(f"attribute message version {ver}")
            n = int(np.prod(shape)) if shape else 1
            if dt is None and self._is_vlen_string(q_dt):
                out[name] = np.array(self._vlen_strings(q, n), dtype=object).reshape(shape)
                continue
            if dt is None:
                continue  # an attribute type the Keras weight layout does not need
            out[name] = np.frombuffer(self.b, dtype=dt, count=n, offset=q).reshape(shape)
        return out

    # ---- variable-length strings (global heap)
    def _is_vlen_string(self, p):
        return (self.b[p] & 0x0F) == 9 and (self.b[p + 1] & 0x0F) == 1

    def _gheap_object(self, coll, index):
        b = self.b
        if b[coll:coll + 4] != b"GCOL":
            raise H5Error(f"bad global heap signature at {coll}")
        size = self.u(coll + 8, self.sl)
        p, end = coll + 8 + self.sl, coll + size
        while p + 8 + self.sl <= end:
            idx, osz = self.u(p, 2), self.u(p + 8, self.sl)
            data = p + 8 + self.sl
            if idx == index:
                return self.b[data:data + osz]
            if idx == 0:
                break
            p = data + (osz + 7) // 8 * 8
        raise H5Error(f"global heap object {index} not found in collection {coll}")

    def _vlen_strings(self, q, n):
        out, step = [], 4 + self.so + 4
        for i in range(n):
            e = q + i * step
            length, coll, idx = self.u(e, 4), self.off(e + 4), self.u(e + 4 + self.so, 4)
            out.append(self._gheap_object(coll, idx)[:length].decode())
        return out

    # ---- groups
    def children(self, addr):
        """{name: object header address} of a symbol-table group."""
        btree = heap = None
        for mtype, p, _ in self.messages(addr):
            if mtype == 0x11:
                btree, heap = self.off(p), self.off(p + self.so)
        if btree is None:
            raise NotImplementedError(f"object at {addr} is not a symbol-table group")
        if self.b[heap:heap + 4] != b"HEAP":
            raise H5Error("bad local heap signature")
        data = self.off(heap + 8 + 2 * self.sl)
        out = {}

        def name_at(o):
            e = self.b.index(b"\x00", data + o)
            return self.b[data + o:e].decode()

        def walk(node):
            b = self.b
            if b[node:node + 4] == b"TREE":
                level, used = b[node + 5], self.u(node + 6, 2)
                p = node + 8 + 2 * self.so + self.sl  # past siblings and key 0
                for _ in range(used):
                    walk(self.off(p))
                    p += self.so + self.sl
            elif b[node:node + 4] == b"SNOD":
                n = self.u(node + 6, 2)
                p = node + 8
                for _ in range(n):
                    out[name_at(self.off(p))] = self.off(p + self.so)
                    p += 2 * self.so + 24
            else:
                raise H5Error(f"bad group node signature at {node}")

        walk(btree)
        return out

    # ---- datasets
    def dataset(self, addr):
        dt = shape = None
        layout = None
        for mtype, p, _ in self.messages(addr):
            if mtype == 0x03:
                dt = self.datatype(p)
            elif mtype == 0x01:
                shape = self.dataspace(p)
            elif mtype == 0x08:
                layout = p
            elif mtype == 0x0B:
                raise NotImplementedError("filtered (compressed) dataset storage")
        if dt is None or shape is None or layout is None:
            raise H5Error(f"object at {addr} is not a dataset")
        n = int(np.prod(shape)) if shape else 1
        ver = self.b[layout]
        if ver == 3:
            cls = self.b[layout + 1]
            if cls == 0:  # compact
                q = layout + 4
            elif cls == 1:  # contiguous
                a = self.off(layout + 2)
                if self.undefined(a):
                    return np.zeros(shape, dt)
                q = self.base + a
            else:
                raise NotImplementedError("chunked dataset storage")
        elif ver in (1, 2):
            nd, cls = self.b[layout + 1], self.b[layout + 2]
            if cls == 1:
                a = self.off(layout + 8)
                if self.undefined(a):
                    return np.zeros(shape, dt)
                q = self.base + a
            elif cls == 0:
                q = layout + 8 + 4 * nd + 4
            else:
                raise NotImplementedError("chunked dataset storage")
        else:
            raise NotImplementedError(f"data layout message version {ver}")
        return np.frombuffer(self.b, dtype=dt, count=n, offset=q).reshape(shape).copy()

    def lookup(self, path):
        addr = self.root
        for part in [p for p in path.split("/") if p]:
            kids = self.children(addr)
            if part not in kids:
                raise KeyError(path)
            addr = kids[part]
        return addr


def _strings(a):
    return [x.decode() if isinstance(x, bytes) else str(x) for x in np.asarray(a).reshape(-1)]


def read_keras_weights(path: str):
    """The weights of a Keras HDF5 model file, in the model's layer order:
    a list of (layer name, [(weight name, float array), ...]) with each array
    in Keras's own layout (Conv2D kernels [kh, kw, cin, cout], biases [cout])."""
    f = _File(path)
    try:
        top = f.lookup("model_weights")
    except KeyError:
        top = f.root
    attrs = f.attributes(top)
    if "layer_names" not in attrs:
        raise H5Error(f"{path}: no 'layer_names' attribute (not a Keras weight file)")
    layers = []
    for lname in _strings(attrs["layer_names"]):
        g = f.children(top)[lname]
        wnames = _strings(f.attributes(g).get("weight_names", np.zeros(0, "S1")))
        ws = []
        for wn in wnames:
            addr = g
            for part in [p for p in wn.split("/") if p]:
                addr = f.children(addr)[part]
            ws.append((wn, f.dataset(addr)))
        layers.append((lname, ws))
    return layers


def cnn_params_from_keras(layers, nb_layers: int, cin: int, nout: int, filters: int = 32):
    """Flattens the weights of the reference's ``cnn`` (neural_network.py:9-66:
    nb_layers Conv2D 3x3 with bias, then a 1x1 Conv2D head) into the parameter
    vector of ``igm_b200.cnn.CNN`` (Keras order, kernels [kh][kw][cin][cout]),
    checking every shape."""
    convs = [ws for _, ws in layers if ws]
    if len(convs) != nb_layers + 1:
        raise ValueError(f"the file has {len(convs)} layers with weights, the network {nb_layers + 1}")
    flat = []
    for i, ws in enumerate(convs):
        kern = [a for n, a in ws if "kernel" in n]
        bias = [a for n, a in ws if "bias" in n]
        if len(kern) != 1 or len(bias) != 1:
            raise ValueError(f"layer {i}: expected one kernel and one bias, got {[n for n, _ in ws]}")
        k, bvec = kern[0], bias[0]
        ci = cin if i == 0 else filters
        want = (1, 1, filters, nout) if i == nb_layers else (3, 3, ci, filters)
        if tuple(k.shape) != want or tuple(bvec.shape) != (want[-1],):
            raise ValueError(f"layer {i}: kernel {tuple(k.shape)} / bias {tuple(bvec.shape)}, expected {want}")
        flat += [k.astype(np.float32).reshape(-1), bvec.astype(np.float32).reshape(-1)]
    return np.concatenate(flat)


# ---------------------------------------------------------------------------
# writer
# ---------------------------------------------------------------------------
# The same subset, written the way h5py lays out a Keras model file: superblock
# version 0 (8-byte offsets and lengths, group leaf K 4, internal K 16),
# version-1 object headers, symbol-table groups (one level-0 B-tree node over
# symbol-table nodes of at most 8 entries, a local heap whose data segment ends
# in a free block), contiguous little-endian IEEE datasets with an explicit
# fill-value message, and version-1 attributes.  String attributes are
# fixed-length, null-padded ASCII (numpy "S" arrays, which Keras decodes like
# the variable-length strings h5py writes for Python str).
_LEAF_K, _INTERNAL_K = 4, 16
_UNDEF = b"\xff" * 8
# datatype messages (class 1, version 1, little-endian, implied mantissa msb):
# size; bit offset, precision; exponent location, size; mantissa location, size; bias
_DT_F32 = bytes([0x11, 0x20, 0x1F, 0x00]) + (4).to_bytes(4, "little") + bytes(
    [0, 0, 32, 0, 23, 8, 0, 23]) + (127).to_bytes(4, "little")
_DT_F64 = bytes([0x11, 0x20, 0x3F, 0x00]) + (8).to_bytes(4, "little") + bytes(
    [0, 0, 64, 0, 52, 11, 0, 52]) + (1023).to_bytes(4, "little")
# fill value message version 2: allocation late, write if set, value defined, size 0
_FILL = bytes([2, 2, 2, 1, 0, 0, 0, 0])


def _pad8(b: bytes) -> bytes:
    return b + b"\x00" * (-len(b) % 8)


def _q(v: int) -> bytes:
    return int(v).to_bytes(8, "little")


def _dataspace(shape) -> bytes:
    """Version-1 dataspace; rank 0 is a scalar, otherwise max dims = dims."""
    if len(shape) == 0:
        return bytes([1, 0, 0, 0, 0, 0, 0, 0])
    return bytes([1, len(shape), 1, 0, 0, 0, 0, 0]) + b"".join(_q(d) for d in shape) * 2


def _attribute(name: str, value) -> bytes:
    """Version-1 attribute message: str / bytes -> scalar fixed-length string,
    a list of str -> 1-D array of fixed-length strings, an empty list -> the
    empty float64 array Keras writes for a layer without weights."""
    if isinstance(value, (str, bytes)):
        data = value.encode() if isinstance(value, str) else value
        size, shape, raw = max(1, len(data)), (), data
        dt = bytes([0x13, 0x01, 0, 0]) + size.to_bytes(4, "little")
        raw = raw.ljust(size, b"\x00")
    elif len(value) == 0:
        dt, shape, raw = _DT_F64, (0,), b""
    else:
        items = [v.encode() if isinstance(v, str) else bytes(v) for v in value]
        size = max(1, max(len(v) for v in items))
        dt = bytes([0x13, 0x01, 0, 0]) + size.to_bytes(4, "little")
        shape, raw = (len(items),), b"".join(v.ljust(size, b"\x00") for v in items)
    nm = name.encode() + b"\x00"
    ds = _dataspace(shape)
    head = bytes([1, 0]) + len(nm).to_bytes(2, "little") + len(dt).to_bytes(2, "little") + len(ds).to_bytes(2, "little")
    return head + _pad8(nm) + _pad8(dt) + _pad8(ds) + raw


class _Writer:
    """Lays the file out bottom-up: datasets, then each group's heap, symbol
    table nodes, B-tree node and object header, the root group last, then
    the superblock at offset 0."""

    SUPERBLOCK = 96

    def __init__(self):
        self.buf = bytearray(self.SUPERBLOCK)

    def alloc(self, data: bytes) -> int:
        self.buf += b"\x00" * (-len(self.buf) % 8)
        addr = len(self.buf)
        self.buf += data
        return addr

    def object_header(self, messages) -> int:
        """messages: (type, data, flags); version-1 header, one chunk."""
        body = b""
        for mtype, data, flags in messages:
            data = _pad8(data)
            if len(data) > 0xFFFF:
                raise H5Error(f"header message of {len(data)} bytes (at most 65535)")
            body += mtype.to_bytes(2, "little") + len(data).to_bytes(2, "little") + bytes([flags, 0, 0, 0]) + data
        head = bytes([1, 0]) + len(messages).to_bytes(2, "little") + (1).to_bytes(4, "little") + \
            len(body).to_bytes(4, "little") + bytes(4)
        return self.alloc(head + body)

    def dataset(self, array) -> tuple:
        a = np.ascontiguousarray(array)
        if a.dtype == np.float32:
            dt = _DT_F32
        elif a.dtype == np.float64:
            dt = _DT_F64
        else:
            raise NotImplementedError(f"dataset dtype {a.dtype}")
        data = a.astype(a.dtype.newbyteorder("<"), copy=False).tobytes()
        addr = self.alloc(data) if data else None
        layout = bytes([3, 1]) + (_q(addr) if addr is not None else _UNDEF) + _q(len(data))
        oh = self.object_header([(0x01, _dataspace(a.shape), 0), (0x03, dt, 1), (0x05, _FILL, 1),
                                 (0x08, layout, 0)])
        return oh, None

    def group(self, children: dict, attrs: dict) -> tuple:
        """children: name -> (object header, (btree, heap) for a group else None)."""
        names = sorted(children, key=lambda s: s.encode())
        heap = bytearray(8)  # offset 0: the empty name, key 0 of the B-tree
        offs = {}
        for n in names:
            offs[n] = len(heap)
            heap += _pad8(n.encode() + b"\x00")
        free = len(heap)
        heap += _q(1) + _q(16)  # one free block, the last of the free list (next = 1)
        heap_addr = self.alloc(bytes(32))  # the heap's header, its data segment right after it
        data = self.alloc(bytes(heap))
        self.buf[heap_addr:heap_addr + 32] = b"HEAP" + bytes(4) + _q(len(heap)) + _q(free) + _q(data)
        nodes, keys = [], [0]
        cap = 2 * _LEAF_K
        for c in range(0, len(names), cap):
            chunk = names[c:c + cap]
            ent = b""
            for n in chunk:
                oh, cache = children[n]
                if cache is None:
                    ent += _q(offs[n]) + _q(oh) + bytes(8) + bytes(16)
                else:
                    ent += _q(offs[n]) + _q(oh) + (1).to_bytes(4, "little") + bytes(4) + _q(cache[0]) + _q(cache[1])
            node = b"SNOD" + bytes([1, 0]) + len(chunk).to_bytes(2, "little") + ent
            nodes.append(self.alloc(node.ljust(8 + cap * 40, b"\x00")))
            keys.append(offs[chunk[-1]])
        if len(nodes) > 2 * _INTERNAL_K:
            raise NotImplementedError(f"group of {len(names)} members (a one-node B-tree holds 256)")
        tree = b"TREE" + bytes([0, 0]) + len(nodes).to_bytes(2, "little") + _UNDEF + _UNDEF
        for k, ch in zip(keys, nodes):
            tree += _q(k) + _q(ch)
        tree += _q(keys[-1])
        btree = self.alloc(tree.ljust(24 + (4 * _INTERNAL_K + 1) * 8, b"\x00"))
        msgs = [(0x11, _q(btree) + _q(heap_addr), 0)] + [(0x0C, _attribute(k, v), 0) for k, v in attrs.items()]
        return self.object_header(msgs), (btree, heap_addr)

    def finish(self, root) -> bytes:
        oh, (btree, heap) = root
        sb = _SIG + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + _LEAF_K.to_bytes(2, "little") + \
            _INTERNAL_K.to_bytes(2, "little") + bytes(4)
        sb += _q(0) + _UNDEF + _q(len(self.buf)) + _UNDEF
        sb += _q(0) + _q(oh) + (1).to_bytes(4, "little") + bytes(4) + _q(btree) + _q(heap)
        assert len(sb) == self.SUPERBLOCK
        self.buf[:self.SUPERBLOCK] = sb
        return bytes(self.buf)


def write_h5(path: str, tree: dict, attrs: dict = None):
    """Writes a nested dict as an HDF5 file: a dict value is a group (its
    attributes under the key ``"__attrs__"``), an ndarray a float32 / float64
    dataset; ``attrs`` are the root group's attributes."""
    w = _Writer()

    def build(node, node_attrs):
        kids = {}
        for name, v in node.items():
            if name == "__attrs__":
                continue
            if isinstance(v, dict):
                kids[name] = build(v, v.get("__attrs__", {}))
            else:
                kids[name] = w.dataset(v)
        return w.group(kids, node_attrs)

    data = w.finish(build(tree, attrs or {}))
    with open(path, "wb") as f:
        f.write(data)


_KERAS_INIT = {"glorot_uniform": "GlorotUniform", "he_normal": "HeNormal", "he_uniform": "HeUniform"}


def keras_cnn_config(nb_layers: int, cin: int, nout: int, filters: int = 32, alpha: float = 0.01,
                     init: str = "glorot_uniform") -> dict:
    """The Keras Functional-model configuration of the reference's ``cnn``
    (neural_network.py:9-66, no dropout): an input of ``cin`` channels,
    nb_layers 3x3 'same' Conv2D of ``filters`` each followed by the one shared
    LeakyReLU layer (node k of it applied to conv k), a 1x1 'valid' Conv2D
    head of ``nout`` channels -- the layout tf.keras 2.15 writes."""
    def initializer(cls):
        return {"module": "keras.initializers", "class_name": cls, "config": {} if cls == "Zeros" else {"seed": None},
                "registered_name": None}

    def conv(name, f, k, padding, src, node):
        return {"class_name": "Conv2D",
                "config": {"name": name, "trainable": True, "dtype": "float32", "filters": f, "kernel_size": [k, k],
                           "strides": [1, 1], "padding": padding, "data_format": "channels_last",
                           "dilation_rate": [1, 1], "groups": 1, "activation": "linear", "use_bias": True,
                           "kernel_initializer": initializer(_KERAS_INIT.get(init, "GlorotUniform")),
                           "bias_initializer": initializer("Zeros"), "kernel_regularizer": None,
                           "bias_regularizer": None, "activity_regularizer": None, "kernel_constraint": None,
                           "bias_constraint": None},
                "name": name, "inbound_nodes": [[[src, node, 0, {}]]]}

    cname = lambda l: "conv2d" if l == 0 else f"conv2d_{l}"  # noqa: E731
    layers = [{"class_name": "InputLayer",
               "config": {"batch_input_shape": [None, None, None, cin], "dtype": "float32", "sparse": False,
                          "ragged": False, "name": "input_1"},
               "name": "input_1", "inbound_nodes": []}]
    layers.append(conv(cname(0), filters, 3, "same", "input_1", 0))
    layers.append({"class_name": "LeakyReLU",
                   "config": {"name": "leaky_re_lu", "trainable": True, "dtype": "float32",
                              "alpha": float(np.float32(alpha))},
                   "name": "leaky_re_lu", "inbound_nodes": [[[cname(l), 0, 0, {}]] for l in range(nb_layers)]})
    for l in range(1, nb_layers):
        layers.append(conv(cname(l), filters, 3, "same", "leaky_re_lu", l - 1))
    layers.append(conv(cname(nb_layers), nout, 1, "valid", "leaky_re_lu", nb_layers - 1))
    return {"class_name": "Functional",
            "config": {"name": "model", "trainable": True, "layers": layers, "input_layers": [["input_1", 0, 0]],
                       "output_layers": [[cname(nb_layers), 0, 0]]}}


def write_keras_cnn(path: str, variables, nb_layers: int, cin: int, nout: int, filters: int = 32,
                    alpha: float = 0.01, init: str = "glorot_uniform", keras_version: str = "2.15.0"):
    """Saves the reference's ``cnn`` as a Keras HDF5 model file
    (``state.iceflow_model.save("model.h5")``, emulate.py:341), loadable by
    ``tf.keras.models.load_model(..., compile=False)`` (emulate.py:86-88) and
    by ``read_keras_weights``: the attributes keras_version, backend and
    model_config at the root; the group model_weights with layer_names and,
    per layer, weight_names and the datasets <layer>/<layer>/kernel:0, bias:0.
    ``variables``: the Keras-ordered kernels [kh, kw, cin, cout] and biases."""
    import json
    if len(variables) != 2 * (nb_layers + 1):
        raise ValueError(f"{len(variables)} variables for {nb_layers + 1} convolutions")
    cname = lambda l: "conv2d" if l == 0 else f"conv2d_{l}"  # noqa: E731
    order = ["input_1", cname(0), "leaky_re_lu"] + [cname(l) for l in range(1, nb_layers + 1)]
    mw = {"__attrs__": {"layer_names": order, "backend": "tensorflow", "keras_version": keras_version}}
    for name in order:
        if not name.startswith("conv2d"):
            mw[name] = {"__attrs__": {"weight_names": []}}
            continue
        l = 0 if name == "conv2d" else int(name.split("_")[1])
        k = np.asarray(variables[2 * l], np.float32)
        b = np.asarray(variables[2 * l + 1], np.float32)
        mw[name] = {"__attrs__": {"weight_names": [f"{name}/kernel:0", f"{name}/bias:0"]},
                    name: {"kernel:0": k, "bias:0": b}}
    mw["top_level_model_weights"] = {"__attrs__": {"weight_names": []}}
    config = json.dumps(keras_cnn_config(nb_layers, cin, nout, filters, alpha, init))
    write_h5(path, {"model_weights": mw},
             {"keras_version": keras_version, "backend": "tensorflow", "model_config": config})
