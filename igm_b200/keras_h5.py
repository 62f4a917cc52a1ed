"""Read-only loader for the Keras HDF5 weight files the reference ships and
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
