"""The Keras HDF5 writer (igm_b200.keras_h5.write_keras_cnn).  CPU only.

What save_iceflow_model writes must be what the reference's
``tf.keras.models.load_model(".../model.h5", compile=False)``
(emulate.py:86-88) reads.  Neither h5py nor TensorFlow is installable here,
so the file is checked three ways:

* round trip: the reader (igm_b200.keras_h5.read_keras_weights) gives back
  every tensor bit for bit, with the layer and weight names in Keras's order;
* against the file tf.keras 2.15 wrote for the reference's 16 x 32 network
  (tests/golden/keras_h5_layout.json, made by tests/golden/make_golden.py from
  the shipped pinnbp_5_4_cnn_16_32_2_1_e/model.h5): the model_config string
  is byte-identical (SHA-256), the layer_names / weight_names attributes and
  the superblock's format fields are equal, and a kernel dataset's
  dataspace, datatype and fill-value messages are the same bytes;
* the invariants the HDF5 library checks when it opens a symbol-table group:
  B-tree keys (heap offsets of the largest name of each child node), sorted
  symbol-table nodes of at most 2K entries, local-heap free lists ending in
  the null offset 1, the end-of-file address.
"""

import hashlib
import json
import os

import numpy as np
import pytest

from igm_b200.keras_h5 import _File, keras_cnn_config, read_keras_weights, write_h5, write_keras_cnn

HERE = os.path.dirname(os.path.abspath(__file__))


def golden():
    with open(os.path.join(HERE, "golden", "keras_h5_layout.json")) as f:
        return json.load(f)


def variables(nb_layers, cin, nout, seed=0):
    rng = np.random.default_rng(seed)
    v = []
    for l in range(nb_layers):
        v += [rng.normal(size=(3, 3, cin if l == 0 else 32, 32)).astype(np.float32),
              rng.normal(size=32).astype(np.float32)]
    return v + [rng.normal(size=(1, 1, 32, nout)).astype(np.float32), rng.normal(size=nout).astype(np.float32)]


@pytest.mark.parametrize("nb_layers,cin,nout", [(16, 5, 20), (8, 5, 10), (2, 3, 4)])
def test_round_trip(tmp_path, nb_layers, cin, nout):
    v = variables(nb_layers, cin, nout, seed=nb_layers)
    p = str(tmp_path / "model.h5")
    write_keras_cnn(p, v, nb_layers, cin, nout)
    layers = read_keras_weights(p)
    names = ["input_1", "conv2d", "leaky_re_lu"] + [f"conv2d_{l}" for l in range(1, nb_layers + 1)]
    assert [n for n, _ in layers] == names
    flat = [(wn, a) for _, ws in layers for wn, a in ws]
    assert len(flat) == len(v)
    for (wn, a), b in zip(flat, v):
        assert a.dtype == np.float32 and a.shape == b.shape and np.array_equal(a, b), wn
    f = _File(p)
    attrs = f.attributes(f.root)
    cfg = json.loads(attrs["model_config"].tobytes().rstrip(b"\x00"))
    assert cfg == keras_cnn_config(nb_layers, cin, nout)
    assert attrs["backend"].tobytes() == b"tensorflow"


def test_matches_the_file_tf_keras_wrote():
    g = golden()
    f_ref = g["file"].split("/")[-2]  # pinnbp_5_4_cnn_16_32_2_1_e: Nz 5 -> 10 outputs
    nz, nb_layers = int(f_ref.split("_")[1]), int(f_ref.split("_")[4])
    cfg = json.dumps(keras_cnn_config(nb_layers, 5, 2 * nz)).encode()
    assert len(cfg) == g["model_config_len"]
    assert hashlib.sha256(cfg).hexdigest() == g["model_config_sha256"]


def test_layout_matches_the_file_tf_keras_wrote(tmp_path):
    g = golden()
    p = str(tmp_path / "model.h5")
    write_keras_cnn(p, variables(16, 5, 10), 16, 5, 10, keras_version=g["keras_version"])
    f = _File(p)
    assert f.b[8:24].hex() == g["superblock_format"]
    assert sorted(f.attributes(f.root)) == g["root_attributes"]
    mw = f.lookup("model_weights")
    a = f.attributes(mw)
    assert sorted(a) == g["model_weights_attributes"]
    assert [x.decode() for x in a["layer_names"]] == g["layer_names"]
    kids = f.children(mw)
    for name, want in g["weight_names"].items():
        got = np.asarray(f.attributes(kids[name])["weight_names"]).reshape(-1)
        assert [x.decode() for x in got] == want, name
        if not want:
            assert got.dtype == np.float64  # the empty array Keras writes for a layer without weights
    kern = f.children(f.children(kids["conv2d"])["conv2d"])["kernel:0"]
    msgs = {"0x%02x" % t: f.b[q - 8:q + n].hex() for t, q, n in f.messages(kern) if t in (1, 3, 5)}
    assert msgs == g["kernel_messages"]
    assert [f.b[q:q + 2].hex() for t, q, n in f.messages(kern) if t == 8] == [g["kernel_layout_version_class"]]
    assert "top_level_model_weights" in kids


def _check_group(f, addr, seen):
    """The invariants of a symbol-table group (version-1 B-tree, level 0)."""
    u = f.u
    btree = heap = None
    for t, q, _ in f.messages(addr):
        if t == 0x11:
            btree, heap = f.off(q), f.off(q + 8)
    assert f.b[heap:heap + 4] == b"HEAP" and f.b[heap + 4] == 0
    dsize, free, data = u(heap + 8, 8), u(heap + 16, 8), f.off(heap + 24)
    assert f.b[data:data + 8] == bytes(8)  # offset 0: the empty name
    while free != 1:  # the free list: blocks inside the segment, ending in offset 1
        assert free % 8 == 0 and free + 16 <= dsize
        nxt, size = u(data + free, 8), u(data + free + 8, 8)
        assert size >= 16 and free + size <= dsize
        free = nxt
    name = lambda o: f.b[data + o:f.b.index(b"\x00", data + o)]  # noqa: E731
    assert f.b[btree:btree + 4] == b"TREE" and f.b[btree + 4] == 0 and f.b[btree + 5] == 0
    used = u(btree + 6, 2)
    assert f.b[btree + 8:btree + 24] == b"\xff" * 16  # no siblings
    q = btree + 24
    keys, nodes = [u(q, 8)], []
    for _ in range(used):
        nodes.append(f.off(q + 8))
        keys.append(u(q + 16, 8))
        q += 16
    assert keys[0] == 0
    names = []
    for i, node in enumerate(nodes):
        assert f.b[node:node + 6] == b"SNOD\x01\x00"
        n = u(node + 6, 2)
        assert 1 <= n <= 8
        chunk = [name(f.off(node + 8 + 40 * k)) for k in range(n)]
        assert name(keys[i + 1]) == chunk[-1]  # the key after a child: its largest name
        names += chunk
        for k in range(n):
            e = node + 8 + 40 * k
            child = f.off(e + 8)
            if u(e + 16, 4) == 1:  # a group, its B-tree and heap cached in the entry
                assert child not in seen
                seen.add(child)
                tc, hc = f.off(e + 24), f.off(e + 32)
                assert [(f.off(q2), f.off(q2 + 8)) for t, q2, _ in f.messages(child) if t == 0x11] == [(tc, hc)]
                _check_group(f, child, seen)
    assert names == sorted(names) and len(set(names)) == len(names)


def test_hdf5_invariants(tmp_path):
    p = str(tmp_path / "model.h5")
    write_keras_cnn(p, variables(16, 5, 20), 16, 5, 20)
    f = _File(p)
    assert f.u(40, 8) == len(f.b)  # end-of-file address
    root_btree, root_heap = f.off(80), f.off(88)
    assert f.u(72, 4) == 1
    assert [(f.off(q), f.off(q + 8)) for t, q, _ in f.messages(f.root) if t == 0x11] == [(root_btree, root_heap)]
    _check_group(f, f.root, set())
    # model_weights has 20 members: three symbol-table nodes under its B-tree
    mw = f.lookup("model_weights")
    assert len(f.children(mw)) == 20


def test_empty_and_nested_groups(tmp_path):
    p = str(tmp_path / "t.h5")
    a = np.arange(6, dtype=np.float64).reshape(2, 3)
    write_h5(p, {"g": {"__attrs__": {"s": "x", "l": ["ab", "c"]}, "h": {}, "d": a}, "e": np.zeros(0, np.float32)},
             {"top": "value"})
    f = _File(p)
    _check_group(f, f.root, set())
    g = f.lookup("g")
    assert sorted(f.children(g)) == ["d", "h"]
    assert np.array_equal(f.dataset(f.lookup("g/d")), a)
    assert f.dataset(f.lookup("e")).shape == (0,)
    at = f.attributes(g)
    assert at["s"].tobytes() == b"x" and [x.decode() for x in at["l"]] == ["ab", "c"]
    assert f.children(f.lookup("g/h")) == {}


def test_scales_folded_into_the_keras_network():
    """keras_variables: the Keras network on the raw fields (the reference's
    emulator input, utils.py:147-158) computes what this package's network
    computes on the scaled fields with its output scale -- FP32, the oracle's
    forward."""
    import torch

    from igm_b200.emulator import keras_variables
    from oracle import iceflow_oracle as O

    class Net:  # the attributes keras_variables reads
        def __init__(self, v, scales, out_scale):
            self._v, self.scales, self.out_scale = v, np.asarray(scales, np.float32), out_scale

        def get_variables(self):
            return self._v

    v = variables(3, 5, 6, seed=5)
    for a in v:
        a *= 0.2
    scales, out_scale = [1 / 300.0, 1 / 3000.0, 1 / 100.0, 10.0, 1 / 50.0], 200.0
    kv = keras_variables(Net(v, scales, out_scale))
    g = O.valley_glacier(24, 30, 100.0, seed=2, varying_coeffs=True)
    fl = [torch.as_tensor(g[k]).float() for k in ("thk", "usurf", "arrhenius", "slidingco")]
    X = O.fieldin_to_X(fl + [torch.full_like(fl[0], 100.0)]).double()
    t = lambda a: torch.as_tensor(a).double()  # noqa: E731
    Y_raw = O.cnn_forward(X, [t(a) for a in kv[0::2]], [t(a) for a in kv[1::2]])
    Xs = X * torch.as_tensor(scales, dtype=torch.float64)
    Y = O.cnn_forward(Xs, [t(a) for a in v[0::2]], [t(a) for a in v[1::2]], out_scale=out_scale)
    assert float((Y_raw - Y).norm() / Y.norm()) < 1e-6
