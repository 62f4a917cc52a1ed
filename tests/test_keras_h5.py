"""The Keras HDF5 emulator loader (igm_b200.keras_h5).  CPU only.

tests/golden/keras_h5.json holds what the loader read from every emulator the
reference ships (tests/golden/make_golden.py): here that summary is checked
against the architecture each emulator's directory name states
(emulate.py:37-62: pinnbp_<Nz>_<spacing>_cnn_<layers>_<filters>_<dim_arrhenius>_1_<basis>)
and against the reference's network (neural_network.py:9-66: 3x3 convolutions
with bias, then a 1x1 head to 2 Nz outputs); the conversion into the
network's parameter vector is checked on synthetic layers."""

import json
import os

import numpy as np
import pytest

from igm_b200.keras_h5 import cnn_params_from_keras

HERE = os.path.dirname(os.path.abspath(__file__))


def summary():
    with open(os.path.join(HERE, "golden", "keras_h5.json")) as f:
        return json.load(f)


def test_every_shipped_emulator_has_the_named_architecture():
    s = summary()
    named = [k for k in s if os.path.basename(k).startswith("pinnbp_")]
    assert len(named) >= 10
    for key in named:
        parts = os.path.basename(key).split("_")
        nz, layers, filters, dim_a = int(parts[1]), int(parts[4]), int(parts[5]), int(parts[6])
        assert parts[3] == "cnn"
        convs = s[key]
        assert len(convs) == layers + 1, key
        cin = 5 if dim_a == 2 else 5 + nz - 1
        for i, lay in enumerate(convs):
            shapes = {w["name"].split("/")[-1]: tuple(w["shape"]) for w in lay["weights"]}
            k = shapes["kernel:0"]
            want = (1, 1, filters, 2 * nz) if i == layers else (3, 3, cin if i == 0 else filters, filters)
            assert k == want, (key, i, k, want)
            assert shapes["bias:0"] == (want[-1],)
        # weights of a trained network: finite, of order 0.01-1, not all zero
        sq = sum(w["sumsq"] for lay in convs for w in lay["weights"])
        n = sum(int(np.prod(w["shape"])) for lay in convs for w in lay["weights"])
        assert np.isfinite(sq) and 1e-4 < sq / n < 1.0, (key, sq / n)


def test_default_emulator_is_present():
    """The reference's default configuration (Nz 10, spacing 4, 16 x 32 CNN,
    2-D arrhenius, Lagrange) loads pinnbp_10_4_cnn_16_32_2_1_a."""
    from igm_b200.config import default_cfg
    from igm_b200.emulator import emulator_dir_name
    name = emulator_dir_name(default_cfg())
    assert name == "pinnbp_10_4_cnn_16_32_2_1_a"
    assert name in summary()


def _layers(nb_layers, cin, nout, f=32, seed=0):
    rng = np.random.default_rng(seed)
    out = [("input_1", [])]
    for i in range(nb_layers + 1):
        shape = (1, 1, f, nout) if i == nb_layers else (3, 3, cin if i == 0 else f, f)
        name = "conv2d" if i == 0 else f"conv2d_{i}"
        out.append((name, [(f"{name}/kernel:0", rng.normal(size=shape).astype(np.float32)),
                           (f"{name}/bias:0", rng.normal(size=shape[-1]).astype(np.float32))]))
        out.append((f"leaky_re_lu_{i}", []))
    return out


def test_parameter_vector_is_in_keras_order():
    layers = _layers(2, 5, 20)
    vec = cnn_params_from_keras(layers, 2, 5, 20)
    expect = np.concatenate([a.reshape(-1) for _, ws in layers for _, a in ws])
    np.testing.assert_array_equal(vec, expect)
    assert vec.size == (9 * 5 * 32 + 32) + (9 * 32 * 32 + 32) + (32 * 20 + 20)


def test_mismatched_architectures_are_rejected():
    with pytest.raises(ValueError):
        cnn_params_from_keras(_layers(2, 5, 20), 3, 5, 20)   # layer count
    with pytest.raises(ValueError):
        cnn_params_from_keras(_layers(2, 14, 20), 2, 5, 20)  # 3-D arrhenius inputs
    with pytest.raises(ValueError):
        cnn_params_from_keras(_layers(2, 5, 20, f=16), 2, 5, 20)  # 16 filters


def test_non_hdf5_file_is_rejected(tmp_path):
    from igm_b200.keras_h5 import H5Error, read_keras_weights
    p = tmp_path / "model.h5"
    p.write_bytes(b"not an hdf5 file at all")
    with pytest.raises(H5Error):
        read_keras_weights(str(p))
