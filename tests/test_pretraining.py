"""Host logic of the pretraining process (igm_b200/processes/pretraining.py
against igm/processes/pretraining/pretraining.py): the augmentation against
TensorFlow's image ops restated on [batch, y, x], the test-case list, the
learning-rate schedule and the direct name.  CPU only."""

import numpy as np

from igm_b200.config import default_cfg
from igm_b200.processes import pretraining as PT


def test_aug_matches_tf_image_ops():
    M = np.arange(2 * 3 * 5, dtype=np.float32).reshape(2, 3, 5)
    # tf.image.rot90 turns the image a quarter counter-clockwise: the first column becomes the last row
    r = PT._aug(M, [1, 0, 0, 0])
    assert r.shape == (2, 5, 3)
    np.testing.assert_array_equal(r[0, -1, :], M[0, :, 0])
    np.testing.assert_array_equal(r[0, 0, :], M[0, :, -1])
    np.testing.assert_array_equal(PT._aug(M, [0, 1, 0, 0]), M[:, :, ::-1])   # flip_left_right
    np.testing.assert_array_equal(PT._aug(M, [0, 0, 1, 0]), M[:, ::-1, :])   # flip_up_down
    np.testing.assert_array_equal(PT._aug(M, [0, 0, 0, 1]), M.transpose(0, 2, 1))  # transpose
    np.testing.assert_array_equal(PT._aug(M, [4, 0, 0, 0]), M)
    # the order of the reference: rotations, then the flips, then the transpose
    np.testing.assert_array_equal(PT._aug(M, [2, 1, 1, 1]), M.transpose(0, 2, 1))


def test_par_list_and_schedule():
    cfg = default_cfg(with_processes=("pretraining",))
    pt = cfg.processes.pretraining
    par = PT.par_list(pt, ["/d/test/a", "/d/test/b"])
    assert len(par) == 12  # per case: the middle, two arrhenius, two slidingco, the next coarsening
    assert par[0] == ["/d/test/a", 3, 78.0, 10000.0, 0]
    assert par[1][2] == 0.25 * 5.0 + 0.75 * 151.0 and par[2][2] == 0.75 * 5.0 + 0.25 * 151.0
    assert par[5][4] == 1 and par[6][0] == "/d/test/b"
    assert PT._code(par[0]) == "a_3_A78_C10000.0_R0"
    lr = cfg.processes.iceflow.emulator.lr
    assert PT.learning_rate(cfg, 0) == lr
    assert abs(PT.learning_rate(cfg, 100) - lr * 0.9) < 1e-15
    assert abs(PT.learning_rate(cfg, 2500) - lr) < 1e-15  # restart
    assert PT._direct_name(cfg) == "pinnbp_10_4_cnn_16_32_2_1"


def test_save_writes_the_reference_keras_file_beside_the_npz(tmp_path):
    """pretraining.py:350-351, 491-492: the models are saved as Keras HDF5
    files (model-<epoch>.h5, model.h5); beside each, the .npz this package's
    loader reads.  The .h5 holds the network on raw fields: the input scales
    folded into the first kernel, the output scale into the head."""
    import torch

    from igm_b200.keras_h5 import read_keras_weights

    rng = np.random.default_rng(3)
    nb_layers, cin, nout = 2, 5, 6
    shapes = [(3, 3, cin, 32), (32,), (3, 3, 32, 32), (32,), (1, 1, 32, nout), (nout,)]
    arrays = [rng.normal(size=s).astype(np.float32) for s in shapes]

    class Net:  # the attributes _save reads
        L, alpha, opt_iterations, out_scale = nb_layers, 0.01, 7, 50.0
        scales = np.asarray([1 / 300.0, 1 / 3000.0, 1 / 100.0, 10.0, 1 / 50.0], np.float32)
        params = torch.as_tensor(np.concatenate([a.reshape(-1) for a in arrays]))
        m = torch.zeros_like(params)
        v = torch.zeros_like(params)

        def get_variables(self):
            return [a.copy() for a in arrays]

    net = Net()
    net.cin, net.nout = cin, nout
    PT._save(net, str(tmp_path / "model-4.npz"), "he_normal")
    assert (tmp_path / "model-4.npz").exists()
    layers = read_keras_weights(str(tmp_path / "model-4.h5"))
    got = [a for _, ws in layers for _, a in ws]
    want = [a.copy() for a in arrays]
    want[0] = want[0] * net.scales[None, None, :cin, None]
    want[-2] = want[-2] * np.float32(net.out_scale)
    want[-1] = want[-1] * np.float32(net.out_scale)
    assert len(got) == len(want)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    saved = np.load(tmp_path / "model-4.npz")
    assert np.array_equal(saved["params"], net.params.numpy()) and int(saved["iterations"]) == 7
