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
