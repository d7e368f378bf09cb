"""The oracle restatement against golden fixtures produced by the reference."""
import hashlib

import numpy as np
import pytest


@pytest.mark.parametrize("case", ["ties_q005", "box2"])
def test_ksg_detail_matches_reference(oracle, golden, case):
    g = golden[case]
    x, k = g["x"], int(g["k"])
    X, psi = oracle.prepare(x)
    for p, (a1, a2) in enumerate(g["detail_pairs"]):
        d = oracle.ksg_pair_detail(X, psi, k, int(a1), int(a2))
        np.testing.assert_array_equal(d["nx"], g["detail_nx"][p])
        np.testing.assert_array_equal(d["ny"], g["detail_ny"][p])
        np.testing.assert_array_equal(d["kth"], g["detail_kth"][p])
        np.testing.assert_array_equal(d["epsx"], g["detail_epsx"][p])
        np.testing.assert_array_equal(d["epsy"], g["detail_epsy"][p])
        np.testing.assert_array_equal(d["dk"], g["detail_dk"][p])
        assert d["mi"] == g["detail_mi"][p]


@pytest.mark.parametrize("case", ["ties_q005", "box2"])
def test_matrices_match_reference(oracle, golden, case):
    g = golden[case]
    x = g["x"]
    np.testing.assert_array_equal(oracle.ksg_matrix(x, int(g["k"])), g["ksg"])
    np.testing.assert_array_equal(oracle.gauss_matrix(x), g["gauss"])
    np.testing.assert_array_equal(oracle.gcmi_matrix(x), g["gcmi"])
    np.testing.assert_array_equal(oracle.te_matrix(x, int(g["te_k"]), int(g["te_lag"])), g["te"])


def test_small_config(oracle, golden, small_x):
    g = golden["small"]
    assert hashlib.sha256(small_x.tobytes()).hexdigest() == str(g["sha256"])
    k = int(g["k"])
    np.testing.assert_array_equal(oracle.ksg_matrix(small_x, k), g["ksg"])
    np.testing.assert_array_equal(oracle.gauss_matrix(small_x), g["gauss"])
    np.testing.assert_array_equal(oracle.gcmi_matrix(small_x), g["gcmi"])
    X, psi = oracle.prepare(small_x)
    for p, (a1, a2) in enumerate(g["detail_pairs"]):
        d = oracle.ksg_pair_detail(X, psi, k, int(a1), int(a2))
        np.testing.assert_array_equal(d["nx"], g["detail_nx"][p])
        np.testing.assert_array_equal(d["ny"], g["detail_ny"][p])
        np.testing.assert_array_equal(d["kth"], g["detail_kth"][p])


def test_small_te(oracle, golden, small_x):
    g = golden["small"]
    np.testing.assert_array_equal(oracle.te_matrix(small_x, int(g["k"]), 1), g["te"])


