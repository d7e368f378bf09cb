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


def test_reference_size_pairs(oracle):
    """The restatement against the reference at 247 x 2000, k = 100: four of
    the fixture's pairs query by query, and four TE ordered pairs at lag 5."""
    from gmx_correlation_b200.synth import config_traj
    from tests.conftest import GOLDEN
    x = config_traj("ref")
    with np.load(GOLDEN / "ref247.npz") as z:
        g = {k: z[k] for k in z.files}
    assert hashlib.sha256(x.tobytes()).hexdigest() == str(g["sha256"])
    X, psi = oracle.prepare(x)
    mi = g["mi"]
    for q in (0, 7, 19, 31):
        a1, a2 = (int(v) for v in g["detail_pairs"][q])
        d = oracle.ksg_pair_detail(X, psi, int(g["k"]), a1, a2)
        np.testing.assert_array_equal(d["nx"], g["detail_nx"][q].astype(np.int32))
        np.testing.assert_array_equal(d["ny"], g["detail_ny"][q].astype(np.int32))
        assert d["mi"] == mi[a1 * (a1 - 1) // 2 + a2]
    with np.load(GOLDEN / "te247.npz") as z:
        t = {k: z[k] for k in z.files}
    li = list(t["lags"]).index(5)
    for q in (0, 5, 11, 22):
        a1, a2 = (int(v) for v in t["pairs"][q])
        assert oracle.te_pair(x, int(t["k"]), 5, a1, a2)["te"] == t["te"][li, q]
