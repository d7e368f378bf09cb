"""The oracle restatement against the reference compiled from its sources,
on fresh seeded inputs (skipped where the reference library is absent)."""
import numpy as np
import pytest

from gmx_correlation_b200.synth import center, raw_positions, synth_traj

ref_mod = pytest.importorskip("oracle")


@pytest.fixture(scope="module")
def ref():
    if not ref_mod.Reference.available():
        pytest.skip("reference library not built and sources absent")
    return ref_mod.Reference()


CASES = [
    # (natoms, nframes, quantum or None, seed, k)
    (5, 257, None, 11, 7),
    (5, 200, 0.1, 12, 10),
    (4, 150, 0.2, 13, 60),
    (4, 100, 0.05, 14, 49),   # box count 2
    (5, 400, 0.02, 15, 1),
    (4, 333, None, 16, 150),
]


@pytest.mark.parametrize("n,T,q,seed,k", CASES)
def test_ksg_counts_and_mi(oracle, ref, n, T, q, seed, k):
    pos = raw_positions(n, T, 4, 0.1, seed=seed)
    if q:
        pos = np.round(pos / q) * q
    x, _ = center(pos)
    X, psi = oracle.prepare(x)
    Xr, psir = ref.prepare(x)
    np.testing.assert_array_equal(X, Xr)
    np.testing.assert_array_equal(psi, psir)
    for a1 in range(1, n):
        for a2 in range(a1):
            d = oracle.ksg_pair_detail(X, psi, k, a1, a2)
            r = ref.ksg_pair_detail(x, k, a1, a2)
            for key in ("nx", "ny", "kth", "epsx", "epsy", "dk"):
                np.testing.assert_array_equal(d[key], r[key], err_msg=f"{key} pair {a1},{a2}")
            assert d["mi"] == r["mi"]


def test_matrices_small(oracle, ref):
    x = synth_traj(9, 300, 6, 0.07, seed=21, fp32=True)
    np.testing.assert_array_equal(oracle.ksg_matrix(x, 8), ref.ksg_matrix(x, 8))
    np.testing.assert_array_equal(oracle.gauss_matrix(x), ref.gauss_matrix(x))
    np.testing.assert_array_equal(oracle.gcmi_matrix(x), ref.gcmi_matrix(x))
    for lag in (1, 5, 10):
        np.testing.assert_array_equal(oracle.te_matrix(x, 6, lag), ref.te_matrix(x, 6, lag))


def test_te_too_few_frames(oracle, ref):
    x = synth_traj(3, 12, 2, 0.1, seed=3)
    assert not oracle.te_matrix(x, 10, 5).any()
    assert not ref.te_matrix(x, 10, 5).any()


def test_center_matches_generator(oracle):
    pos = raw_positions(7, 90, 3, 0.1, seed=5, fp32=True)
    x1, xav1 = center(pos)
    x2, xav2 = oracle.center(pos)
    np.testing.assert_array_equal(x1, x2)
    np.testing.assert_array_equal(xav1, xav2)
