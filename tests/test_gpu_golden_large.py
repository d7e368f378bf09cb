"""The GPU path against the reference's own results at the reference-size and
larger workloads (fixtures written by tests/golden/make_golden_large.py from
the reference compiled from its unmodified sources).

* the whole 247 x 2000, k = 100 KSG matrix: all 30,381 pair MI values
  bit-identical, n_x / n_y of 32 pairs query by query, max |dr| = 0;
* 600 x 4000 and 1000 x 5000, k = 100: 20 seeded pairs each, MI
  bit-identical and every query's counts equal (sha256 digests);
* the row-length and k variants (3000 / 5000 / 9000 frames, k = 300): whole
  matrices and every pair's counts;
* transfer entropy at 247 x 2000, k = 100, lags 1 / 5 / 10 on 24 ordered
  pairs, bit-identical.

The inputs are regenerated by gmx_correlation_b200.synth; each fixture holds
the sha256 of the coordinates it was made from, so an input drift fails as
such rather than as a result mismatch."""
import hashlib

import numpy as np
import pytest

from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu

R_TOL = 6e-4  # the reference's own CPU-vs-legacy gap (README.md:204)


def _load(name):
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def _sha(x):
    return hashlib.sha256(np.ascontiguousarray(x, np.float64).tobytes()).hexdigest()


def _digest(nx, ny):
    h = hashlib.sha256(np.ascontiguousarray(nx, np.int32).tobytes())
    h.update(np.ascontiguousarray(ny, np.int32).tobytes())
    return h.hexdigest()[:16]


def _packed(mat):
    n = mat.shape[0]
    return np.array([mat[a1, a2] for a1 in range(1, n) for a2 in range(a1)])


def _max_dr(gc, a, b):
    return float(np.max(np.abs(gc.pearsify(np.asarray(a, float).copy()) - gc.pearsify(np.asarray(b, float).copy()))))


def test_reference_size_matrix_equals_reference(gc):
    """north star's acceptance case: the whole 247 x 2000, k = 100 matrix."""
    from gmx_correlation_b200.synth import config_traj
    g = _load("ref247")
    x = config_traj(str(g["config"]))
    assert _sha(x) == str(g["sha256"])
    k = int(g["k"])
    mat = gc.kraskov_corrmatrix(x, k)
    got = _packed(mat)
    want = g["mi"]
    dr = _max_dr(gc, got[None, :], want[None, :])
    print(f"247x2000 k=100: {np.count_nonzero(got != want)} of {len(want)} pairs differ, max |dr| = {dr:.3g}")
    np.testing.assert_array_equal(got, want)
    assert dr <= R_TOL
    pairs = g["detail_pairs"]
    plist = np.array([a1 * (a1 - 1) // 2 + a2 for a1, a2 in pairs], np.int64)
    part, nx, ny = gc.kraskov_corrmatrix(x, k, pair_list=plist, detail=True)
    np.testing.assert_array_equal(nx, g["detail_nx"].astype(np.int32))
    np.testing.assert_array_equal(ny, g["detail_ny"].astype(np.int32))
    for a1, a2 in pairs:
        assert part[a1, a2] == mat[a1, a2]


@pytest.mark.parametrize("name", ["s600", "s1000"])
def test_large_configurations_sampled_pairs(gc, name):
    """600 x 4000 (several query blocks) and 1000 x 5000 (the largest
    configuration), k = 100, on the reference's pair results."""
    from gmx_correlation_b200.synth import synth_traj
    g = _load("sizes")
    n, T, q, seed, k = (int(v) for v in g[f"{name}_shape"])
    x = synth_traj(n, T, q, float(g[f"{name}_sigma_l"]), seed=seed, fp32=True)
    assert _sha(x) == str(g[f"{name}_sha256"])
    pairs = g[f"{name}_pairs"]
    plist = np.array([a1 * (a1 - 1) // 2 + a2 for a1, a2 in pairs], np.int64)
    mat, nx, ny = gc.kraskov_corrmatrix(x, k, pair_list=plist, detail=True)
    got = np.array([mat[a1, a2] for a1, a2 in pairs])
    np.testing.assert_array_equal(got, g[f"{name}_mi"])
    digests = [_digest(nx[i], ny[i]) for i in range(len(pairs))]
    assert digests == [str(d) for d in g[f"{name}_count_digest"]]
    assert _max_dr(gc, got[None, :], g[f"{name}_mi"][None, :]) <= R_TOL


@pytest.mark.parametrize("v", [0, 1, 2, 3])
def test_row_length_and_k_variants_equal_reference(gc, v):
    """Rows of 2999 / 4999 / 8999 entries (register, wide and bitonic row
    sorts) and k = 300 (entries below the bound counted apart): whole matrices
    and every pair's per-query counts."""
    from gmx_correlation_b200.synth import synth_traj
    g = _load("variants")
    n, T, k = (int(s) for s in g[f"v{v}_shape"])
    x = synth_traj(n, T, 4, 0.08, seed=n + T + k, fp32=True)
    assert _sha(x) == str(g[f"v{v}_sha256"])
    mat, nx, ny = gc.kraskov_corrmatrix(x, k, detail=True)
    np.testing.assert_array_equal(mat, g[f"v{v}_ksg"])
    digests = [_digest(nx[i], ny[i]) for i in range(nx.shape[0])]
    assert digests == [str(d) for d in g[f"v{v}_count_digest"]]


def test_transfer_entropy_reference_size(gc):
    """TE(a2 -> a1) at 247 x 2000, k = 100, lags 1 / 5 / 10 on 24 ordered
    pairs: the values, and every query's three counts (sha256 digests)."""
    torch = pytest.importorskip("torch")
    from gmx_correlation_b200.synth import config_traj
    g = _load("te247")
    x = config_traj(str(g["config"]))
    assert _sha(x) == str(g["sha256"])
    k = int(g["k"])
    n, T = x.shape[0], x.shape[1]
    d_xyz = torch.from_numpy(x).cuda()
    d_te = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    for li, lag in enumerate(g["lags"]):
        plan = gc.TePlan(n, T, k, int(lag))
        assert plan.is_walk
        plan.run(d_xyz.data_ptr(), d_te.data_ptr())
        plan.sync()
        te = d_te.cpu().numpy()
        got = np.array([te[a1, a2] for a1, a2 in g["pairs"]])
        np.testing.assert_array_equal(got, g["te"][li])
        np.testing.assert_array_equal(te, gc.te_matrix(x, k, int(lag)))
        for q, (a1, a2) in enumerate(g["pairs"]):
            nxp, nxf, nyp = plan.counts(int(a1), int(a2))
            h = hashlib.sha256(nxp.astype(np.int32).tobytes())
            h.update(nxf.astype(np.int32).tobytes())
            h.update(nyp.astype(np.int32).tobytes())
            assert h.hexdigest()[:16] == str(g["count_digest"][li, q]), (lag, a1, a2)
        plan.close()
