"""Gaussian, GCMI and transfer entropy on the GPU against the reference.

TE: per-query counts are exact and summed in query order with the same
digamma table, so the matrix is bit-identical.  Gaussian / GCMI: the
co-moment sums and LU determinants are bit-identical; log/erf/exp come from
CUDA's libdevice instead of glibc (1-2 ulp), hence rtol 1e-12 on MI."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["ties_q005", "box2"])
def test_golden_cases(gc, golden, case):
    g = golden[case]
    x = g["x"]
    np.testing.assert_allclose(gc.gauss_corrmatrix(x), g["gauss"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(gc.gcmi_corrmatrix(x), g["gcmi"], rtol=1e-12, atol=1e-14)
    np.testing.assert_array_equal(gc.te_matrix(x, int(g["te_k"]), int(g["te_lag"])), g["te"])


def test_small_config(gc, golden, small_x):
    g = golden["small"]
    np.testing.assert_allclose(gc.gauss_corrmatrix(small_x), g["gauss"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(gc.gcmi_corrmatrix(small_x), g["gcmi"], rtol=1e-12, atol=1e-14)
    np.testing.assert_array_equal(gc.te_matrix(small_x, int(g["k"]), 1), g["te"])


def test_reference_size_gauss_gcmi(gc, oracle):
    from gmx_correlation_b200.synth import config_traj
    x = config_traj("ref")
    for got, want in ((gc.gauss_corrmatrix(x), oracle.gauss_matrix(x)),
                      (gc.gcmi_corrmatrix(x), oracle.gcmi_matrix(x))):
        np.testing.assert_allclose(got, want, rtol=1e-11, atol=1e-13)
        r1, r2 = gc.pearsify(got.copy()), gc.pearsify(want.copy())
        assert np.max(np.abs(r1 - r2)) <= 1e-9


@pytest.mark.parametrize("lag", [1, 5, 10])
def test_te_lags(gc, oracle, lag):
    from gmx_correlation_b200.synth import synth_traj
    x = synth_traj(12, 700, 6, 0.08, seed=31, fp32=True)
    np.testing.assert_array_equal(gc.te_matrix(x, 20, lag), oracle.te_matrix(x, 20, lag))


def test_te_too_few_frames_is_zero(gc):
    from gmx_correlation_b200.synth import synth_traj
    x = synth_traj(3, 12, 2, 0.1, seed=3)
    assert not gc.te_matrix(x, 10, 5).any()


@pytest.mark.parametrize("n,T,k,lag,grid", [
    (12, 900, 20, 1, 0.0),
    (9, 1500, 100, 5, 0.0),
    (8, 500, 10, 2, 0.02),   # coordinates on a 0.02 nm grid: exact distance ties at eps
])
def test_te_fast_path_equals_exact(gc, n, T, k, lag, grid):
    """The FP32 TE kernel with FP64 repair gives the exact kernel's matrix,
    bit for bit, also when many distances tie at eps."""
    from gmx_correlation_b200.synth import synth_traj
    x = synth_traj(n, T, 4, 0.08, seed=n * T + k)
    if grid:
        x = np.round(x / grid) * grid
    fast = gc.te_matrix(x, k, lag)
    exact = gc.te_matrix(x, k, lag, path=gc.PATH_EXACT_FP64)
    np.testing.assert_array_equal(fast, exact)


@pytest.mark.parametrize("n,T,k,lag,grid", [
    (12, 900, 20, 1, 0.0),
    (9, 1500, 100, 5, 0.0),
    (8, 500, 10, 2, 0.02),    # exact distance ties at eps
    (6, 3000, 100, 10, 0.0),  # rows of 2989 entries: the 512-thread row sort
    (7, 700, 30, 0, 0.0),     # lag 0: future and past coincide
    (10, 1200, 300, 1, 0.0),  # k >= 256: values below the bound counted apart
    (5, 200, 190, 3, 0.0),    # k close to N_valid - 1
])
def test_te_walk_equals_exact(gc, n, T, k, lag, grid):
    """The sorted-row TE walk gives the exact FP64 kernel's matrix bit for bit."""
    from gmx_correlation_b200.synth import synth_traj
    x = synth_traj(n, T, 4, 0.08, seed=7 * n + T + k + lag, fp32=not grid)
    if grid:
        x = np.round(x / grid) * grid
    plan = gc.TePlan(n, T, k, lag)
    assert plan.is_walk
    plan.close()
    np.testing.assert_array_equal(gc.te_matrix(x, k, lag), gc.te_matrix(x, k, lag, path=gc.PATH_EXACT_FP64))


def test_te_walk_counts_equal_oracle(gc, oracle):
    """Per-query counts n_xp, n_xfxp, n_ypxp of the walk against the oracle."""
    torch = pytest.importorskip("torch")
    from gmx_correlation_b200.synth import synth_traj
    x = synth_traj(16, 1000, 6, 0.08, seed=77, fp32=True)
    n, T, k, lag = 16, 1000, 50, 3
    plan = gc.TePlan(n, T, k, lag)
    d_xyz = torch.from_numpy(x).cuda()
    d_te = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    plan.run(d_xyz.data_ptr(), d_te.data_ptr())
    plan.sync()
    assert plan.handoffs < 0.01 * plan.pairs * (T - lag)
    for a1, a2 in [(0, 1), (5, 3), (15, 0), (7, 12)]:
        d = oracle.te_pair(x, k, lag, a1, a2)
        nxp, nxf, nyp = plan.counts(a1, a2)
        np.testing.assert_array_equal(nxp, d["nxp"])
        np.testing.assert_array_equal(nxf, d["nxfxp"])
        np.testing.assert_array_equal(nyp, d["nypxp"])
        assert d_te[a1, a2].item() == d["te"]
    plan.close()


def test_gcmi_beyond_the_shared_memory_sort(gc, oracle):
    """More than 16384 frames: the copula scores come from rank counting
    instead of the shared-memory sort, with the reference's midranks (ties
    from 0.01 nm rounding)."""
    from gmx_correlation_b200.synth import synth_traj
    x = np.round(synth_traj(4, 17000, 3, 0.08, seed=5) / 0.01) * 0.01
    np.testing.assert_allclose(gc.gcmi_corrmatrix(x), oracle.gcmi_matrix(x), rtol=1e-11, atol=1e-13)


def test_more_than_65535_frames(gc):
    """Counts above 16 bits (the exact kernels' two-plane layout): KSG of a
    65,600-frame pair against the reference itself (oracle/_ref), and the
    per-query counts against the reference's own neighbour search."""
    from oracle import Reference
    from gmx_correlation_b200.synth import synth_traj
    ref = Reference()
    x = synth_traj(2, 65600, 2, 0.08, seed=9, fp32=True)
    mat, nx, ny = gc.kraskov_corrmatrix(x, 4, detail=True)
    np.testing.assert_array_equal(mat, ref.ksg_matrix(x, 4))
    d = ref.ksg_pair_detail(x, 4, 1, 0)
    np.testing.assert_array_equal(nx[0], d["nx"])
    np.testing.assert_array_equal(ny[0], d["ny"])
    assert nx.max() > 0 and mat[1, 0] == d["mi"]
