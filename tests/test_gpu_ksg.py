"""KSG on the GPU against the reference's results: per-query counts n_x/n_y
bit-exact and MI bit-identical (same counts, same digamma table, same
frame-order summation), so max |dr| is 0 within the 6e-4 bar."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

R_TOL = 6e-4  # the reference's own CPU-vs-legacy gap (README.md:204)


def pair_index(a1, a2):
    return a1 * (a1 - 1) // 2 + a2


@pytest.mark.parametrize("case", ["ties_q005", "box2"])
@pytest.mark.parametrize("path", [0, 1])
def test_golden_tie_cases(gc, golden, case, path):
    g = golden[case]
    mat, nx, ny = gc.kraskov_corrmatrix(g["x"], int(g["k"]), path=path, detail=True)
    np.testing.assert_array_equal(nx, g["detail_nx"])
    np.testing.assert_array_equal(ny, g["detail_ny"])
    np.testing.assert_array_equal(mat, g["ksg"])


@pytest.mark.parametrize("path", [0, 1])
def test_small_config_bitwise(gc, golden, small_x, path):
    g = golden["small"]
    mat, nx, ny = gc.kraskov_corrmatrix(small_x, int(g["k"]), path=path, detail=True)
    np.testing.assert_array_equal(mat, g["ksg"])
    for p, (a1, a2) in enumerate(g["detail_pairs"]):
        q = pair_index(int(a1), int(a2))
        np.testing.assert_array_equal(nx[q], g["detail_nx"][p])
        np.testing.assert_array_equal(ny[q], g["detail_ny"][p])
    r_gpu, r_ref = gc.pearsify(mat.copy()), gc.pearsify(g["ksg"].copy())
    assert np.max(np.abs(r_gpu - r_ref)) <= R_TOL


def test_reference_size_sampled_pairs(gc, oracle):
    """247 atoms x 2000 frames, k=100, float32-rounded positions: the full
    GPU matrix, then 10 sampled pairs checked query by query."""
    from gmx_correlation_b200.synth import config_traj
    x = config_traj("ref")
    k = 100
    mat = gc.kraskov_corrmatrix(x, k)
    assert mat.shape == (247, 247)
    np.testing.assert_array_equal(np.diag(mat), 2000.0)
    np.testing.assert_array_equal(mat, mat.T)
    X, psi = oracle.prepare(x)
    rng = np.random.default_rng(2024)
    max_dr = 0.0
    for _ in range(10):
        a1 = int(rng.integers(1, 247))
        a2 = int(rng.integers(0, a1))
        d = oracle.ksg_pair_detail(X, psi, k, a1, a2)
        p = pair_index(a1, a2)
        _, nx, ny = gc.kraskov_corrmatrix(x, k, pairs=(p, p + 1), detail=True)
        np.testing.assert_array_equal(nx[0], d["nx"])
        np.testing.assert_array_equal(ny[0], d["ny"])
        assert mat[a1, a2] == d["mi"]
        r1 = gc.pearsify(np.array([[mat[a1, a2]]]))[0, 0]
        r2 = gc.pearsify(np.array([[d["mi"]]]))[0, 0]
        max_dr = max(max_dr, abs(r1 - r2))
    assert max_dr <= R_TOL


def test_fast_path_reference_size(gc):
    """The FP32 walk handles nearly every query itself and agrees with the
    exact FP64 kernels on every pair of the 247 x 2000, k=100 matrix."""
    torch = pytest.importorskip("torch")
    from gmx_correlation_b200.synth import config_traj
    x = config_traj("ref")
    n, T = x.shape[0], x.shape[1]
    d_xyz = torch.from_numpy(x).cuda()
    fast = gc.KsgPlan(n, T, 100)
    exact = gc.KsgPlan(n, T, 100, path=gc.PATH_EXACT_FP64)
    assert fast.is_fast and not exact.is_fast
    out_f = torch.zeros(fast.pairs, dtype=torch.float64, device="cuda")
    out_e = torch.zeros_like(out_f)
    s = torch.cuda.Stream()
    fast.run(d_xyz.data_ptr(), out_f.data_ptr(), s.cuda_stream)
    exact.run(d_xyz.data_ptr(), out_e.data_ptr(), s.cuda_stream)
    torch.cuda.synchronize()
    fast.sync()
    exact.sync()
    assert fast.handoffs < 0.01 * fast.pairs * T, fast.handoff_reasons
    np.testing.assert_array_equal(out_f.cpu().numpy(), out_e.cpu().numpy())
    fast.close()
    exact.close()


@pytest.mark.parametrize("n,T,k", [
    (6, 3000, 100),   # rows of 2999 entries: 16 register slots per thread in the row sort
    (5, 5000, 50),    # 4999 entries: 32 slots; coordinate rows too long to stage
    (4, 9000, 100),   # 8999 entries: beyond the bucket pass, bitonic row sort
    (10, 1200, 300),  # k >= 256: entries below the lower bound counted apart from the histogram
])
def test_fast_path_long_rows_and_large_k(gc, n, T, k):
    """The fast path's row-length and k variants agree with the exact FP64
    kernels on every pair."""
    torch = pytest.importorskip("torch")
    from gmx_correlation_b200.synth import synth_traj
    x = synth_traj(n, T, 4, 0.08, seed=n + T + k, fp32=True)
    d_xyz = torch.from_numpy(x).cuda()
    fast = gc.KsgPlan(n, T, k)
    exact = gc.KsgPlan(n, T, k, path=gc.PATH_EXACT_FP64)
    assert fast.is_fast
    out_f = torch.zeros(fast.pairs, dtype=torch.float64, device="cuda")
    out_e = torch.zeros_like(out_f)
    s = torch.cuda.Stream()
    fast.run(d_xyz.data_ptr(), out_f.data_ptr(), s.cuda_stream)
    exact.run(d_xyz.data_ptr(), out_e.data_ptr(), s.cuda_stream)
    torch.cuda.synchronize()
    fast.sync()
    exact.sync()
    assert fast.handoffs < 0.05 * fast.pairs * T, fast.handoff_reasons
    np.testing.assert_array_equal(out_f.cpu().numpy(), out_e.cpu().numpy())
    fast.close()
    exact.close()


def test_fast_path_several_query_blocks(gc):
    """600 atoms x 4000 frames needs its sorted rows in several query blocks
    (blocks of 768 queries, the last one partial): listed pairs through the
    fast path equal the exact FP64 kernels."""
    from gmx_correlation_b200.synth import synth_traj
    x = synth_traj(600, 4000, 16, 0.08, seed=11, fp32=True)
    rng = np.random.default_rng(2)
    a1 = rng.integers(1, 600, size=24)
    a2 = np.array([rng.integers(0, a) for a in a1])
    plist = np.unique(a1 * (a1 - 1) // 2 + a2).astype(np.int64)
    fast = gc.kraskov_corrmatrix(x, 100, pair_list=plist)
    exact = gc.kraskov_corrmatrix(x, 100, pair_list=plist, path=gc.PATH_EXACT_FP64)
    np.testing.assert_array_equal(fast, exact)
    assert np.count_nonzero(fast[np.tril_indices(600, -1)]) == len(plist)


def test_shard_equals_full(gc, small_x):
    full = gc.kraskov_corrmatrix(small_x, 10)
    part = gc.kraskov_corrmatrix(small_x, 10, pairs=(100, 777))
    n = small_x.shape[0]
    for p in range(n * (n - 1) // 2):
        a1 = int((1 + np.sqrt(1 + 8 * p)) // 2)
        while a1 * (a1 - 1) // 2 > p:
            a1 -= 1
        while (a1 + 1) * a1 // 2 <= p:
            a1 += 1
        a2 = p - a1 * (a1 - 1) // 2
        want = full[a1, a2] if 100 <= p < 777 else 0.0
        assert part[a1, a2] == want and part[a2, a1] == want
    np.testing.assert_array_equal(np.diag(part), 2000.0)


def test_pair_list_matches_full_matrix(gc, golden, small_x):
    g = golden["small"]["ksg"]
    rng = np.random.default_rng(5)
    plist = rng.choice(64 * 63 // 2, size=300, replace=False)
    for path in (0, 1):
        part, nx, ny = gc.kraskov_corrmatrix(small_x, 10, pair_list=plist, path=path, detail=True)
        full, fnx, fny = gc.kraskov_corrmatrix(small_x, 10, path=path, detail=True)
        for q, p in enumerate(plist):
            a1 = int((1 + np.sqrt(1 + 8 * p)) // 2)
            while a1 * (a1 - 1) // 2 > p:
                a1 -= 1
            while (a1 + 1) * a1 // 2 <= p:
                a1 += 1
            a2 = p - a1 * (a1 - 1) // 2
            assert part[a1, a2] == g[a1, a2] and part[a2, a1] == g[a1, a2]
            np.testing.assert_array_equal(nx[q], fnx[p])
            np.testing.assert_array_equal(ny[q], fny[p])


def test_prepare_and_wrap_bitwise(gc, oracle, small_x):
    X, psi, scal = gc.kraskov_prepare(small_x)
    Xo, psio = oracle.prepare(small_x)
    np.testing.assert_array_equal(X, Xo)
    np.testing.assert_array_equal(psi, psio)
    for a1, a2 in [(1, 0), (50, 3), (63, 62)]:
        d = oracle.ksg_pair_detail(Xo, psio, 10, a1, a2)
        assert gc.kraskov_wrap(X, psi, a1, a2, 10) == d["mi"]


def test_device_resident_plan(gc, golden, small_x):
    torch = pytest.importorskip("torch")
    n, T = small_x.shape[0], small_x.shape[1]
    d_xyz = torch.from_numpy(small_x).cuda()
    plan = gc.KsgPlan(n, T, 10)
    out = torch.zeros(plan.pairs, dtype=torch.float64, device="cuda")
    for _ in range(2):
        plan.run(d_xyz.data_ptr(), out.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        plan.sync()
    assert plan.launches >= 1 and plan.kernel_ms > 0
    assert plan.is_fast
    # the fast path answers nearly every query itself on smooth data
    assert plan.handoffs < 0.05 * plan.pairs * T, plan.handoff_reasons
    g = golden["small"]["ksg"]
    want = np.array([g[a1, a2] for a1 in range(1, n) for a2 in range(a1)])  # p = a1(a1-1)/2 + a2
    np.testing.assert_array_equal(out.cpu().numpy(), want)
    plan.close()


def test_bad_inputs_are_errors(gc, small_x):
    x = small_x[:4].copy()
    x[2, :, 1] = 0.0
    with pytest.raises(gc.GCError) as e:
        gc.kraskov_corrmatrix(x, 5)
    assert e.value.status == 4
    x = small_x[:4].copy()
    x[1, 7, 0] = np.nan
    with pytest.raises(gc.GCError) as e:
        gc.kraskov_corrmatrix(x, 5)
    assert e.value.status == 5


def test_k_equal_to_frames_minus_one(gc, oracle):
    from gmx_correlation_b200.synth import synth_traj
    x = synth_traj(4, 40, 3, 0.1, seed=9)
    np.testing.assert_array_equal(gc.kraskov_corrmatrix(x, 39), oracle.ksg_matrix(x, 39))
    np.testing.assert_array_equal(gc.kraskov_corrmatrix(x, 1), oracle.ksg_matrix(x, 1))


@pytest.mark.parametrize("n,T,k", [(64, 500, 10), (20, 3000, 100), (10, 1200, 300)])
def test_hbm_gather_variant_equals_default(gc, n, T, k):
    """GC_VARIANT_HBM_GATHER (the walk reads the other marginal from unsorted
    distance rows in HBM) gives the default walk's matrix bit for bit."""
    torch = pytest.importorskip("torch")
    from gmx_correlation_b200.synth import synth_traj
    x = synth_traj(n, T, 6, 0.08, seed=n + 3 * T + k, fp32=True)
    d_xyz = torch.from_numpy(x).cuda()
    outs = []
    for variant in (gc.VARIANT_DEFAULT, gc.VARIANT_HBM_GATHER):
        plan = gc.KsgPlan(n, T, k, variant=variant)
        out = torch.zeros(plan.pairs, dtype=torch.float64, device="cuda")
        plan.run(d_xyz.data_ptr(), out.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        plan.sync()
        assert plan.is_fast
        outs.append(out.cpu().numpy())
        plan.close()
    np.testing.assert_array_equal(outs[0], outs[1])
