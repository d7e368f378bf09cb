"""Batched KSG over trajectories of uneven atom counts, frame counts and k:
every matrix equals the single-trajectory result bit for bit, on the first
(autotuned, graph-captured) call and on the replay."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_batch_matches_single_trajectory_runs(gc):
    from gmx_correlation_b200.synth import synth_traj
    specs = [(40, 700, 10, 1), (25, 1300, 20, 2), (60, 500, 5, 3), (33, 2100, 50, 4)]
    xs = [synth_traj(n, T, 6, 0.06, seed, fp32=True) for (n, T, k, seed) in specs]
    ks = [k for (_, _, k, _) in specs]
    singles = [gc.kraskov_corrmatrix(x, k) for x, k in zip(xs, ks)]
    for _ in range(2):
        mats = gc.ksg_batch(xs, ks)
        for m, ref in zip(mats, singles):
            np.testing.assert_array_equal(m, ref)
    gc.ksg_batch_release()


def test_batch_single_trajectory_and_errors(gc, small_x, golden):
    g = golden["small"]
    (m,) = gc.ksg_batch([small_x], [int(g["k"])])
    np.testing.assert_array_equal(m, g["ksg"])
    with pytest.raises(gc.GCError):
        gc.ksg_batch([small_x], [small_x.shape[1]])  # k must be below nframes
    gc.ksg_batch_release()


def test_batch_several_waves(gc):
    """A 420 x 4000 trajectory's sorted rows exceed the batch's row budget,
    so its queries run in several waves beside a small trajectory; both
    matrices equal the single-trajectory results."""
    from gmx_correlation_b200.synth import synth_traj
    xs = [synth_traj(420, 4000, 8, 0.08, 5, fp32=True), synth_traj(30, 600, 4, 0.06, 6, fp32=True)]
    ks = [100, 10]
    singles = [gc.kraskov_corrmatrix(x, k) for x, k in zip(xs, ks)]
    mats = gc.ksg_batch(xs, ks)
    for m, ref in zip(mats, singles):
        np.testing.assert_array_equal(m, ref)
    gc.ksg_batch_release()
    gc.release_cache()


def test_batched_uneven_workload_all_estimators(gc):
    """The batched uneven workload (16 trajectories, 50-400 atoms, 500-4000
    frames, k in {10, 50, 100}): KSG, GCMI and TE at lags 1 / 5 / 10 through
    the batched entry points equal the single-trajectory results bit for bit,
    and sampled pairs of every trajectory equal the reference's values
    (tests/golden/batch.npz)."""
    import hashlib

    from gmx_correlation_b200.synth import batch_specs, batch_traj
    from tests.conftest import GOLDEN
    specs = batch_specs()
    xs = [batch_traj(sp) for sp in specs]
    ks = [sp["k"] for sp in specs]
    with np.load(GOLDEN / "batch.npz") as z:
        g = {k: z[k] for k in z.files}
    out = gc.corr_batch(xs, ks, lags=(1, 5, 10))
    # a repeated call replays the captured graph of the last batch
    again = gc.te_batch(xs, ks, 10)
    for i in range(len(xs)):
        np.testing.assert_array_equal(again[i], out["te"][10][i])
    gc.batch_release()  # the batches' workspaces (tens of GB) before the single-trajectory runs
    for i, (x, k) in enumerate(zip(xs, ks)):
        assert hashlib.sha256(x.tobytes()).hexdigest() == str(g[f"b{i}_sha256"])
        np.testing.assert_array_equal(out["ksg"][i], gc.kraskov_corrmatrix(x, k))
        np.testing.assert_array_equal(out["gcmi"][i], gc.gcmi_corrmatrix(x))
        pairs = g[f"b{i}_pairs"]
        np.testing.assert_array_equal([out["ksg"][i][a1, a2] for a1, a2 in pairs], g[f"b{i}_ksg"])
        np.testing.assert_allclose([out["gcmi"][i][a1, a2] for a1, a2 in pairs], g[f"b{i}_gcmi"],
                                   rtol=1e-11, atol=1e-13)
        a1, a2 = (int(v) for v in pairs[0])
        for li, lag in enumerate((1, 5, 10)):
            te = out["te"][lag][i]
            np.testing.assert_array_equal(te, gc.te_matrix(x, k, lag))
            assert (te[a1, a2], te[a2, a1]) == tuple(g[f"b{i}_te"][li])
    plist = [np.array([a1 * (a1 - 1) // 2 + a2 for a1, a2 in g[f"b{i}_pairs"]]) for i in range(len(xs))]
    for i, (x, k) in enumerate(zip(xs, ks)):
        _, nx, ny = gc.kraskov_corrmatrix(x, k, pair_list=plist[i], detail=True)
        for q in range(len(plist[i])):
            h = hashlib.sha256(nx[q].astype(np.int32).tobytes())
            h.update(ny[q].astype(np.int32).tobytes())
            assert h.hexdigest()[:16] == str(g[f"b{i}_count_digest"][q])
    gc.release_cache()


def test_te_batch_short_trajectory_is_zero(gc):
    """A trajectory with nframes - lag <= k gives an all-zero TE matrix inside a
    batch, as te_matrix does; the others are unaffected."""
    from gmx_correlation_b200.synth import synth_traj
    xs = [synth_traj(6, 30, 3, 0.1, seed=1), synth_traj(9, 400, 4, 0.08, seed=2, fp32=True)]
    outs = gc.te_batch(xs, [28, 10], 3)
    assert not outs[0].any()
    np.testing.assert_array_equal(outs[1], gc.te_matrix(xs[1], 10, 3))
    gc.batch_release()


def test_tuned_walk_shape_fits_longer_rows_of_its_class(gc):
    """The autotuner remembers a walk shape per (frames / 256, k); a later
    trajectory of the same class with more frames (4000 after 3840) gets the
    shape clamped to what its staged rows leave room for."""
    from gmx_correlation_b200.synth import synth_traj
    gc.ksg_batch([synth_traj(12, 3840, 4, 0.08, 3, fp32=True)], [100])
    gc.batch_release()
    x = synth_traj(6, 4000, 4, 0.08, 4, fp32=True)
    np.testing.assert_array_equal(gc.kraskov_corrmatrix(x, 100),
                                  gc.kraskov_corrmatrix(x, 100, path=gc.PATH_EXACT_FP64))
    gc.release_cache()
