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
