"""The learned KSG screen on the GPU: feature kernel and network kernels
against the float64 restatement in oracle/screen_ref.py, training, the
screened matrix against plain KSG, and what the trained network gains over
the estimate available without it."""
import numpy as np
import pytest

from oracle import screen_ref as sr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def traj():
    from gmx_correlation_b200.synth import synth_traj
    return synth_traj(24, 700, 6, 0.06, 9, fp32=True, quad=0.4)


def test_features_match_oracle(gc, traj):
    T = traj.shape[1]
    raw = gc.screen_features(traj, 15)
    P = traj.shape[0] * (traj.shape[0] - 1) // 2
    assert raw.shape == (P, gc.SCREEN_RAW)
    from gmx_correlation_b200.screen import pair_atoms
    a1, a2 = pair_atoms(np.arange(P))
    ref = sr.pair_features(traj, 15, a1, a2)
    # scalar features: float32 outputs of float64 arithmetic
    np.testing.assert_allclose(raw[:, :sr.BASE], ref[:, :sr.BASE], rtol=2e-5, atol=2e-6)
    # rank-bin histogram: a frame whose float32 projection ties or sits on a
    # rounding boundary may land in a neighbouring bin
    d = np.abs(raw[:, sr.BASE:] - ref[:, sr.BASE:]) * T
    assert d.max() <= 2.0 + 1e-3
    assert (d > 1e-3).mean() < 0.01
    # the projected form equals the raw cells projected on the same basis
    rng = np.random.default_rng(0)
    pm = raw[:, sr.BASE:].mean(0).astype(np.float32)
    pc = np.linalg.qr(rng.standard_normal((64, sr.COMP)))[0].T.astype(np.float32)
    proj = gc.screen_features(traj, 15, pca=(pm, pc))
    assert proj.shape == (P, gc.SCREEN_IN)
    np.testing.assert_array_equal(proj[:, :sr.BASE], raw[:, :sr.BASE])
    np.testing.assert_allclose(proj[:, sr.BASE:], (raw[:, sr.BASE:] - pm) @ pc.T, atol=2e-6)
    # a pair list and a shard give the same rows
    plist = np.array([5, 17, 200, 3, P - 1])
    np.testing.assert_array_equal(gc.screen_features(traj, 15, pair_list=plist), raw[plist])
    np.testing.assert_array_equal(gc.screen_features(traj, 15, pairs=(40, 90)), raw[40:90])


def _model(gc, members=2, seed=3):
    rng = np.random.default_rng(seed)
    m = gc.ScreenModel(members, seed)
    fm = rng.standard_normal(gc.SCREEN_IN).astype(np.float32) * 0.1
    fs = rng.uniform(0.5, 2.0, gc.SCREEN_IN).astype(np.float32)
    m.set_input(fm, fs, np.zeros(64, np.float32), np.zeros((sr.COMP, 64), np.float32))
    return m, fm, fs


def test_forward_matches_oracle(gc):
    m, fm, fs = _model(gc)
    rng = np.random.default_rng(4)
    F = rng.standard_normal((777, gc.SCREEN_IN)).astype(np.float32)
    Y = m.predict(F)
    P = m.get_params()
    X = sr.standardise(F, fm, fs)
    for z in range(m.members):
        yb, _ = sr.forward(P[z], X, bf16_ops=True)
        ye, _ = sr.forward(P[z], X)
        np.testing.assert_allclose(Y[z], yb, atol=2e-3 * np.abs(yb).max() + 1e-5)
        assert np.abs(Y[z] - ye).max() < 3e-2 * np.abs(ye).max() + 1e-4


def test_gradients_match_oracle(gc):
    """GPU backward (BF16 operands, FP32 accumulation) against the float64
    restatement with the same rounding (tight) and exact (loose)."""
    m, fm, fs = _model(gc, members=2, seed=5)
    rng = np.random.default_rng(6)
    n = 300
    F = rng.standard_normal((n, gc.SCREEN_IN)).astype(np.float32)
    t = rng.uniform(0.1, 0.7, n).astype(np.float32)
    G, loss = m.grad(F, t)
    P = m.get_params()
    for z in range(m.members):
        gb, lb = sr.member_grad(P[z], F, t, fm, fs, bf16_ops=True)
        ge, le = sr.member_grad(P[z], F, t, fm, fs)
        assert abs(loss[z] - lb) <= 1e-3 * lb
        g = G[z].astype(np.float64)
        rel_b = np.linalg.norm(g - gb) / np.linalg.norm(gb)
        rel_e = np.linalg.norm(g - ge) / np.linalg.norm(ge)
        cos_e = g @ ge / (np.linalg.norm(g) * np.linalg.norm(ge))
        assert rel_b < 5e-3, rel_b
        assert rel_e < 3e-2 and cos_e > 0.999, (rel_e, cos_e)
        # every parameter block is checked, biases included
        for lo, hi in [(sr.OFF_W1, sr.OFF_B1), (sr.OFF_B1, sr.OFF_W2), (sr.OFF_W2, sr.OFF_B2),
                       (sr.OFF_B3, sr.OFF_W4), (sr.OFF_W4, sr.OFF_B4), (sr.OFF_B4, sr.OFF_B4 + 1)]:
            blk = np.linalg.norm(g[lo:hi] - gb[lo:hi]) / (np.linalg.norm(gb[lo:hi]) + 1e-12)
            assert blk < 1e-2, (lo, blk)
        assert np.all(G[z][sr.N_PARAMS:] == 0)


def test_training_reduces_loss_and_is_deterministic(gc):
    rng = np.random.default_rng(8)
    n = 6000
    F = rng.standard_normal((n, gc.SCREEN_IN)).astype(np.float32)
    w = rng.standard_normal(gc.SCREEN_IN) / np.sqrt(gc.SCREEN_IN)
    t = (0.4 + 0.2 * np.tanh(F @ w) + 0.05 * np.sin(2 * F[:, 0])).astype(np.float32)
    outs = []
    for _ in range(2):
        m, _, _ = _model(gc, members=3, seed=11)
        loss = m.train(F, t, epochs=25, batch=500, lr=3e-3, seed=2)
        outs.append((loss, m.get_params()))
    loss = outs[0][0]
    assert loss[-1] < 0.05 * loss[0], loss
    np.testing.assert_array_equal(outs[0][1], outs[1][1])


def test_screened_matrix_uses_exact_ksg(gc, small_x):
    k = 10
    plain = gc.pearsify(gc.kraskov_corrmatrix(small_x, k))
    m, _, _ = _model(gc, members=2, seed=12)
    # flag everything: the screened matrix is plain KSG, bit for bit
    r_all, rep = gc.ksg_screened(small_x, k, m, sigma_max=-1.0, margin=0.0, audit_frac=0.0)
    np.testing.assert_array_equal(r_all, plain)
    assert rep["exact"] == rep["pairs"] == rep["flagged"]
    # flag nothing: only the audit sample is exact, the rest is the prediction
    r_aud, rep = gc.ksg_screened(small_x, k, m, sigma_max=np.inf, margin=0.0, audit_frac=0.1, seed=99)
    n = small_x.shape[0]
    iu = np.tril_indices(n, -1)
    exact = r_aud[iu] == plain[iu]
    assert rep["flagged"] == 0 and rep["exact"] == rep["audited"] == round(0.1 * rep["pairs"])
    assert exact.sum() >= rep["audited"]
    raw = gc.screen_features(small_x, k, pca=(np.zeros(64, np.float32), np.zeros((sr.COMP, 64), np.float32)))
    pred = np.maximum(m.predict(raw).mean(0), 0.0)
    from gmx_correlation_b200.screen import pair_atoms
    a1, a2 = pair_atoms(np.arange(rep["pairs"]))
    got = r_aud[a1, a2]
    kept = got != plain[a1, a2]
    np.testing.assert_allclose(got[kept], pred[kept], rtol=1e-6, atol=1e-7)
    # the report's audit error is the error of the predictions it kept
    audited = np.nonzero(~kept & (np.abs(pred - plain[a1, a2]) > 0))[0]
    assert rep["audit_accepted"] == rep["audited"]
    assert abs(rep["audit_max_dr"] - np.abs(pred[audited] - plain[a1, a2][audited]).max()) < 1e-6
    assert rep["final_max_dr"] == 0.0


def test_trained_network_gains_over_gaussian_estimate(gc):
    """Trained on KSG matrices of generated trajectories, the network's r
    error on unseen trajectories is well below that of the estimate the
    features give without it (the Gaussian MI's r)."""
    from gmx_correlation_b200 import screen as S
    raw, r, tid, _ = S.build_dataset(24, 500, 20, seed=3, natoms=(50, 90), nframes=(500, 900), log=None)
    ts = S.train_screen(raw, r, tid, members=3, epochs=40, batch=512, lr=2e-3, seed=1, calib_frac=0.2,
                        log=None)
    rng = np.random.default_rng(77)
    x, _ = S.random_trajectory(rng, (70, 70), (800, 800))
    rawe, re, _ = S.sample_pairs(x, 20, 1500, rng)
    F = S.project(rawe, ts.pca)
    pred = ts.model.predict(F).mean(0)
    net = np.sqrt(np.mean((pred - re) ** 2))
    base = np.sqrt(np.mean((S.r_of_mi(rawe[:, 0]) - re) ** 2))
    print(f"held-out rms |dr|: network {net:.4f}, Gaussian-MI estimate {base:.4f}; meta {ts.meta}")
    assert net < 0.5 * base
