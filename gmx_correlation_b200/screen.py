"""Training, calibration and storage of the learned KSG screen.

The screen predicts the KSG r(MI) of an atom pair from the cheap feature row
of gc_screen_features and lets gc_ksg_screened run exact KSG only where the
prediction cannot be trusted.  Everything here drives the library's own GPU
kernels: the training targets are KSG matrices this library computes on
generated trajectories, and the networks are trained and evaluated by its
BF16 tensor-core kernels.  numpy does only the bookkeeping (sampling, the
64 -> 17 histogram PCA basis, the feature standardisation, calibration).

    python -m gmx_correlation_b200.screen train --out screen_model.npz
    python -m gmx_correlation_b200.screen eval --model screen_model.npz
    python -m gmx_correlation_b200.screen study > study.json

`study` measures, on the 247 x 2000, k = 100 workload, how many pairs any
affordable predictor could leave to its prediction at audited max
|dr| <= 1e-2, and what that would save (see study()).
"""

from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from . import (SCREEN_BASE, SCREEN_COMP, SCREEN_IN, ScreenModel, kraskov_corrmatrix, ksg_screened,
               screen_features)
from .synth import synth_traj

DEFAULT_MODEL = Path(__file__).resolve().parent / "screen_model.npz"


def r_of_mi(mi):
    """pearsify's r(MI) for 3-D marginals: sqrt(1 - exp(-2 MI / 3)), 0 for MI <= 0."""
    mi = np.asarray(mi, np.float64)
    return np.where(mi > 0, np.sqrt(1.0 - np.exp(-2.0 * np.maximum(mi, 0.0) / 3.0)), 0.0)


def pair_atoms(p):
    """(a1, a2) of pair indices p = a1 (a1 - 1) / 2 + a2, a2 < a1."""
    p = np.asarray(p, np.int64)
    a1 = ((1 + np.sqrt(1 + 8 * p.astype(np.float64))) // 2).astype(np.int64)
    a1 -= (a1 * (a1 - 1) // 2 > p)
    a1 += ((a1 + 1) * a1 // 2 <= p)
    return a1, p - a1 * (a1 - 1) // 2


def random_trajectory(rng, natoms=(100, 300), nframes=(1000, 3000)):
    """One generated trajectory with randomised generator settings."""
    n = int(rng.integers(natoms[0], natoms[1] + 1))
    T = int(rng.integers(nframes[0], nframes[1] + 1))
    spec = dict(natoms=n, nframes=T, n_modes=int(rng.integers(4, 25)), sigma_l=float(rng.uniform(0.03, 0.12)),
                quad=float(rng.uniform(0.0, 0.5)), noise=float(rng.uniform(0.01, 0.05)),
                seed=int(rng.integers(1 << 31)))
    x = synth_traj(n, T, spec["n_modes"], spec["sigma_l"], spec["seed"], fp32=True, quad=spec["quad"],
                   noise=spec["noise"])
    return x, spec


def sample_pairs(x, k, npairs, rng, device=-1):
    """Raw feature rows (m, 87) and exact KSG r (m,) of m random pairs."""
    n = x.shape[0]
    P = n * (n - 1) // 2
    plist = np.sort(rng.choice(P, size=min(npairs, P), replace=False)).astype(np.int64)
    raw = screen_features(x, k, pair_list=plist, device=device)
    mat = kraskov_corrmatrix(x, k, pair_list=plist, device=device)
    a1, a2 = pair_atoms(plist)
    return raw, r_of_mi(mat[a1, a2]), plist


def fit_pca(cells, ncomp=SCREEN_COMP):
    """Mean (64,) and the leading ncomp principal axes (ncomp, 64)."""
    cells = np.asarray(cells, np.float64)
    mean = cells.mean(0)
    _, _, vt = np.linalg.svd(cells - mean, full_matrices=False)
    return mean.astype(np.float32), vt[:ncomp].astype(np.float32)


def project(raw, pca):
    """Raw rows (m, 87) -> network inputs (m, 40), as the feature kernel
    computes them when given the basis."""
    raw = np.asarray(raw, np.float32)
    tail = (raw[:, SCREEN_BASE:] - pca[0]) @ pca[1].T
    return np.concatenate([raw[:, :SCREEN_BASE], tail], 1).astype(np.float32)


def calibrate(pred_mean, pred_sd, r_true, tol, q=1.0):
    """Largest ensemble spread s such that every calibration pair with
    spread <= s has |r_hat - r| <= tol (or, with q < 1, the q-quantile of
    the error); returns (s, accepted fraction).  s = -1 accepts nothing."""
    order = np.argsort(pred_sd, kind="stable")
    err = np.abs(pred_mean[order] - r_true[order])
    if q >= 1.0:
        bad = np.nonzero(err > tol)[0]
        m = bad[0] if len(bad) else len(err)
    else:
        # running quantile: accept the longest prefix whose q-quantile <= tol
        m = 0
        for j in range(1, len(err) + 1, max(1, len(err) // 400)):
            if np.quantile(err[:j], q) <= tol:
                m = j
    if m == 0:
        return -1.0, 0.0
    return float(pred_sd[order][m - 1]), m / len(err)


class TrainedScreen:
    """A trained ensemble with its input transform and calibration."""

    def __init__(self, model: ScreenModel, feat_mean, feat_sd, pca, meta):
        self.model, self.feat_mean, self.feat_sd, self.pca, self.meta = model, feat_mean, feat_sd, pca, meta

    def save(self, path):
        np.savez_compressed(path, params=self.model.get_params(), members=self.model.members,
                            feat_mean=self.feat_mean, feat_sd=self.feat_sd, pca_mean=self.pca[0],
                            pca_comp=self.pca[1], sigma_max=self.model.sigma_max, margin=self.model.margin,
                            meta=json.dumps(self.meta))

    @classmethod
    def load(cls, path=DEFAULT_MODEL, device=-1):
        z = np.load(path, allow_pickle=False)
        m = ScreenModel(int(z["members"]), 0, device)
        m.set_params(z["params"])
        m.set_input(z["feat_mean"], z["feat_sd"], z["pca_mean"], z["pca_comp"])
        m.sigma_max, m.margin = float(z["sigma_max"]), float(z["margin"])
        return cls(m, z["feat_mean"], z["feat_sd"], (z["pca_mean"], z["pca_comp"]), json.loads(str(z["meta"])))


def build_dataset(ntraj, pairs_per_traj, k, seed, natoms=(100, 300), nframes=(1000, 3000), device=-1, log=print):
    rng = np.random.default_rng(seed)
    raws, rs, tid, specs = [], [], [], []
    t0 = time.time()
    for i in range(ntraj):
        x, spec = random_trajectory(rng, natoms, nframes)
        raw, r, _ = sample_pairs(x, k, pairs_per_traj, rng, device)
        raws.append(raw)
        rs.append(r)
        tid.append(np.full(len(r), i))
        specs.append(spec)
        if log and (i + 1) % 20 == 0:
            log(f"  trajectory {i + 1}/{ntraj}: {sum(len(v) for v in rs)} pairs, {time.time() - t0:.1f} s")
    return np.concatenate(raws), np.concatenate(rs), np.concatenate(tid), specs


def train_screen(raw, r, tid, *, members=4, epochs=40, batch=1024, lr=2e-3, seed=0, calib_frac=0.15,
                 tol=1e-2, device=-1, log=print):
    """Fits the basis, standardisation and ensemble on all trajectories but a
    held-out calibration set, then calibrates the spread threshold on it."""
    rng = np.random.default_rng(seed)
    ids = np.unique(tid)
    calib_ids = rng.choice(ids, size=max(1, int(round(calib_frac * len(ids)))), replace=False)
    cal = np.isin(tid, calib_ids)
    tr = ~cal
    pca = fit_pca(raw[tr, SCREEN_BASE:])
    F = project(raw, pca)
    fmean = F[tr].mean(0)
    fsd = F[tr].std(0)
    fsd = np.where(fsd > 1e-12, fsd, 1.0).astype(np.float32)
    model = ScreenModel(members, seed, device)
    model.set_input(fmean, fsd, pca[0], pca[1])
    t0 = time.time()
    loss = model.train(F[tr], r[tr], epochs=epochs, batch=batch, lr=lr, seed=seed)
    train_s = time.time() - t0
    Y = model.predict(F[cal])
    mean, sd = Y.mean(0), Y.std(0)
    err = mean - r[cal]
    gauss_r = r_of_mi(raw[cal, 0])
    sigma, frac = calibrate(mean, sd, r[cal], tol)
    model.sigma_max, model.margin = sigma, 0.0
    meta = dict(train_pairs=int(tr.sum()), calib_pairs=int(cal.sum()), trajectories=int(len(ids)),
                epochs=epochs, batch=batch, lr=lr, members=members, train_seconds=round(train_s, 2),
                final_loss=float(loss[-1]), calib_rms=float(np.sqrt((err ** 2).mean())),
                calib_max=float(np.abs(err).max()), gauss_rms=float(np.sqrt(((gauss_r - r[cal]) ** 2).mean())),
                tol=tol, sigma_max=sigma, calib_accept_frac=frac)
    if log:
        log("  " + json.dumps(meta))
    return TrainedScreen(model, fmean, fsd, pca, meta)


def _plan_ms(x, k, device=-1, reps=3):
    """Device time (CUDA events) of the KSG neighbour kernels for one matrix."""
    import torch

    from . import KsgPlan
    n, T = x.shape[0], x.shape[1]
    d_xyz = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    plan = KsgPlan(n, T, k, device=device)
    out = torch.zeros(plan.pairs, dtype=torch.float64, device="cuda")
    ms = []
    for _ in range(reps + 1):
        plan.run(d_xyz.data_ptr(), out.data_ptr())
        plan.sync()
        ms.append(plan.kernel_ms)
    plan.close()
    return float(np.median(ms[1:]))


def _packed(mat):
    n = mat.shape[0]
    a1, a2 = np.tril_indices(n, -1)
    return mat[a1, a2]


def _err_stats(err, tol):
    a = np.abs(err)
    return {"rms": float(np.sqrt(np.mean(err ** 2))), "q50": float(np.quantile(a, 0.5)),
            "q99": float(np.quantile(a, 0.99)), "q999": float(np.quantile(a, 0.999)), "max": float(a.max()),
            "within_tol": float(np.mean(a <= tol))}


def study(model_path=DEFAULT_MODEL, k=100, tol=1e-2, coverage=0.999, audit_frac=0.05, seed=5, device=-1):
    """How far can screening go at audited max |dr| <= tol on the reference-size
    workload (247 x 2000, k = 100)?

    Predictors of the exact KSG r, from cheapest: the committed MLP ensemble
    (features + network, about 2 ms); KSG with k = 25 and k = 10 on the same
    frames; KSG with k = 50 on every second frame.  For each: its error
    distribution against exact k = 100 KSG over all 30,381 pairs, and
    `within_tol`, the fraction of pairs whose error is within tol (the most
    any rule could keep, even one that knew every error).  Then the best
    practical rule: a linear model of r on every predictor, fitted on a random
    half of the pairs, whose residual quantile at `coverage` is calibrated per
    bin of the predictors' disagreement (|r_k25 - r_mlp|) on that half and
    applied to the other half (conformal, split by pairs).  The reported
    speed-up of a screened matrix counts the predictors' cost, exact KSG on
    the pairs the rule does not keep and on the audit sample."""
    import torch  # noqa: F401  (KsgPlan device buffers)

    from .synth import config_traj
    x = config_traj("ref")
    ts = TrainedScreen.load(model_path, device)
    out = {"workload": "247 atoms x 2000 frames, k=100 (the bench matrix)", "tol": tol, "coverage": coverage}
    r100 = r_of_mi(_packed(kraskov_corrmatrix(x, k, device=device)))
    t100 = _plan_ms(x, k, device)
    cand = {}
    t0 = time.perf_counter()
    F = screen_features(x, k, pca=ts.pca, device=device)
    Y = ts.model.predict(F)
    t_mlp = (time.perf_counter() - t0) * 1e3
    cand["mlp"] = (Y.mean(0), t_mlp)
    for kk in (25, 10):
        cand[f"ksg_k{kk}"] = (r_of_mi(_packed(kraskov_corrmatrix(x, kk, device=device))), _plan_ms(x, kk, device))
    xs = np.ascontiguousarray(x[:, ::2])
    cand["ksg_half_frames_k50"] = (r_of_mi(_packed(kraskov_corrmatrix(xs, k // 2, device=device))),
                                   _plan_ms(xs, k // 2, device))
    out["exact_ms"] = t100
    out["spread_vs_error_spearman"] = float(np.corrcoef(np.argsort(np.argsort(Y.std(0))),
                                                       np.argsort(np.argsort(np.abs(Y.mean(0) - r100))))[0, 1])
    out["predictors"] = {name: dict(_err_stats(r - r100, tol), cost_ms=c, cost_vs_exact=c / t100)
                         for name, (r, c) in cand.items()}
    # device cost of the MLP path (features + network), from the screened run's report
    _, rep = ksg_screened(x, k, ts.model, sigma_max=float("inf"), margin=0.0, device=device)
    out["predictors"]["mlp"]["cost_ms"] = rep["ms_features"] + rep["ms_mlp"]
    out["predictors"]["mlp"]["cost_vs_exact"] = out["predictors"]["mlp"]["cost_ms"] / t100
    costs = {name: out["predictors"][name]["cost_ms"] for name in cand}
    # practical rules: a linear model of r on a set of predictors, fitted on a
    # random half of the pairs; its residual quantile at `coverage` is
    # calibrated on that half per decile of the predictors' disagreement and
    # the pairs of the other half in deciles whose quantile is within tol are
    # kept (split conformal by pairs)
    rng = np.random.default_rng(seed)
    P = len(r100)
    A = np.zeros(P, bool)
    A[rng.choice(P, P // 2, replace=False)] = True
    B = ~A

    def rule(names, tol_):
        X = np.column_stack([np.ones(P)] + [cand[nm][0] for nm in names])
        coef, *_ = np.linalg.lstsq(X[A], r100[A], rcond=None)
        res = X @ coef - r100
        dis = np.abs(cand[names[-1]][0] - cand[names[0]][0]) if len(names) > 1 else np.zeros(P)
        edges = np.quantile(dis[A], np.linspace(0, 1, 11))
        keep = np.zeros(P, bool)
        for b in range(10):
            inA = A & (dis >= edges[b]) & (dis <= edges[b + 1])
            inB = B & (dis >= edges[b]) & (dis <= edges[b + 1])
            if inA.any() and np.quantile(np.abs(res[inA]), coverage) <= tol_:
                keep |= inB
        cost = sum(costs[nm] for nm in names)
        kept = float(keep[B].mean())
        exact_share = (1.0 - kept) + kept * audit_frac
        return dict(_err_stats(res[B], tol_), tol=tol_, cost_ms=cost, kept_fraction=kept,
                    kept_max_dr=float(np.abs(res[keep]).max()) if keep.any() else 0.0,
                    speedup_vs_plain=t100 / (cost + exact_share * t100))

    out["rules"] = {}
    for names in (["mlp"], ["mlp", "ksg_half_frames_k50"], list(cand)):
        key = "+".join(names)
        out["rules"][key] = [rule(names, t) for t in (tol, 0.015, 0.02, 0.03)]
    # the ceiling of the cheapest predictor: keep every pair whose MLP error is
    # within tol (it needs an error oracle no rule has)
    f = out["predictors"]["mlp"]["within_tol"]
    out["mlp_oracle_ceiling_speedup"] = t100 / (costs["mlp"] + ((1 - f) + f * audit_frac) * t100)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", default=str(DEFAULT_MODEL))
    t.add_argument("--ntraj", type=int, default=200)
    t.add_argument("--pairs", type=int, default=2000, help="sampled pairs per trajectory")
    t.add_argument("--k", type=int, default=100)
    t.add_argument("--epochs", type=int, default=40)
    t.add_argument("--members", type=int, default=4)
    t.add_argument("--seed", type=int, default=7)
    t.add_argument("--tol", type=float, default=1e-2)
    e = sub.add_parser("eval")
    e.add_argument("--model", default=str(DEFAULT_MODEL))
    e.add_argument("--natoms", type=int, default=600)
    e.add_argument("--nframes", type=int, default=4000)
    e.add_argument("--k", type=int, default=100)
    s = sub.add_parser("study")
    s.add_argument("--model", default=str(DEFAULT_MODEL))
    a = ap.parse_args(argv)
    if a.cmd == "study":
        print(json.dumps(study(a.model)))
        return
    if a.cmd == "train":
        print(f"generating {a.ntraj} trajectories ...", flush=True)
        raw, r, tid, _ = build_dataset(a.ntraj, a.pairs, a.k, a.seed)
        ts = train_screen(raw, r, tid, members=a.members, epochs=a.epochs, seed=a.seed, tol=a.tol)
        ts.save(a.out)
        print(f"saved {a.out}")
    else:
        ts = TrainedScreen.load(a.model)
        x = synth_traj(a.natoms, a.nframes, 16, 0.08, 11, fp32=True)
        rm, rep = ksg_screened(x, a.k, ts.model)
        print(json.dumps(rep))


if __name__ == "__main__":
    main()
