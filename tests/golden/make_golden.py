"""Generates the golden fixtures in this directory from the REFERENCE itself.

    python tests/golden/make_golden.py

Every expected value here comes out of oracle/_ref/libgcref.so, i.e. the
unmodified scdantu/gmx_correlation sources (lib/correlation_core.cpp,
lib/kraskov.cpp, lib/gcmi.cpp, lib/transfer_entropy.cpp) compiled in this
container; the per-query KSG detail comes from replaying mir_xnyn's loop
through the reference's own make_box2ind / neiK / neiE.  The reference's own
test-suite holds no golden vectors for its C++ path, so these fixtures are
what pins the oracle restatement and the GPU path.

Cases:
  ties_q005  6 atoms x 300 frames, positions quantised to 0.05 nm (many exact
             ties at the k-th distance), k=5; TE k=5 lag=2.
  box2       6 atoms x 64 frames quantised to 0.05 nm, k=40: the degenerate
             2x2 grid (inveps = 0) of the reference's neighbour search.
  small      64 atoms x 500 frames, 8 latent modes, loadings 0.05 nm, k=10,
             float64 positions; inputs regenerated from the seed (sha256
             recorded), matrices for KSG, Gaussian, GCMI and TE (k=10, lag=1).
  writers    correl.dat / XPM text of a 5x5 matrix with the 2000 diagonal.
"""

from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from gmx_correlation_b200.synth import center, raw_positions  # noqa: E402
from oracle import Reference  # noqa: E402


def quantised(natoms, nframes, q, seed):
    pos = raw_positions(natoms, nframes, 4, 0.1, seed=seed)
    x, _ = center(np.round(pos / q) * q)
    return x


def detail_all_pairs(ref, x, k):
    n = x.shape[0]
    out = {}
    pairs = [(a1, a2) for a1 in range(1, n) for a2 in range(a1)]
    for key in ("nx", "ny", "kth"):
        out[key] = np.zeros((len(pairs), x.shape[1]), np.int32)
    for key in ("epsx", "epsy", "dk"):
        out[key] = np.zeros((len(pairs), x.shape[1]))
    out["mi"] = np.zeros(len(pairs))
    for p, (a1, a2) in enumerate(pairs):
        d = ref.ksg_pair_detail(x, k, a1, a2)
        for key in ("nx", "ny", "kth", "epsx", "epsy", "dk"):
            out[key][p] = d[key]
        out["mi"][p] = d["mi"]
    out["pairs"] = np.array(pairs, np.int32)
    return out


def make_tie_case(ref, name, natoms, nframes, q, seed, k, te_k, te_lag):
    x = quantised(natoms, nframes, q, seed)
    d = detail_all_pairs(ref, x, k)
    np.savez_compressed(
        HERE / f"{name}.npz", x=x, k=k, te_k=te_k, te_lag=te_lag,
        ksg=ref.ksg_matrix(x, k), gauss=ref.gauss_matrix(x), gcmi=ref.gcmi_matrix(x),
        te=ref.te_matrix(x, te_k, te_lag), **{f"detail_{kk}": v for kk, v in d.items()})


def coords_sha(x):
    return hashlib.sha256(np.ascontiguousarray(x, np.float64).tobytes()).hexdigest()


def main():
    ref = Reference()
    make_tie_case(ref, "ties_q005", 6, 300, 0.05, 7, 5, 5, 2)
    make_tie_case(ref, "box2", 6, 64, 0.05, 7, 40, 10, 1)

    from gmx_correlation_b200.synth import synth_traj
    x = synth_traj(64, 500, 8, 0.05, seed=1)
    k = 10
    pairs = [(1, 0), (37, 12), (63, 62)]
    det = [ref.ksg_pair_detail(x, k, a1, a2) for a1, a2 in pairs]
    np.savez_compressed(
        HERE / "small.npz", natoms=64, nframes=500, n_modes=8, sigma_l=0.05, seed=1, k=k,
        sha256=coords_sha(x), ksg=ref.ksg_matrix(x, k), gauss=ref.gauss_matrix(x),
        gcmi=ref.gcmi_matrix(x), te=ref.te_matrix(x, k, 1), detail_pairs=np.array(pairs, np.int32),
        detail_nx=np.stack([d["nx"] for d in det]), detail_ny=np.stack([d["ny"] for d in det]),
        detail_kth=np.stack([d["kth"] for d in det]), detail_epsx=np.stack([d["epsx"] for d in det]),
        detail_epsy=np.stack([d["epsy"] for d in det]))

    m = np.array([[2000.0, 0.1234567, -0.5, 3.0e-7, 12345.678],
                  [0.25, 2000.0, 0.0, 1.5, -2.25],
                  [0.75, 0.125, 2000.0, 0.999999, 1e-12],
                  [0.5, 0.3333333333, 0.6666666667, 2000.0, 42.0],
                  [7.0, 8.0, 9.0, 10.0, 2000.0]])
    np.save(HERE / "writers_matrix.npy", m)
    ref.write_matrix(m, HERE / "writers_correl.dat")
    r = ref.pearsify(m)
    ref.write_matrix(r, HERE / "writers_correl_r.dat")
    ref.write_xpm(r, HERE / "writers_correl.xpm", "sel correlation matrix", "r(MI)")
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
