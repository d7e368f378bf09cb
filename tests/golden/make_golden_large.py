"""Generates the reference-size golden fixtures from the REFERENCE itself.

    python tests/golden/make_golden_large.py [--only NAME ...]

Every expected value comes out of oracle/_ref/libgcref.so: the unmodified
scdantu/gmx_correlation sources (lib/correlation_core.cpp, lib/kraskov.cpp,
lib/transfer_entropy.cpp, ...) compiled in this container.  Per-query KSG
counts come from replaying mir_xnyn's loop through the reference's own
make_box2ind / neiK / neiE (oracle/ref_shim.cpp, gcref_ksg_pair_detail).
Inputs are regenerated from gmx_correlation_b200.synth with the recorded
settings; the sha256 of the coordinates is stored so a test can tell an
input drift from a result mismatch.

Fixtures:
  ref247    the whole 247 x 2000, k = 100 KSG matrix (lib/correlation_core.cpp
            kraskov_corrmatrix, OpenMP, all host threads; about 10 minutes on
            8 cores) as the 30,381 packed pair MI values p = a1(a1-1)/2 + a2,
            plus the per-query counts n_x / n_y of 32 seeded pairs.
  te247     transfer entropy at 247 x 2000, k = 100, lags 1 / 5 / 10 on 24
            seeded ordered pairs.  TE(a2 -> a1) reads only atoms a1 and a2
            (lib/transfer_entropy.cpp:114-204), so each value is the
            reference's te_matrix on the two-atom trajectory (a1, a2); the
            per-query counts come from the oracle restatement, which must
            reproduce the reference's TE value bit for bit on every pair.
  sizes     KSG pair MI and per-query count digests of 20 seeded pairs each
            of 600 x 4000 (seed 11) and 1000 x 5000 (seed 5), k = 100.
  variants  whole KSG matrices and per-pair count digests of the row-length
            and k variants (3000 / 5000 / 9000-frame rows, k = 300).
  batch     the batched uneven workload (synth.batch_specs: 16 trajectories,
            50-400 atoms, 500-4000 frames, k in {10, 50, 100}): per
            trajectory the KSG MI and count digest of 2 seeded pairs, the
            reference's GCMI of those pairs, and TE at lags 1 / 5 / 10 of both
            orders of one pair (two-atom te_matrix, as for te247).

A count digest is the first 16 hex digits of sha256(nx as int32 || ny as
int32), so a 5000-frame pair costs 16 bytes instead of 40 KB.
"""

from __future__ import annotations

import argparse
import hashlib
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from gmx_correlation_b200.synth import CONFIGS, batch_specs, batch_traj, config_traj, synth_traj  # noqa: E402
from oracle import Oracle, Reference  # noqa: E402

# Shapes of the sampled-size and variant fixtures (atoms, frames, modes,
# loading sigma, seed, k).
SIZES = {
    "s600": (600, 4000, 16, 0.08, 11, 100),
    "s1000": (1000, 5000, 16, 0.08, 5, 100),
}
VARIANTS = [(6, 3000, 100), (5, 5000, 50), (4, 9000, 100), (10, 1200, 300)]


def coords_sha(x):
    return hashlib.sha256(np.ascontiguousarray(x, np.float64).tobytes()).hexdigest()


def count_digest(nx, ny):
    h = hashlib.sha256(np.ascontiguousarray(nx, np.int32).tobytes())
    h.update(np.ascontiguousarray(ny, np.int32).tobytes())
    return h.hexdigest()[:16]


def seeded_pairs(n, count, seed):
    rng = np.random.default_rng(seed)
    out = set()
    while len(out) < count:
        a1 = int(rng.integers(1, n))
        a2 = int(rng.integers(0, a1))
        out.add((a1, a2))
    return sorted(out)


def packed(mat):
    n = mat.shape[0]
    return np.array([mat[a1, a2] for a1 in range(1, n) for a2 in range(a1)])


def make_ref247(ref):
    c = CONFIGS["ref"]
    x = config_traj("ref")
    k = c["k"]
    t0 = time.time()
    mat = ref.ksg_matrix(x, k)
    print(f"ref247: whole matrix {time.time() - t0:.0f} s", flush=True)
    pairs = seeded_pairs(c["natoms"], 32, 2026)
    nx = np.zeros((len(pairs), c["nframes"]), np.uint16)
    ny = np.zeros_like(nx)
    for q, (a1, a2) in enumerate(pairs):
        d = ref.ksg_pair_detail(x, k, a1, a2)
        assert d["mi"] == mat[a1, a2], (a1, a2)
        nx[q], ny[q] = d["nx"], d["ny"]
    np.savez_compressed(HERE / "ref247.npz", config="ref", k=k, sha256=coords_sha(x), mi=packed(mat),
                        detail_pairs=np.array(pairs, np.int32), detail_nx=nx, detail_ny=ny)


def make_te247(ref, orc):
    c = CONFIGS["ref"]
    x = config_traj("ref")
    k = c["k"]
    lags = [1, 5, 10]
    upairs = seeded_pairs(c["natoms"], 12, 77)
    ordered = []
    for a1, a2 in upairs:
        ordered += [(a1, a2), (a2, a1)]
    te = np.zeros((len(lags), len(ordered)))
    dig = np.empty((len(lags), len(ordered)), dtype="<U16")
    t0 = time.time()
    for li, lag in enumerate(lags):
        for a1, a2 in upairs:
            sub = np.ascontiguousarray(x[[a1, a2]])
            m = ref.te_matrix(sub, k, lag)  # m[0,1] = TE(a2 -> a1), m[1,0] = TE(a1 -> a2)
            for (t1, t2), v in (((a1, a2), m[0, 1]), ((a2, a1), m[1, 0])):
                q = ordered.index((t1, t2))
                te[li, q] = v
                d = orc.te_pair(x, k, lag, t1, t2)
                assert d["te"] == v, (lag, t1, t2, d["te"], v)
                h = hashlib.sha256(d["nxp"].astype(np.int32).tobytes())
                h.update(d["nxfxp"].astype(np.int32).tobytes())
                h.update(d["nypxp"].astype(np.int32).tobytes())
                dig[li, q] = h.hexdigest()[:16]
    print(f"te247: {time.time() - t0:.0f} s", flush=True)
    np.savez_compressed(HERE / "te247.npz", config="ref", k=k, sha256=coords_sha(x), lags=np.array(lags),
                        pairs=np.array(ordered, np.int32), te=te, count_digest=dig)


def make_sizes(ref):
    out = {}
    for name, (n, T, q, sl, seed, k) in SIZES.items():
        t0 = time.time()
        x = synth_traj(n, T, q, sl, seed=seed, fp32=True)
        pairs = seeded_pairs(n, 20, 900 + seed)
        mi = np.zeros(len(pairs))
        dig = []
        for p, (a1, a2) in enumerate(pairs):
            d = ref.ksg_pair_detail(x, k, a1, a2)
            mi[p] = d["mi"]
            dig.append(count_digest(d["nx"], d["ny"]))
        out[f"{name}_shape"] = np.array([n, T, q, seed, k])
        out[f"{name}_sigma_l"] = sl
        out[f"{name}_sha256"] = coords_sha(x)
        out[f"{name}_pairs"] = np.array(pairs, np.int32)
        out[f"{name}_mi"] = mi
        out[f"{name}_count_digest"] = np.array(dig)
        print(f"sizes {name}: {time.time() - t0:.0f} s", flush=True)
    np.savez_compressed(HERE / "sizes.npz", **out)


def make_variants(ref):
    out = {}
    for i, (n, T, k) in enumerate(VARIANTS):
        t0 = time.time()
        x = synth_traj(n, T, 4, 0.08, seed=n + T + k, fp32=True)
        mat = ref.ksg_matrix(x, k)
        dig = []
        for a1 in range(1, n):
            for a2 in range(a1):
                d = ref.ksg_pair_detail(x, k, a1, a2)
                assert d["mi"] == mat[a1, a2]
                dig.append(count_digest(d["nx"], d["ny"]))
        out[f"v{i}_shape"] = np.array([n, T, k])
        out[f"v{i}_sha256"] = coords_sha(x)
        out[f"v{i}_ksg"] = mat
        out[f"v{i}_count_digest"] = np.array(dig)
        print(f"variant {n}x{T} k={k}: {time.time() - t0:.0f} s", flush=True)
    np.savez_compressed(HERE / "variants.npz", **out)


def make_batch(ref):
    out = {}
    t0 = time.time()
    for i, sp in enumerate(batch_specs()):
        x = batch_traj(sp)
        n, k = sp["natoms"], sp["k"]
        pairs = seeded_pairs(n, 2, 500 + i)
        mi, dig = [], []
        for a1, a2 in pairs:
            d = ref.ksg_pair_detail(x, k, a1, a2)
            mi.append(d["mi"])
            dig.append(count_digest(d["nx"], d["ny"]))
        g = ref.gcmi_matrix(x)
        a1, a2 = pairs[0]
        te = np.zeros((3, 2))
        for li, lag in enumerate((1, 5, 10)):
            m = ref.te_matrix(np.ascontiguousarray(x[[a1, a2]]), k, lag)
            te[li] = (m[0, 1], m[1, 0])  # TE(a2 -> a1), TE(a1 -> a2)
        out[f"b{i}_sha256"] = coords_sha(x)
        out[f"b{i}_pairs"] = np.array(pairs, np.int32)
        out[f"b{i}_ksg"] = np.array(mi)
        out[f"b{i}_count_digest"] = np.array(dig)
        out[f"b{i}_gcmi"] = np.array([g[p1, p2] for p1, p2 in pairs])
        out[f"b{i}_te"] = te
        print(f"batch {i}: {n}x{sp['nframes']} k={k} ({time.time() - t0:.0f} s)", flush=True)
    np.savez_compressed(HERE / "batch.npz", lags=np.array([1, 5, 10]), **out)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--only", nargs="*", default=None, help="subset of: ref247 te247 sizes variants batch")
    a = ap.parse_args(argv)
    want = set(a.only or ["variants", "sizes", "te247", "batch", "ref247"])
    ref, orc = Reference(), Oracle()
    if "batch" in want:
        make_batch(ref)
    if "variants" in want:
        make_variants(ref)
    if "sizes" in want:
        make_sizes(ref)
    if "te247" in want:
        make_te247(ref, orc)
    if "ref247" in want:
        make_ref247(ref)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
