"""Seeded synthetic MD-like trajectories with the reference's shapes.

The reference analyses real trajectories read through GROMACS; here seeded
synthetic inputs stand in for them.  Each atom fluctuates around a point of
a cubic lattice (0.38 nm spacing) as a sum of Q latent Gaussian AR(1) modes
(phi = 0.9) mapped through random per-atom 3xQ loadings, plus a quadratic
coupling term and iid noise:

    x_a(t) = mu_a + L_a m(t) + quad * L_a (m(t)^2 - 1) + noise * eps      [nm]

The quadratic term is read element-wise on the modes (m_q(t)^2 - 1, a
zero-mean nonlinear coupling through the same loadings).  With ``fp32`` the
positions are rounded to float32 first and the double-precision path gets
exactly those values promoted to double.

``center`` restates the front end's mean-centring of
src/gmx_correlation.cpp:195-223 (sequential frame sum, divide, subtract), so
the result is the mean-centred ``t_traj`` coordinate block
``x[atom][frame][3]`` that every estimator entry point takes.
"""

from __future__ import annotations

import numpy as np

__all__ = ["raw_positions", "center", "synth_traj", "CONFIGS", "batch_specs"]

# Generator settings of the reference-shaped workloads.
CONFIGS = {
    "small": dict(natoms=64, nframes=500, n_modes=8, sigma_l=0.05, k=10, fp32=False, seed=1),
    "ref": dict(natoms=247, nframes=2000, n_modes=16, sigma_l=0.08, k=100, fp32=True, seed=2),
    "large": dict(natoms=1000, nframes=5000, n_modes=16, sigma_l=0.08, k=100, fp32=True, seed=5),
}


def raw_positions(natoms: int, nframes: int, n_modes: int = 8, sigma_l: float = 0.05,
                  seed: int = 0, fp32: bool = False, phi: float = 0.9, quad: float = 0.3,
                  noise: float = 0.02, spacing: float = 0.38) -> np.ndarray:
    """Absolute positions, shape (natoms, nframes, 3), float64."""
    rng = np.random.Generator(np.random.Philox(seed))
    q = n_modes
    modes = np.empty((nframes, q))
    modes[0] = rng.standard_normal(q)
    innov = np.sqrt(1.0 - phi * phi)
    shocks = rng.standard_normal((max(nframes - 1, 0), q))
    for t in range(1, nframes):
        modes[t] = phi * modes[t - 1] + innov * shocks[t - 1]
    load = rng.normal(0.0, sigma_l, size=(natoms, 3, q))
    fluct = np.einsum("adq,tq->atd", load, modes)
    fluct += quad * np.einsum("adq,tq->atd", load, modes * modes - 1.0)
    fluct += noise * rng.standard_normal((natoms, nframes, 3))
    side = max(1, int(np.ceil(natoms ** (1.0 / 3.0) - 1e-9)))
    idx = np.arange(natoms)
    mu = spacing * np.stack([idx % side, (idx // side) % side, idx // (side * side)], axis=1)
    pos = mu[:, None, :] + fluct
    if fp32:
        pos = pos.astype(np.float32).astype(np.float64)
    return np.ascontiguousarray(pos)


def center(pos: np.ndarray):
    """Mean-centre per atom as src/gmx_correlation.cpp:195-223 does.

    Returns (x, xav): x has the shape of ``pos``; xav is (natoms, 3).  The
    frame sum is sequential (np.add.accumulate), matching the reference's
    loop, so the doubles are identical to the reference front end's.
    """
    pos = np.asarray(pos, dtype=np.float64)
    nframes = pos.shape[1]
    xav = np.add.accumulate(pos, axis=1)[:, -1, :] / nframes
    x = pos - xav[:, None, :]
    return np.ascontiguousarray(x), xav


def synth_traj(natoms: int, nframes: int, n_modes: int = 8, sigma_l: float = 0.05,
               seed: int = 0, fp32: bool = False, **kw) -> np.ndarray:
    """Mean-centred t_traj coordinates (natoms, nframes, 3) float64."""
    x, _ = center(raw_positions(natoms, nframes, n_modes, sigma_l, seed, fp32, **kw))
    return x


def config_traj(name: str) -> np.ndarray:
    c = CONFIGS[name]
    return synth_traj(c["natoms"], c["nframes"], c["n_modes"], c["sigma_l"], c["seed"], c["fp32"])


def batch_specs(count: int = 16, seed: int = 3):
    """The batched uneven workload: `count` independent trajectories with
    atoms uniform in [50, 400], frames uniform in [500, 4000] and k drawn from
    {10, 50, 100}; each entry holds the generator settings of one trajectory
    (16 latent modes, loadings 0.08 nm, float32-rounded positions, its own
    seed)."""
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for i in range(count):
        out.append(dict(natoms=int(rng.integers(50, 401)), nframes=int(rng.integers(500, 4001)),
                        k=int(rng.choice([10, 50, 100])), n_modes=16, sigma_l=0.08, fp32=True,
                        seed=1000 * seed + i))
    return out


def batch_traj(spec: dict) -> np.ndarray:
    return synth_traj(spec["natoms"], spec["nframes"], spec["n_modes"], spec["sigma_l"], spec["seed"], spec["fp32"])
