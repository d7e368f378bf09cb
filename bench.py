#!/usr/bin/env python
"""KSG pairs/s on B200 for the reference-size workload: 247 atoms x 2000 frames,
k = 100, float32-rounded synthetic positions (16 latent AR(1) modes, loadings
0.08 nm), the reference's CPU path timed beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one full KSG MI matrix (all 30,381 pairs: normalisation,
neighbour statistics, ordered MI reduction) over coordinates already resident
in HBM; the L2 is flushed (a 256 MiB write) between timed steps.  `value` is
whole-job pairs/s; `e2e` is the same metric through the public C-ABI call
gc_ksg_matrix from pinned host memory (H2D of the coordinates and D2H of the
pair MI inside the timed region).  With N > 1 (torchrun, one rank per GPU)
the same matrix is split into contiguous pair shards, one per rank (the
reference's MPI split, lib/correlation_core.cpp:399-409), and one NCCL
all-gather of the packed pair MI (8 bytes per pair) gives every rank the
whole matrix inside the timed step (strong scaling); timing is max over ranks.

The cpu_baseline object also carries `legacy_gpu`: the reference's own
legacy CUDA KSG kernel (lib/kraskov_gpu.cu, built for sm_100a into
oracle/_ref) timed on a 64-atom slice of the workload.

--impl reference times the reference's own OpenMP CPU implementation
(oracle/_ref, the unmodified lib/*.cpp compiled here) on a bounded random
sample of pairs of the same workload per step, with every host thread.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "KSG pairs/s at 247 atoms×2000 fr k=100; plain vs MLP-screened at |Δr|≤1e-2"
UNIT = "pairs/s"
WORKLOAD = "KSG r(MI) matrix, 247 atoms x 2000 frames, k=100, float32-rounded synthetic positions"
FP32_OPS_PER_EVAL = 12  # 6 |d|, 5 max, 1 threshold compare per joint distance-eval
# The reference's published figure for this matrix: 130.69 s for the 247 x 2000,
# k = 100 KSG matrix on 10 OpenMP threads (README.md:162-166), i.e. 30,381 pairs
# in 130.69 s.  vs_baseline divides the line's value by it.
PUBLISHED_PAIRS_PER_S = 30381 / 130.69


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: str):
        self.gpu = gpu_index
        self.proc = None
        self.path = Path(tempfile.mkstemp(prefix="clocks_", suffix=".csv")[1])

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", self.gpu], stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, flag in zip(names, parts[5:9]):
                if flag.lower() in ("active", "1", "yes"):
                    reasons.add(nm)
        self.path.unlink(missing_ok=True)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "samples": len(sm),
                "reasons": sorted(reasons)}


def traffic_from_profiles(kernel: str):
    """DRAM bytes per launch recorded from an ncu capture (profiles/*.txt)."""
    for f in sorted((ROOT / "profiles").glob("*.txt")):
        for line in f.read_text().splitlines():
            if line.startswith(f"traffic_bytes_per_launch[{kernel}]"):
                try:
                    return float(line.split("=", 1)[1].split()[0])
                except (IndexError, ValueError):
                    return None
    return None


def cpu_baseline_sample(x, k, seconds: float, seed: int = 7):
    """Reference OpenMP KSG (kraskov_prepare + kraskov_wrap, dynamic,1) on a
    random pair sample sized to about `seconds` of work on all host threads."""
    from oracle import Reference
    ref = Reference()
    n = x.shape[0]
    rng = np.random.default_rng(seed)
    threads = os.cpu_count() or 1

    def sample(m):
        a1 = rng.integers(1, n, size=m)
        a2 = np.array([rng.integers(0, a) for a in a1])
        t0 = time.perf_counter()
        ref.ksg_pairs(x, k, a1, a2, nthreads=threads)
        return time.perf_counter() - t0

    m0 = max(threads, 8)
    dt = sample(m0)
    m = int(max(m0, min(4096, m0 * seconds / max(dt, 1e-3))))
    dt = sample(m)
    return {"value": m / dt, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{m} random pairs of the 247x2000 k=100 matrix through the reference's "
                      f"kraskov_prepare+kraskov_wrap OpenMP loop ({dt:.1f} s)"}


_LEGACY_GPU = r"""
import ctypes, json, sys, time
import numpy as np
sys.path.insert(0, sys.argv[1])
from gmx_correlation_b200.synth import CONFIGS, synth_traj
c = CONFIGS["ref"]
L = ctypes.CDLL(sys.argv[2])
L.gcref_last_error.restype = ctypes.c_char_p
dp = ctypes.POINTER(ctypes.c_double)
def run(n, T, k, seed):
    x = np.ascontiguousarray(synth_traj(n, T, c["n_modes"], c["sigma_l"], seed=seed, fp32=c["fp32"]))
    m = np.zeros((n, n))
    t0 = time.perf_counter()
    if L.gcref_ksg_matrix_legacy_gpu(x.ctypes.data_as(dp), n, T, k, m.ctypes.data_as(dp)):
        raise SystemExit(L.gcref_last_error().decode())
    return time.perf_counter() - t0
run(4, 200, 10, 1)  # CUDA context and module load, untimed
n = int(sys.argv[3])
dt = run(n, c["nframes"], c["k"], c["seed"])
print(json.dumps({"value": n * (n - 1) / 2 / dt, "seconds": dt, "pairs": n * (n - 1) // 2}))
"""


def legacy_gpu_sample(natoms: int = 64):
    """The reference's legacy CUDA KSG (lib/kraskov_gpu.cu, one block per pair,
    brute force in FP64) built for sm_100a, through kraskov_corrmatrix_gpu on
    a 64-atom slice of the workload (same frames and k, 2016 pairs), host time
    around the call after an untimed warm-up call.  It runs in a child process
    because the legacy host code exits the process on a CUDA error."""
    so = ROOT / "oracle" / "_ref" / "libgcrefgpu.so"
    if not so.exists():
        return {"unavailable": "oracle/_ref/libgcrefgpu.so not built"}
    try:
        r = subprocess.run([sys.executable, "-c", _LEGACY_GPU, str(ROOT), str(so), str(natoms)],
                           capture_output=True, text=True, timeout=300)
    except subprocess.TimeoutExpired:
        return {"unavailable": "legacy GPU KSG did not finish within 300 s"}
    if r.returncode != 0:
        return {"unavailable": (r.stderr or r.stdout).strip().splitlines()[-1:] or ["failed"]}
    d = json.loads(r.stdout.strip().splitlines()[-1])
    return {"value": d["value"], "unit": UNIT, "kind": "reference",
            "sample": f"{d['pairs']} pairs ({natoms} atoms x 2000 frames, k=100) through the reference's "
                      f"kraskov_corrmatrix_gpu, lib/kraskov_gpu.cu built for sm_100a ({d['seconds']:.2f} s)"}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from gmx_correlation_b200.synth import config_traj
    try:
        from oracle import Reference
        ref = Reference()
    except Exception as e:  # noqa: BLE001
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU library not built: {e}"}))
        return 0
    x = config_traj("ref")
    k, n = 100, x.shape[0]
    threads = os.cpu_count() or 1
    rng = np.random.default_rng(11)
    # size one step to ~8 s of CPU work
    a1 = rng.integers(1, n, size=threads * 2)
    a2 = np.array([rng.integers(0, a) for a in a1])
    t0 = time.perf_counter()
    ref.ksg_pairs(x, k, a1, a2, nthreads=threads)
    rate = len(a1) / (time.perf_counter() - t0)
    per_step = int(max(threads, min(4096, rate * 8.0)))
    times = []
    for s in range(args.warmup + args.steps):
        a1 = rng.integers(1, n, size=per_step)
        a2 = np.array([rng.integers(0, a) for a in a1])
        t0 = time.perf_counter()
        ref.ksg_pairs(x, k, a1, a2, nthreads=threads)
        if s >= args.warmup:
            times.append(time.perf_counter() - t0)
    ms = 1e3 * sum(times) / len(times)
    value = per_step / (ms / 1e3)
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": value / PUBLISHED_PAIRS_PER_S, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "pairs_per_step": per_step, "variant": "plain",
                   "sample": "random pairs of the 30,381-pair matrix, new sample each step"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{per_step} random pairs per step through kraskov_prepare+kraskov_wrap "
                                   f"(OpenMP dynamic,1, {threads} threads)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


def screened_variant(gc, x, k, plain_e2e_s: float, device: int, reps: int = 3):
    """The MLP-screened matrix through gc_ksg_screened (host arrays in and
    out, like the plain e2e leg): the calibrated rule of the committed model
    (flag every pair whose ensemble spread exceeds the spread that kept the
    audited error within 1e-2 on held-out trajectories), and the audit-only
    rule (keep every prediction, exact KSG on the 5% audit sample only)."""
    from gmx_correlation_b200.screen import TrainedScreen
    ts = TrainedScreen.load(device=device)
    n = x.shape[0]
    pairs = n * (n - 1) // 2

    def run(**kw):
        gc.ksg_screened(x, k, ts.model, device=device, **kw)  # warm (plan shapes, pool)
        t0 = time.perf_counter()
        for _ in range(reps):
            _, rep = gc.ksg_screened(x, k, ts.model, device=device, **kw)
        dt = (time.perf_counter() - t0) / reps
        return {"value": pairs / dt, "unit": UNIT, "speedup_vs_plain_e2e": plain_e2e_s / dt,
                "exact_pairs": rep["exact"], "flagged": rep["flagged"], "audited": rep["audited"],
                "audit_accepted": rep["audit_accepted"], "audited_max_dr": rep["audit_max_dr"],
                "audited_rms_dr": rep["audit_rms_dr"], "final_max_dr": rep["final_max_dr"],
                "ms_features": rep["ms_features"], "ms_mlp": rep["ms_mlp"], "ms_ksg": rep["ms_ksg"]}

    cal = run()
    cal["rule"] = {"sigma_max": ts.model.sigma_max, "margin": ts.model.margin, "audit_frac": 0.05,
                   "target_max_dr": 1e-2}
    loose = run(sigma_max=float("inf"), margin=0.0)
    loose["rule"] = {"sigma_max": "inf", "margin": 0.0, "audit_frac": 0.05}
    out = {"model": {k2: ts.meta[k2] for k2 in ("trajectories", "train_pairs", "calib_rms", "gauss_rms",
                                                "calib_accept_frac") if k2 in ts.meta},
           "calibrated_1e-2": cal, "audit_only": loose}
    # what any affordable predictor could do at the bar (gmx_correlation_b200.screen.study)
    from gmx_correlation_b200.screen import study
    st = study(device=device)
    out["study"] = {"exact_ms": st["exact_ms"], "spread_vs_error_spearman": st["spread_vs_error_spearman"],
                    "mlp_error": {k2: st["predictors"]["mlp"][k2] for k2 in ("rms", "q999", "max", "within_tol")},
                    "mlp_oracle_ceiling_speedup": st["mlp_oracle_ceiling_speedup"],
                    "rules": {name: [{k2: r[k2] for k2 in ("tol", "rms", "q999", "max", "kept_fraction",
                                                             "kept_max_dr", "cost_ms", "speedup_vs_plain")}
                                     for r in rules] for name, rules in st["rules"].items()}}
    return out


def large_variant(gc, torch, dev, local: int, mix_ops: float):
    """The largest configuration, 1000 atoms x 5000 frames, k = 100 (499,500
    pairs), one whole matrix per arm from device-resident coordinates: the
    default walk (the other marginal recomputed from coordinates staged in
    shared memory) against the HBM arm (the other marginal read from unsorted
    per-(atom, query) distance rows the row sort also writes to HBM).  Both
    arms keep the sorted rows of the walked marginal in HBM in query blocks of
    a 16 GiB budget.  max |dr| against the reference's MI on the 20 seeded
    pairs of tests/golden/sizes.npz (made by the reference itself)."""
    from gmx_correlation_b200.synth import synth_traj
    with np.load(ROOT / "tests" / "golden" / "sizes.npz") as z:
        n, T, q, seed, k = (int(v) for v in z["s1000_shape"])
        sigma, pairs, want = float(z["s1000_sigma_l"]), z["s1000_pairs"], z["s1000_mi"]
    x = synth_traj(n, T, q, sigma, seed=seed, fp32=True)
    npairs = n * (n - 1) // 2
    d_xyz = torch.from_numpy(x).to(dev)
    d_out = torch.empty(npairs, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    idx = np.array([a1 * (a1 - 1) // 2 + a2 for a1, a2 in pairs])
    lpad = ((T - 1) + 31) // 32 * 32
    out = {"workload": f"KSG r(MI) matrix, {n} atoms x {T} frames, k={k}, float32-rounded synthetic positions",
           "pairs": npairs, "sorted_rows_gb": n * T * lpad * 6 / 1e9}
    for name, variant in (("recompute", gc.VARIANT_DEFAULT), ("hbm_rows", gc.VARIANT_HBM_GATHER)):
        plan = gc.KsgPlan(n, T, k, device=local, variant=variant)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plan.run(d_xyz.data_ptr(), d_out.data_ptr(), stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        plan.sync()
        ms, kms = e0.elapsed_time(e1), plan.kernel_ms
        got = d_out.cpu().numpy()[idx]
        r1 = gc.pearsify(got[None, :].copy())
        r2 = gc.pearsify(np.asarray(want, float)[None, :].copy())
        evals = npairs * T * (T - 1)
        row_bytes = out["sorted_rows_gb"] * 1e9 * (2 if variant == gc.VARIANT_DEFAULT else 2 + 4 / 6 * 2)
        out[name] = {"value": npairs / (ms / 1e3), "unit": UNIT, "ms_per_matrix": ms, "kernel_ms": kms,
                     "distance_evals_per_s": evals / (kms / 1e3),
                     "roofline_frac": evals * FP32_OPS_PER_EVAL / (kms / 1e3) / mix_ops,
                     "rows_hbm_gbs": row_bytes / (kms / 1e3) / 1e9,
                     "handed_to_exact": plan.handoffs, "walk_entries_per_query": round(plan.walk_mean, 1),
                     "audited_pairs": int(len(idx)), "audited_max_dr": float(np.max(np.abs(r1 - r2))),
                     "audited_bitwise": bool(np.array_equal(got, want))}
        plan.close()
        gc.release_cache()
    out["faster"] = min(("recompute", "hbm_rows"), key=lambda a: out[a]["ms_per_matrix"])
    out["note"] = ("rows_hbm_gbs: the sorted rows written once and read once (plus the unsorted rows of "
                   "the HBM arm, written and read once) over the neighbour kernels' time; a lower bound")
    return out


def batch_variant(gc, local: int):
    """The batched uneven workload (synth.batch_specs: 16 trajectories, 50-400
    atoms, 500-4000 frames, k in {10, 50, 100}) through the batched entry
    points, host arrays in and out: KSG MI, GCMI and TE at lag 1.
    The first call of each (autotuning, graph capture) is untimed; the timed
    second call replays the captured graphs."""
    from gmx_correlation_b200.synth import batch_specs, batch_traj
    specs = batch_specs()
    xs = [batch_traj(sp) for sp in specs]
    ks = [sp["k"] for sp in specs]
    pairs = sum(x.shape[0] * (x.shape[0] - 1) // 2 for x in xs)
    out = {"workload": "16 trajectories, atoms U[50,400], frames U[500,4000], k in {10,50,100}",
           "trajectories": len(xs), "pairs": pairs, "ordered_pairs": 2 * pairs,
           "timing": "host time of the second call (the first tunes and captures the graph)"}

    def timed(fn):
        fn()
        t0 = time.perf_counter()
        fn()
        return time.perf_counter() - t0

    dt = timed(lambda: gc.ksg_batch(xs, ks, device=local))
    out["ksg"] = {"value": pairs / dt, "unit": UNIT, "seconds": dt}
    dt = timed(lambda: gc.gcmi_batch(xs, device=local))
    out["gcmi"] = {"value": pairs / dt, "unit": UNIT, "seconds": dt}
    gc.batch_release()
    # lag 1 here; lags 5 and 10 run the same kernels (the GPU tests cover them)
    dt = timed(lambda: gc.te_batch(xs, ks, 1, device=local))
    out["te_lag1"] = {"value": 2 * pairs / dt, "unit": "ordered pairs/s", "seconds": dt}
    gc.batch_release()
    return out


TE_OPS_PER_EVAL = 18  # 9 |d|, 8 max, 1 threshold compare per 9-D joint distance-eval


def te_variant(gc, torch, x, k: int, lag: int, dev, local: int, mix_ops: float, reps: int = 3,
               cpu: bool = True):
    """Transfer entropy TE(a2 -> a1) of every ordered pair at the same
    workload (lib/transfer_entropy.cpp:63-221), lag `lag`: the device-resident
    TE plan timed with CUDA events (L2 flushed between runs), the end-to-end
    gc_te_matrix call from pinned host memory, and the reference's own OpenMP
    te_matrix on a 16-atom subset of the trajectory (240 ordered pairs)."""
    n, T = x.shape[0], x.shape[1]
    nv = T - lag
    d_xyz = torch.from_numpy(x).to(dev)
    d_te = torch.zeros((n, n), dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    plan = gc.TePlan(n, T, k, lag, device=local)
    # a real stream handle: the legacy default stream is handle 0, which the
    # plan reads as "the library's own stream", and the events would then
    # bracket nothing
    stream = torch.cuda.Stream(dev)
    plan.run(d_xyz.data_ptr(), d_te.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize(dev)
    plan.sync()
    step, kern = [], []
    for _ in range(reps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plan.run(d_xyz.data_ptr(), d_te.data_ptr(), stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        step.append(e0.elapsed_time(e1))
        kern.append(plan.kernel_ms)
    plan.sync()
    pairs = plan.pairs
    ms, kms = statistics.mean(step), statistics.mean(kern)
    evals = pairs * nv * (nv - 1)
    out = {"metric": "TE ordered pairs/s", "value": pairs / (ms / 1e3), "unit": "pairs/s", "lag": lag, "k": k,
           "ms_per_matrix": ms, "kernel_ms": kms, "ordered_pairs": pairs,
           "path": "sorted-row walk + exact fp64 repair" if plan.is_walk else "fp32 brute force + fp64 repair",
           "handed_to_exact": plan.handoffs, "walk_entries_per_query": round(plan.walk_mean, 1),
           "gpu_launches": plan.launches,
           "roofline": {"bound": "fp32", "achieved": evals * TE_OPS_PER_EVAL / (kms / 1e3) / 1e12,
                        "peak": mix_ops / 1e12, "unit": "TOP/s",
                        "frac": evals * TE_OPS_PER_EVAL / (kms / 1e3) / mix_ops,
                        "distance_evals_per_s": evals / (kms / 1e3),
                        "note": "reuse-normalised: T(T-1) 9-D evals per ordered pair x 18 ops over the "
                                "neighbour kernels' time"}}
    plan.close()
    x_pinned = torch.from_numpy(x).pin_memory().numpy()
    gc.te_matrix(x_pinned, k, lag, device=local)
    t0 = time.perf_counter()
    for _ in range(reps):
        gc.te_matrix(x_pinned, k, lag, device=local)
    e2e = (time.perf_counter() - t0) / reps
    out["e2e"] = {"value": pairs / e2e, "unit": "pairs/s", "h2d_bytes_per_step": int(x.nbytes),
                  "d2h_bytes_per_step": int(n * n * 8)}
    if cpu:
        try:
            from oracle import Reference
            ref = Reference()
            sub = np.ascontiguousarray(x[:16])
            threads = os.cpu_count() or 1
            t0 = time.perf_counter()
            ref.te_matrix(sub, k, lag, nthreads=threads)
            dt = time.perf_counter() - t0
            out["cpu_baseline"] = {"value": 16 * 15 / dt, "unit": "pairs/s", "cores": threads, "kind": "reference",
                                   "sample": f"te_matrix on atoms 0-15 of the workload (240 ordered pairs, "
                                             f"{dt:.1f} s, OpenMP)"}
        except Exception as e:  # noqa: BLE001
            out["cpu_baseline"] = {"unavailable": str(e)}
    return out


def run_ours(args):
    import torch

    import gmx_correlation_b200 as gc
    from gmx_correlation_b200.synth import CONFIGS, synth_traj

    ws, rank, local = dist_env()
    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    else:
        torch.cuda.set_device(local)
    c = CONFIGS["ref"]
    natoms = args.natoms or c["natoms"]
    from gmx_correlation_b200.shard import gather_pairs, pair_shard, sharded_ksg_matrix
    x = synth_traj(natoms, c["nframes"], c["n_modes"], c["sigma_l"], seed=c["seed"], fp32=c["fp32"])
    n, T, k = x.shape[0], x.shape[1], c["k"]
    npairs = n * (n - 1) // 2
    pb, pe = pair_shard(npairs, rank, ws)
    dev = torch.device("cuda", local)
    if args.te_only:  # the transfer-entropy object alone (profiling runs)
        if rank == 0:
            mix_ops, _ = gc.probe_fp32(local)
            print(json.dumps(te_variant(gc, torch, x, k, 1, dev, local, mix_ops, reps=args.steps, cpu=False)))
        return 0
    d_xyz = torch.from_numpy(x).to(dev)
    d_out = torch.empty(max(pe - pb, 1), dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    plan = gc.KsgPlan(n, T, k, device=local, path=args.path, pairs=(pb, pe) if ws > 1 else None)
    stream = torch.cuda.Stream(dev)  # a real stream handle (the legacy default stream is 0)
    torch.cuda.set_stream(stream)

    def step():
        plan.run(d_xyz.data_ptr(), d_out.data_ptr(), stream.cuda_stream)
        if pg:  # every rank gets the whole packed pair list
            gather_pairs(d_out[: pe - pb], npairs, pg)

    for _ in range(args.warmup):
        step()
        torch.cuda.synchronize(dev)
        plan.sync()

    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    gpu_index = vis.split(",")[local] if vis else str(local)
    sampler = ClockSampler(gpu_index)
    if pg:
        pg.barrier()
    torch.cuda.synchronize(dev)
    sampler.start()
    step_ms, kern_ms = [], []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        step_ms.append(e0.elapsed_time(e1))
        kern_ms.append(plan.kernel_ms)
    torch.cuda.synchronize(dev)
    if pg:
        pg.barrier()
    clocks = sampler.stop()
    plan.sync()
    handoffs = plan.handoffs
    walk_mean = plan.walk_mean
    reasons = {k: v for k, v in plan.handoff_reasons.items() if v}
    total_ms = sum(step_ms)
    launches = plan.launches * args.steps
    if pg:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = npairs / (ms_per_step / 1e3)  # one whole matrix per step, over all ranks

    # end to end through the public C-ABI call, pinned host input (with N > 1
    # each rank's shard, then the all-gather of the packed pair values)
    x_pinned = torch.from_numpy(x).pin_memory().numpy()

    def e2e_call():
        if pg:
            sharded_ksg_matrix(x_pinned, k, pg)
        else:
            gc.kraskov_corrmatrix(x_pinned, k, device=local)

    e2e_call()
    e2e_steps = max(1, args.steps)
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_call()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    if pg:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_s = float(t.item())

    if rank == 0:
        mix_ops, fma_flops = gc.probe_fp32(local)
        kms = statistics.mean(kern_ms)
        kname = "ksg_neighbour_kernels" if plan.is_fast else "ksg_exact_kernel"
        evals = (pe - pb) * T * (T - 1)  # this rank's shard
        achieved = evals * FP32_OPS_PER_EVAL / (kms / 1e3)
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "strong" if ws > 1 else "weak",
            "vs_baseline": value / PUBLISHED_PAIRS_PER_S if natoms == c["natoms"] else None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD if natoms == c["natoms"] else WORKLOAD.replace("247", str(natoms)),
                       "variant": "plain", "pairs_per_gpu": pe - pb,
                       "parallelism": f"pair shards over {ws} GPUs + NCCL all-gather" if ws > 1 else "one GPU",
                       "l2": "256 MiB flush between timed steps",
                       "path": "fp32 sorted-row walk + exact fp64 repair" if plan.is_fast else "exact-fp64 brute force",
                       "handed_to_exact": handoffs, "queries": (pe - pb) * T,
                       "walk_entries_per_query": round(walk_mean, 1), "handoff_reasons": reasons},
            "e2e": {"value": npairs / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(x.nbytes),
                    "d2h_bytes_per_step": int(npairs * 8)},
            "gpu_launches": launches,
            "roofline": {"bound": "fp32", "achieved": achieved / 1e12, "peak": mix_ops / 1e12, "unit": "TOP/s",
                         "frac": achieved / mix_ops, "traffic": traffic_from_profiles(kname),
                         "kernel": kname, "kernel_ms": kms,
                         "distance_evals_per_s": evals / (kms / 1e3),
                         "peak_note": "measured FADD+FMNMX lane-op rate of this GPU (gc_probe_fp32); "
                                      f"FFMA {fma_flops / 1e12:.1f} TFLOP/s"},
            "clocks": clocks,
        }
        # the end-to-end objects that create plans per call run first, while
        # the device pool holds only blocks of this workload's sizes; the
        # batched and 1000 x 5000 objects (tens of GB each) run last
        if ws == 1 and not args.no_te:
            try:
                out["te"] = te_variant(gc, torch, x, k, 1, dev, local, mix_ops, cpu=not args.no_cpu_baseline)
            except Exception as e:  # noqa: BLE001
                out["te"] = {"unavailable": str(e)}
        if ws == 1 and not args.no_screen:
            try:
                out["screened"] = screened_variant(gc, x_pinned, k, e2e_s, local)
            except Exception as e:  # noqa: BLE001
                out["screened"] = {"unavailable": str(e)}
        if ws == 1 and not args.no_batch:
            gc.release_cache()
            try:
                out["batch"] = batch_variant(gc, local)
            except Exception as e:  # noqa: BLE001
                out["batch"] = {"unavailable": str(e)}
        if ws == 1 and not args.no_large:
            gc.release_cache()
            try:
                out["large"] = large_variant(gc, torch, dev, local, mix_ops)
            except Exception as e:  # noqa: BLE001
                out["large"] = {"unavailable": str(e)}
        if ws == 1 and not args.no_cpu_baseline:
            try:
                out["cpu_baseline"] = cpu_baseline_sample(x, k, args.cpu_seconds)
                out["cpu_baseline"]["legacy_gpu"] = legacy_gpu_sample()
            except Exception as e:  # noqa: BLE001
                out["cpu_baseline"] = {"unavailable": str(e)}
        print(json.dumps(out))
    plan.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-screen", action="store_true", help="skip the MLP-screened variant")
    ap.add_argument("--no-te", action="store_true", help="skip the transfer-entropy object")
    ap.add_argument("--no-large", action="store_true", help="skip the 1000 x 5000 configuration")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched uneven workload")
    ap.add_argument("--te-only", action="store_true", help="time the transfer-entropy object alone")
    ap.add_argument("--natoms", type=int, default=0, help="smaller atom count (profiling cases only)")
    ap.add_argument("--path", type=int, default=0, help="0 fast (default), 1 exact FP64")
    args = ap.parse_args(argv)
    args.warmup = max(args.warmup, 3)  # timing rule: at least three untimed warm-up steps
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
