"""gc_ksg_pair_mi_noalloc: the KSG entry point for callers that cannot
allocate device memory (for example a plugin whose host application owns
all device memory through its own pool).  It takes every piece of scratch
from one fixed array inside the library; the caller brings the device
buffers for the coordinates and the result.

Checked through the C ABI against gc_ksg_matrix (the allocating entry
point) on two calls in a row with different shapes, so contents the first
call leaves in the shared array cannot leak into the second.  Both compute
exact neighbour counts, so the pair MI must be bit-identical.  This file is
collected last so that a run stopping at the first failure has already run
every other test; it also passes on its own in a fresh process."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pairs_of(mat):
    n = mat.shape[0]
    return np.array([mat[a1, a2] for a1 in range(1, n) for a2 in range(a1)])


def _call(gc, torch, x, k):
    n, T = x.shape[0], x.shape[1]
    d_xyz = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    d_out = torch.full((n * (n - 1) // 2,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    gc.ksg_pair_mi_noalloc(d_xyz.data_ptr(), n, T, k, d_out.data_ptr(), 0)
    return d_out.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice(gc):
    torch = pytest.importorskip("torch")
    from gmx_correlation_b200.synth import synth_traj
    xa = synth_traj(40, 700, 6, 0.08, seed=41, fp32=True)
    xb = synth_traj(17, 333, 4, 0.05, seed=42)
    got_a = _call(gc, torch, xa, 12)
    got_b = _call(gc, torch, xb, 5)
    np.testing.assert_array_equal(got_a, _pairs_of(gc.kraskov_corrmatrix(xa, 12)))
    np.testing.assert_array_equal(got_b, _pairs_of(gc.kraskov_corrmatrix(xb, 5)))


def test_noalloc_rejects_sizes_beyond_its_limit(gc):
    torch = pytest.importorskip("torch")
    d = torch.zeros(65 * 100 * 3, dtype=torch.float64, device="cuda")
    out = torch.zeros(65 * 64 // 2, dtype=torch.float64, device="cuda")
    with pytest.raises(gc.GCError) as e:
        gc.ksg_pair_mi_noalloc(d.data_ptr(), 65, 100, 5, out.data_ptr(), 0)
    assert e.value.status == 1 and "limited to 64 atoms and 1024 frames" in str(e.value)
    with pytest.raises(gc.GCError) as e:
        gc.ksg_pair_mi_noalloc(d.data_ptr(), 4, 1025, 5, out.data_ptr(), 0)
    assert e.value.status == 1


def test_noalloc_call_reserves_no_device_memory(gc):
    """After the first call (which, under lazy module loading, is what reserves
    the fixed array), a call leaves the device's free memory unchanged."""
    torch = pytest.importorskip("torch")
    from gmx_correlation_b200.synth import synth_traj
    x = synth_traj(24, 500, 4, 0.08, seed=43, fp32=True)
    first = _call(gc, torch, x, 8)
    d_xyz = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    d_out = torch.zeros(24 * 23 // 2, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    gc.ksg_pair_mi_noalloc(d_xyz.data_ptr(), 24, 500, 8, d_out.data_ptr(), 0)
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    np.testing.assert_array_equal(d_out.cpu().numpy(), first)


def test_noalloc_nonfinite_input_then_valid_call(gc):
    """A NaN coordinate reports GC_ERR_NONFINITE through the shared status
    word; the next valid call clears it and still equals gc_ksg_matrix."""
    torch = pytest.importorskip("torch")
    from gmx_correlation_b200.synth import synth_traj
    x = synth_traj(9, 300, 4, 0.08, seed=44)
    bad = x.copy()
    bad[3, 17, 1] = np.nan
    with pytest.raises(gc.GCError) as e:
        _call(gc, torch, bad, 6)
    assert e.value.status == 5
    np.testing.assert_array_equal(_call(gc, torch, x, 6), _pairs_of(gc.kraskov_corrmatrix(x, 6)))
