"""MILCA entry points on the host side (no GPU needed): argument errors are
reported before any device work, there is no CPU fallback, and the
reference harness runs every function of the family."""
import numpy as np
import pytest

from gmx_correlation_b200.milca import NAMES, default_scal, milca, psi_table


def test_invalid_arguments_fail_before_device(gc):
    rng = np.random.default_rng(0)
    rows = rng.random((2, 60))
    with pytest.raises(gc.GCError, match="K < N") as e:
        milca("mi2", rows, 60)
    assert e.value.status == 1
    with pytest.raises(gc.GCError, match="1-D boxes"):
        milca("red", rows, 3, scal=np.array([1e6, 1e6]))
    with pytest.raises(gc.GCError, match="1024"):
        milca("redK", rng.random((2, 3000)), 1100)
    with pytest.raises(gc.GCError, match="dimx, dimy"):
        milca("mi_xnyn", rng.random((3, 60)), 3, dimx=0, dimy=3)
    with pytest.raises(gc.GCError, match="dim >= 2"):
        milca("redr_embed", rows[:1], 3, dim=1, edim=2, tau=1)
    bad = rows.copy()
    bad[1, 7] = np.nan
    with pytest.raises(gc.GCError) as e:
        milca("mi2", bad, 3)
    assert e.value.status == 5  # GC_ERR_NONFINITE


def test_no_cpu_fallback(gc):
    if gc.gpu_available():
        pytest.skip("a GPU is present")
    with pytest.raises(gc.GCError) as e:
        milca("mi2", np.random.default_rng(1).random((2, 80)), 4)
    assert e.value.status == 2  # GC_ERR_NO_DEVICE


def test_reference_harness_runs_every_function():
    from oracle import Reference

    if not Reference.available():
        pytest.skip("reference not built")
    ref = Reference()
    rng = np.random.default_rng(2)
    N, k = 120, 4
    psi = psi_table(N)
    shapes = {"red": 3, "redc": 3, "redr": 3, "redK": 3, "redr_embed": 2, "mi_xnyn": 4, "mic_xnyn": 4,
              "mir_xnyn": 4, "mi_xnynK": 4, "mi_xnynKembed": 4, "mi_d": 2}
    for name in NAMES:
        D = shapes.get(name, 2)
        rows = rng.random((D, N))
        kw = {}
        if name in ("mi_xnyn", "mic_xnyn", "mir_xnyn", "mi_xnynK"):
            kw = {"dimx": 2, "dimy": 2}
        elif name == "mi_xnynKembed":
            kw = {"dim": 2}
        elif name == "redr_embed":
            kw = {"edim": 2, "tau": 1}
        elif name == "mi_d":
            kw = {"phi": np.array([0.0] + [psi[i] - 1.0 / i for i in range(1, k + 1)]),
                  "minmax": (0.0, 1.0, 0.0, 1.0)}
        out, outf, sorted_rows = ref.milca(name, rows, k, psi=psi, scal=default_scal(rows), **kw)
        vals = outf if name == "mi_d" else out
        assert np.isfinite(vals[: 2 * k if name in ("mi2K", "redK", "mi_xnynK", "mi_xnynKembed", "mi_d") else 2]).any()
        # every function but redr_embed sorts its caller's rows in place
        assert np.array_equal(np.sort(sorted_rows, axis=1), np.sort(rows, axis=1))
        assert (name == "redr_embed") == np.array_equal(sorted_rows, rows), name
