"""Output contract: pearsify and the correl.dat / XPM writers of the product
library (host code, no GPU needed) against the reference's own output."""
import importlib.util
import warnings
from pathlib import Path

import numpy as np
import pytest

from tests.conftest import GOLDEN


def test_write_matrix_bytes(gc, tmp_path):
    m = np.load(GOLDEN / "writers_matrix.npy")
    out = tmp_path / "c.dat"
    gc.write_matrix(m, out)
    assert out.read_bytes() == (GOLDEN / "writers_correl.dat").read_bytes()


def test_pearsify_and_xpm_bytes(gc, tmp_path):
    m = np.load(GOLDEN / "writers_matrix.npy").copy()
    gc.pearsify(m, 3)
    out = tmp_path / "r.dat"
    gc.write_matrix(m, out)
    assert out.read_bytes() == (GOLDEN / "writers_correl_r.dat").read_bytes()
    xpm = tmp_path / "r.xpm"
    gc.write_xpm_matrix(m, xpm, "sel correlation matrix", "r(MI)")
    assert xpm.read_bytes() == (GOLDEN / "writers_correl.xpm").read_bytes()


def test_pearsify_matches_oracle(gc, oracle):
    rng = np.random.default_rng(4)
    m = rng.normal(0.2, 0.5, size=(17, 17))
    m[np.diag_indices(17)] = 2000.0
    want = oracle.pearsify(m)
    got = gc.pearsify(m.copy())
    np.testing.assert_array_equal(got, want)
    assert np.all(got[np.diag_indices(17)] == 1.0)
    assert np.all(got[m <= 0] == 0.0)


def test_read_matrix_round_trip(gc, tmp_path):
    rng = np.random.default_rng(1)
    m = rng.random((23, 23))
    m[np.diag_indices(23)] = 2000.0
    p = tmp_path / "rt.dat"
    gc.write_matrix(m, p)
    back = gc.read_matrix(p)
    np.testing.assert_allclose(back, m, rtol=1e-5, atol=1e-6)
    np.testing.assert_array_equal(np.diag(back), 2000.0)


def test_writer_bad_path(gc):
    import pytest
    with pytest.raises(gc.GCError):
        gc.write_matrix(np.eye(2), "/nonexistent-dir/x.dat")


from oracle import REF_SRC  # noqa: E402

REF_CONSUMER = REF_SRC / "bin" / "analyze_matrix.py"


@pytest.mark.skipif(not REF_CONSUMER.exists(), reason="reference sources not present")
def test_reference_consumer_reads_our_correl_dat(gc, tmp_path):
    """The reference's downstream consumer (bin/analyze_matrix.py:71-102
    read_matrix, :173-190 auto_threshold) reads the correl.dat this library
    writes back to the same matrix, to the writer's %10.6g precision."""
    spec = importlib.util.spec_from_file_location("ref_analyze_matrix", REF_CONSUMER)
    mod = importlib.util.module_from_spec(spec)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")  # its optional plotting/graph imports
        spec.loader.exec_module(mod)
    rng = np.random.default_rng(5)
    m = rng.random((31, 31))
    m = 0.5 * (m + m.T)
    m[np.diag_indices(31)] = 2000.0
    gc.pearsify(m, 3)
    out = tmp_path / "correl.dat"
    gc.write_matrix(m, out)
    theirs = mod.read_matrix(out)
    np.testing.assert_array_equal(theirs, gc.read_matrix(out))
    np.testing.assert_allclose(theirs, m, rtol=1e-5, atol=1e-6)
    iu = np.triu_indices(31, 1)
    vals = theirs[iu][theirs[iu] > 0]
    assert mod.auto_threshold(theirs) == pytest.approx(float(vals.mean() + 0.5 * vals.std()), rel=1e-12)
