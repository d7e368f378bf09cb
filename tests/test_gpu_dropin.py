"""The C++ drop-in interface and the standalone CLI, end to end on the GPU."""
import shutil
import subprocess

import numpy as np
import pytest

from tests.conftest import ROOT

pytestmark = pytest.mark.gpu

PKG = ROOT / "gmx_correlation_b200"


@pytest.fixture(scope="module")
def dropin_bin(tmp_path_factory, gc):
    out = tmp_path_factory.mktemp("dropin") / "dropin_check"
    cxx = "/usr/bin/g++" if shutil.which("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-O1", "-std=c++17", f"-I{PKG / 'csrc' / 'dropin'}", str(ROOT / "tests" / "dropin_check.cpp"),
                    "-o", str(out), f"-L{PKG}", "-lgmxcorr_b200", f"-Wl,-rpath,{PKG}"], check=True)
    return out


def test_dropin_matches_oracle(dropin_bin, oracle, golden, small_x, tmp_path):
    x = small_x[:24].copy()
    n, T = x.shape[0], x.shape[1]
    src = tmp_path / "coords.bin"
    with open(src, "wb") as f:
        np.array([n, T], np.int32).tofile(f)
        x.tofile(f)
    res = subprocess.run([str(dropin_bin), str(src), "10", "2", str(tmp_path) + "/"], capture_output=True,
                         text=True, check=True)
    assert "throw: kraskov_corrmatrix: need at least 2 atoms" in res.stdout
    assert "gpu_available=1" in res.stdout
    assert "kraskov_gpu_probe=1" in res.stdout
    load = lambda name: np.fromfile(tmp_path / name).reshape(n, n)  # noqa: E731
    np.testing.assert_array_equal(load("ksg.bin"), oracle.ksg_matrix(x, 10))
    # legacy kraskov_corrmatrix_gpu on the prepared workspace: every entry written
    np.testing.assert_array_equal(load("ksg_gpu.bin"), oracle.ksg_matrix(x, 10))
    np.testing.assert_allclose(load("gauss.bin"), oracle.gauss_matrix(x), rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(load("gcmi.bin"), oracle.gcmi_matrix(x), rtol=1e-12, atol=1e-14)
    np.testing.assert_array_equal(load("te.bin"), oracle.te_matrix(x, 10, 2))
    X, psi = oracle.prepare(x)
    assert np.fromfile(tmp_path / "wrap.bin")[0] == oracle.ksg_pair_detail(X, psi, 10, 1, 0)["mi"]
    # correl.dat bytes equal the reference writer's on the oracle matrix
    want = tmp_path / "want.dat"
    r = oracle.pearsify(oracle.ksg_matrix(x, 10))
    import gmx_correlation_b200 as gc
    gc.write_matrix(r, want)
    assert (tmp_path / "correl.dat").read_bytes() == want.read_bytes()


def _write_dump(path, x):
    n, T = x.shape[0], x.shape[1]
    with open(path, "w") as f:
        f.write(f"{n} {T}\n")
        for fr in range(T):
            for a in range(n):
                f.write("%.10g %.10g %.10g\n" % tuple(x[a, fr]))


def _read_dump(path):
    with open(path) as f:
        n, T = map(int, f.readline().split())
        v = np.loadtxt(f).reshape(T, n, 3)
    return np.ascontiguousarray(v.transpose(1, 0, 2))


@pytest.mark.parametrize("flags,kind", [([], "ksg"), (["-linear"], "gauss"), (["-gcmi"], "gcmi"),
                                        (["-mi"], "ksg_mi")])
def test_cli_dispatch(gc, oracle, small_x, tmp_path, flags, kind):
    cli = PKG / "gmx_correlation_b200"
    dump = tmp_path / "traj_dump.txt"
    _write_dump(dump, small_x[:16])
    x = _read_dump(dump)
    out = tmp_path / "correl.dat"
    xpm = tmp_path / "correl.xpm"
    subprocess.run([str(cli), "-f", str(dump), "-o", str(out), "-m", str(xpm), "-k", "10", *flags], check=True,
                   capture_output=True)
    if kind == "ksg":
        want = oracle.pearsify(oracle.ksg_matrix(x, 10))
    elif kind == "ksg_mi":
        want = oracle.ksg_matrix(x, 10)
    elif kind == "gauss":
        want = oracle.pearsify(oracle.gauss_matrix(x))
    else:
        want = oracle.pearsify(oracle.gcmi_matrix(x))
    got = gc.read_matrix(out)
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-6)  # %10.6g text
    assert xpm.read_text().startswith("/* XPM */")


def test_cli_te_output(gc, oracle, small_x, tmp_path):
    cli = PKG / "gmx_correlation_b200"
    dump = tmp_path / "traj_dump.txt"
    _write_dump(dump, small_x[:10])
    x = _read_dump(dump)
    ote = tmp_path / "te.dat"
    subprocess.run([str(cli), "-f", str(dump), "-o", str(tmp_path / "c.dat"), "-k", "10", "-te", "-lag", "3", "-ote",
                    str(ote)], check=True, capture_output=True)
    np.testing.assert_allclose(gc.read_matrix(ote), oracle.te_matrix(x, 10, 3), rtol=1e-5, atol=1e-6)


def test_cli_rejects_bad_options(tmp_path):
    cli = PKG / "gmx_correlation_b200"
    r = subprocess.run([str(cli), "-f", "nope.txt", "-fit"], capture_output=True, text=True)
    assert r.returncode != 0 and "fitting" in r.stderr


def test_cli_xtc_input_matches_oracle(gc, oracle, small_x, tmp_path):
    """XTC in, correl.dat out: the KSG matrix of the selected atoms equals the
    oracle's on the positions the oracle's own XTC restatement decodes and
    centres (the reference's frame collection and finishAnalysis)."""
    from oracle import xtc as ox

    cli = PKG / "gmx_correlation_b200"
    frames = np.ascontiguousarray((small_x[:20] + 3.0).transpose(1, 0, 2)).astype(np.float32)
    xtc = tmp_path / "traj.xtc"
    gc.write_trajectory(xtc, frames, precision=10000.0)
    ndx = tmp_path / "index.ndx"
    sel = [1, 4, 5, 9, 12, 13, 17, 20]  # 1-based atom numbers
    ndx.write_text("[ Sel ]\n" + " ".join(map(str, sel)) + "\n")
    out = tmp_path / "correl.dat"
    subprocess.run([str(cli), "-f", str(xtc), "-n", str(ndx), "-sel", "Sel", "-o", str(out), "-k", "10", "-mi"],
                   check=True, capture_output=True)
    pos = np.stack([f[3] for f in ox.read_xtc(xtc)]).transpose(1, 0, 2).astype(np.float64)
    x = ox.center(pos[[s - 1 for s in sel]])
    np.testing.assert_array_equal(gc.read_trajectory(xtc, [s - 1 for s in sel]), x)
    want = tmp_path / "want.dat"
    gc.write_matrix(oracle.ksg_matrix(x, 10), want)
    assert out.read_bytes() == want.read_bytes()
