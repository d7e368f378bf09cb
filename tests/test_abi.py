"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: these run without a GPU)."""
import ctypes
import re

import numpy as np
import pytest

from tests.conftest import ROOT


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(gc_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("gc_ksg_matrix", "gc_gauss_matrix", "gc_gcmi_matrix", "gc_te_matrix", "gc_pearsify",
                 "gc_write_matrix", "gc_write_xpm", "gc_ksg_plan_create", "gc_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol(gc):
    L = ctypes.CDLL(str(gc.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_opts_defaults(gc):
    o = gc._Opts()
    gc.lib().gc_opts_init(ctypes.byref(o))
    assert o.device == -1 and o.path == 0 and o.pair_begin == 0 and o.pair_end == 0


def test_invalid_arguments_fail_before_device(gc):
    x = np.random.default_rng(0).normal(size=(1, 50, 3))
    with pytest.raises(gc.GCError) as e:
        gc.kraskov_corrmatrix(x, 5)
    assert e.value.status == 1 and "at least 2 atoms" in str(e.value)
    x = np.random.default_rng(0).normal(size=(3, 10, 3))
    with pytest.raises(gc.GCError) as e:
        gc.kraskov_corrmatrix(x, 10)
    assert e.value.status == 1 and "nframes must exceed k" in str(e.value)
    with pytest.raises(gc.GCError) as e:
        gc.gcmi_corrmatrix(np.zeros((3, 5, 3)))
    assert e.value.status == 1


def test_no_device_is_an_error_not_a_fallback(gc):
    if gc.lib().gc_device_count() > 0:
        pytest.skip("a CUDA device is present")
    x = np.random.default_rng(0).normal(size=(3, 40, 3))
    with pytest.raises(gc.GCError) as e:
        gc.kraskov_corrmatrix(x, 4)
    assert e.value.status == 2


def test_cpp_dropin_links_every_reference_symbol(gc, tmp_path):
    """The reference front end's C++ calls (lib/correlation_core.h:65-88,
    lib/gcmi.h:8-10, lib/transfer_entropy.h:8-10, lib/kraskov_gpu.h:20,32)
    resolve against the library: tests/dropin_check.cpp, which calls every one
    of them, links (nothing runs here)."""
    import shutil
    import subprocess
    cxx = "/usr/bin/g++" if shutil.which("/usr/bin/g++") else "g++"
    pkg = ROOT / "gmx_correlation_b200"
    res = subprocess.run([cxx, "-O0", "-std=c++17", f"-I{pkg / 'csrc' / 'dropin'}",
                          str(ROOT / "tests" / "dropin_check.cpp"), "-o", str(tmp_path / "dropin_check"),
                          f"-L{pkg}", "-lgmxcorr_b200", "-Wl,--no-undefined"], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr


def test_cpp_dropin_links_every_milca_function(gc, tmp_path):
    """Code written against the MILCA definitions of lib/kraskov.cpp
    (:347-2155, no header in the reference) links against the library through
    csrc/dropin/kraskov_milca.h with the same signatures (nothing runs here)."""
    import shutil
    import subprocess
    src = tmp_path / "milca_check.cpp"
    src.write_text(r'''
#include "kraskov_milca.h"
int main(int argc, char**)
{
    if (argc > 1) // never taken: only the symbols must resolve
    {
        double *x[4] = {}, psi[8] = {}, scal[4] = {}, a = 0, b = 0, c = 0, d = 0, cr[8] = {};
        float  f[8] = {};
        int    *ip = nullptr, **ipp = nullptr;
        double **dpp = nullptr;
        mi2(x, 8, 1, psi, scal, &a, &b);
        mi2c(x, 8, 1, psi, scal, &a);
        mi2r(x, 8, 1, psi, scal, &b);
        mi2r_(x, 8, 1, psi, scal, &b);
        mi2K(x, 8, 1, psi, scal, cr);
        mi2h(x, 8, 1, psi, scal, &a, &b, &c, &d);
        red(x, 2, 8, 1, psi, scal, &a, &b);
        redc(x, 2, 8, 1, psi, scal, &a);
        redr(x, 2, 8, 1, psi, scal, &b);
        redK(x, 2, 8, 1, psi, scal, cr);
        redr_embed(x, 2, 2, 1, 8, 1, psi, &b);
        mi_xnyn(x, 1, 1, 8, 1, psi, scal, &a, &b);
        mic_xnyn(x, 1, 1, 8, 1, psi, scal, &a);
        mir_xnyn(x, 1, 1, 8, 1, psi, scal, &b);
        mi_xnynK(x, 1, 1, 8, 1, psi, scal, cr);
        mi_xnynKembed(x, 1, 8, 1, dpp, dpp, ipp, ip, ip, ipp, ip, ip, psi, cr);
        mi_d(x, 2, 8, 1, f, psi, psi, 0.0, 1.0, 0.0, 1.0);
    }
    return 0;
}
''')
    cxx = "/usr/bin/g++" if shutil.which("/usr/bin/g++") else "g++"
    pkg = ROOT / "gmx_correlation_b200"
    res = subprocess.run([cxx, "-O0", "-std=c++17", f"-I{pkg / 'csrc' / 'dropin'}", str(src),
                          "-o", str(tmp_path / "milca_check"), f"-L{pkg}", "-lgmxcorr_b200", "-Wl,--no-undefined"],
                         capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
