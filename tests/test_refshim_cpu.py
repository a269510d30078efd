"""The CPU-baseline build of the reference's own code (oracle/_ref).

* The MKL-VSL stand-in it links (oracle/refshim/vsl_standin.cpp) is pinned:
  MT19937's published known answer (10000th output 4123659995 for seed
  5489), the inverse-CDF Gaussian within Acklam's stated 1.15e-9 relative
  error of the normal quantile, and uniform / Gaussian banks that pass a
  Kolmogorov-Smirnov test.
* The built reference executable (when present) runs a short quick_test
  input and writes its statistics files.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "oracle", "refshim")
REF = os.path.join(ROOT, "oracle", "_ref", "langevinDynamicsSingleBarrier")
GOLDEN = os.path.join(ROOT, "tests", "golden", "inp")

HARNESS = r"""
#include "vsl_standin.cpp"
extern "C" uint32_t mt_nth(uint32_t seed, int n) {
    Mt19937 m; m.seed(seed); uint32_t v = 0;
    for (int i = 0; i < n; ++i) v = m.next();
    return v;
}
extern "C" double normal_quantile(double p) { return quantile(p); }
"""


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    d = tmp_path_factory.mktemp("shim")
    src = d / "h.cpp"
    src.write_text(HARNESS)
    so = d / "h.so"
    subprocess.run(["g++", "-O2", "-shared", "-fPIC", "-I", SHIM, str(src), "-o", str(so)], check=True)
    h = C.CDLL(str(so))
    h.mt_nth.restype = C.c_uint32
    h.mt_nth.argtypes = [C.c_uint32, C.c_int]
    h.normal_quantile.restype = C.c_double
    h.normal_quantile.argtypes = [C.c_double]
    h.vdRngGaussian.argtypes = [C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_double, C.c_double]
    h.vdRngUniform.argtypes = [C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_double, C.c_double]
    return h


def test_mt19937_known_answer(shim):
    assert shim.mt_nth(5489, 10000) == 4123659995


def test_inverse_cdf_gaussian_accuracy(shim):
    from scipy.stats import norm
    p = np.concatenate([np.linspace(1e-6, 1 - 1e-6, 20001), [1e-300, 1e-100, 1e-20, 1e-10, 0.02425, 0.97575]])
    x = np.array([shim.normal_quantile(v) for v in p])
    ref = norm.ppf(p)
    ok = np.abs(ref) > 1e-12
    assert (np.abs(x - ref)[ok] / np.abs(ref[ok])).max() < 1.15e-9


def test_uniform_and_gaussian_banks(shim):
    from scipy import stats
    s = C.c_void_p()
    shim.vslNewStream(C.byref(s), 0x00200000, 123)
    n = 200_000
    g, u = np.zeros(n), np.zeros(n)
    shim.vdRngGaussian(3, s, n, g.ctypes.data_as(C.POINTER(C.c_double)), 0.0, 1.0)
    shim.vdRngUniform(0, s, n, u.ctypes.data_as(C.POINTER(C.c_double)), 0.0, 1.0)
    shim.vslDeleteStream(C.byref(s))
    assert stats.kstest(g, "norm").pvalue > 1e-3
    assert stats.kstest(u, "uniform").pvalue > 1e-3
    assert u.min() >= 0.0 and u.max() < 1.0


@pytest.mark.skipif(not os.path.exists(REF), reason="reference build absent (make -C oracle ref)")
def test_reference_build_runs_quick_test(tmp_path):
    text = open(os.path.join(GOLDEN, "quick_test__2.0_7.2_m1.0_1.00e-05.inp")).read()
    lines = []
    for ln in text.splitlines():
        w = ln.split()
        key = w[0] if w else ""
        if key == "NUMBEROFSTEPS":
            ln = "NUMBEROFSTEPS 1100000"
        elif key == "FREQSAVE":
            ln = "FREQSAVE 1000"
        elif key in ("WRITERESTART", "WRITEX"):
            ln = f"{key} false"
        lines.append(ln)
    (tmp_path / "q.inp").write_text("\n".join(lines) + "\n")
    r = subprocess.run([REF, "-i", "q.inp"], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    log = (tmp_path / "m1.0_t1.00e-05_0_firstPassageTime.log").read_text()
    assert "# count                         8" in log
    dat = np.fromfile(tmp_path / "m1.0_t1.00e-05_0_firstPassageTime.dat", dtype="<f8")
    assert dat.shape == (8,) and np.all(dat > 0)
