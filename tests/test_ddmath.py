"""The correctly rounded sin / cos / tan / atan / atan2 / acos / exp of
setsm_b200/csrc/vll_ddmath.cuh (used by the orthoimage rasters' map
projection), compiled for the host: against the C library they differ on
about 0.1% of the arguments, and at every such argument checked, the header's
result is the correctly rounded one (300-bit mpmath), i.e. the library is the
one that misrounds."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "native", "ddmath_check.cpp")
CSRC = os.path.join(ROOT, "setsm_b200", "csrc")


@pytest.fixture(scope="module")
def check_output(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path_factory.mktemp("ddmath") / "ddmath_check")
    subprocess.run([cxx, "-O2", "-std=c++17", "-ffp-contract=off", "-I", CSRC, "-o", exe, SRC],
                   check=True)
    return subprocess.run([exe, "100000"], check=True, capture_output=True, text=True).stdout


def test_mismatch_rate_against_the_c_library(check_output):
    counts = {}
    for line in check_output.splitlines():
        f = line.split()
        if f[0] == "count":
            counts[f[1]] = (int(f[2]), int(f[3]))
    assert set(counts) == {"sin", "cos", "tan", "atan", "atan2", "exp", "acos"}
    for name, (n, bad) in counts.items():
        assert n >= 100000
        assert bad / n < 0.003, (name, bad, n)


def test_every_mismatch_is_the_library_misrounding(check_output):
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.prec = 300
    fns = {"sin": mpmath.sin, "cos": mpmath.cos, "tan": mpmath.tan, "atan": mpmath.atan,
           "exp": mpmath.exp, "acos": mpmath.acos}
    checked = 0
    for line in check_output.splitlines():
        f = line.split()
        if f[0] != "diff":
            continue
        vals = [float.fromhex(v) for v in f[2:]]
        if f[1] == "atan2":
            y, x, ours, lib = vals
            true = mpmath.atan2(mpmath.mpf(y), mpmath.mpf(x))
        else:
            x, ours, lib = vals
            true = fns[f[1]](mpmath.mpf(x))
        # ours is the double nearest the exact value
        assert abs(mpmath.mpf(ours) - true) < abs(mpmath.mpf(lib) - true), line
        checked += 1
    assert checked > 50
