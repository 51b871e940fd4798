"""The index-check build (-DMDPD_CHECK) without a GPU.

1. The check macros of the device header, compiled by nvcc into a host program: with
   -DMDPD_CHECK an index inside [0, n) passes, one outside gives 0 and sets status bit 64
   (kErrIndex); without it both macros are the identity and never touch the status word.
2. libmdpd_check.so exports every entry point include/mdpd.h declares and reports itself as the
   check build through mdpd_index_checks(); libmdpd.so reports 0.  Neither call touches a GPU.
"""
import ctypes
import os
import re
import subprocess

import pytest

import mdpd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "usermeso-2.0-mdpd_b200")
CHECK_LIB = os.path.join(PKG, "libmdpd_check.so")

PROBE = r"""
#include "mdpd_dev.cuh"
#include <cstdio>
using namespace mdpd;
static int idx(const BoxDesc &B, long long i, long long n) { return MDPD_IDX(i, n); }
static bool in(const BoxDesc &B, long long i, long long n) { return MDPD_IN(i, n); }
int main()
{
    static BoxState st{};
    static BoxDesc B{};
    B.st = &st;
    B.nlocal = 100, B.ghost_cap = 40, st.nghost = 50;
    const long long cases[][2] = {{5, 10}, {0, 1}, {10, 10}, {-1, 10}, {1LL << 32, 10}};
    for (auto &c : cases) {
        st.status = 0;
        const int r = idx(B, c[0], c[1]);
        printf("idx %d %d\n", r, st.status);
    }
    for (auto &c : cases) {
        st.status = 0;
        const int r = in(B, c[0], c[1]);
        printf("in %d %d\n", r, st.status);
    }
    printf("n_all %d\n", n_all(B));
    return 0;
}
"""


def run_probe(tmp_path, check):
    src = tmp_path / "probe.cu"
    src.write_text(PROBE)
    exe = tmp_path / ("probe_check" if check else "probe")
    cmd = ["nvcc", "-std=c++17", "--expt-relaxed-constexpr", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I" + os.path.join(PKG, "csrc"), "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)]
    if check:
        cmd.insert(1, "-DMDPD_CHECK")
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")


def test_check_macros_flag_and_skip_out_of_range_indices(tmp_path):
    out = run_probe(tmp_path, True)
    # in range: the index itself, no status; out of range: 0 and bit 64
    assert out[:5] == ["idx 5 0", "idx 0 0", "idx 0 64", "idx 0 64", "idx 0 64"]
    assert out[5:10] == ["in 1 0", "in 1 0", "in 0 64", "in 0 64", "in 0 64"]
    # locals plus the ghosts of the last build, capped at the ghost capacity
    assert out[10] == "n_all 140"


def test_normal_build_macros_are_the_identity(tmp_path):
    out = run_probe(tmp_path, False)
    assert out[:4] == ["idx 5 0", "idx 0 0", "idx 10 0", "idx -1 0"]
    assert all(line == "in 1 0" for line in out[5:10])


def test_check_library_exports_and_reports_itself():
    assert os.path.exists(CHECK_LIB), "libmdpd_check.so not built: python usermeso-2.0-mdpd_b200/build.py --check"
    with open(os.path.join(ROOT, "include", "mdpd.h")) as f:
        names = set(re.findall(r"^\s*(?:int|void|const char \*)\s*\*?(mdpd_\w+)\s*\(", f.read(), re.M))
    out = subprocess.run(["nm", "-D", "--defined-only", CHECK_LIB], capture_output=True, text=True).stdout
    assert "mdpd_index_checks" in names
    assert names <= set(re.findall(r" T (mdpd_\w+)", out))
    chk = ctypes.CDLL(CHECK_LIB)
    assert chk.mdpd_index_checks() == 1
    if os.environ.get("MDPD_LIB") is None:
        assert not mdpd.index_checks()
