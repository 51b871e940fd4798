"""Morton rank of the bins (the reorder's bucket order, atom_meso.cu:271-387 visits bins in
Morton order) computed in closed form by morton_rank (csrc/mdpd_dev.cuh), the function the
device kernel k_bin_ranks runs per bin: compiled by nvcc into a host program and checked
against the ranks of a sort of the bins' Morton codes, on grid shapes that are and are not
powers of two.  No GPU."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "usermeso-2.0-mdpd_b200", "csrc")

PROBE = r"""
#include "mdpd_dev.cuh"
#include <cstdio>
#include <cstdlib>
using namespace mdpd;
int main(int argc, char **argv)
{
    const int mx = atoi(argv[1]), my = atoi(argv[2]), mz = atoi(argv[3]);
    for (int b = 0; b < mx * my * mz; ++b)
        printf("%d %llu\n", morton_rank(b % mx, (b / mx) % my, b / (mx * my), mx, my, mz),
               (unsigned long long)morton3(b % mx, (b / mx) % my, b / (mx * my)));
    return 0;
}
"""

SHAPES = [(3, 3, 3), (8, 8, 8), (5, 7, 3), (16, 9, 4), (33, 3, 17), (1, 1, 1), (64, 2, 3)]


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    d = tmp_path_factory.mktemp("morton")
    src = d / "probe.cu"
    src.write_text(PROBE)
    exe = d / "probe"
    subprocess.run(["nvcc", "-std=c++17", "-O1", "-I" + CSRC, str(src), "-o", str(exe)], check=True,
                   capture_output=True)
    return str(exe)


@pytest.mark.parametrize("shape", SHAPES)
def test_rank_equals_sorted_morton_order(probe, shape):
    out = subprocess.run([probe] + [str(m) for m in shape], check=True, capture_output=True, text=True).stdout
    a = np.array([[int(t) for t in line.split()] for line in out.split("\n") if line], dtype=np.uint64)
    rank, code = a[:, 0].astype(np.int64), a[:, 1]
    expect = np.empty(len(code), np.int64)
    expect[np.argsort(code, kind="stable")] = np.arange(len(code))
    assert np.array_equal(rank, expect)
