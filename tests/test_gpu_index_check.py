"""The unit known-answer tests again on the index-check build (libmdpd_check.so, -DMDPD_CHECK):
sort permutation, pair sets, RNG words, density and forces against the oracle, deterministic
replay, wall coupling and fix aboundary/meso.  Every neighbour, bin, bucket and permutation
index those kernels use is bounds-checked there; an index outside its array would set status
bit 64 and fail the run with MDPD_ERR_OVERFLOW naming it.  The tests run in a child pytest with
MDPD_LIB pointing at the check library, so the same assertions hold with the checks compiled in.
"""
import os
import re
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECK_LIB = os.path.join(ROOT, "usermeso-2.0-mdpd_b200", "libmdpd_check.so")
KATS = ["tests/test_gpu_parity.py", "tests/test_gpu_walls.py", "tests/test_gpu_aboundary_meso.py"]


@pytest.mark.gpu
def test_parity_kats_pass_on_the_index_check_build():
    assert os.path.exists(CHECK_LIB), "libmdpd_check.so not built: python usermeso-2.0-mdpd_b200/build.py --check"
    env = dict(os.environ, MDPD_LIB=CHECK_LIB)
    probe = subprocess.run([sys.executable, "-c", "import sys; sys.path.insert(0, 'usermeso-2.0-mdpd_b200'); "
                            "import mdpd; print(mdpd.index_checks())"],
                           cwd=ROOT, env=env, capture_output=True, text=True, timeout=120)
    assert probe.stdout.strip() == "True", probe.stdout + probe.stderr
    r = subprocess.run([sys.executable, "-m", "pytest", "-x", "-q", "-m", "gpu", "-p", "no:cacheprovider"] + KATS,
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    # every collected test of the three files ran and passed
    c = subprocess.run([sys.executable, "-m", "pytest", "--collect-only", "-q", "-m", "gpu", "-p", "no:cacheprovider"]
                       + KATS, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    n = re.search(r"(\d+)(?:/\d+)? tests? collected", c.stdout)
    m = re.search(r"(\d+) passed", r.stdout)
    assert n and m and int(m.group(1)) == int(n.group(1)) >= 20, c.stdout[-1000:] + r.stdout[-2000:]
