"""The command-line driver `lmp_mdpd -in script` (the counterpart of `lmp_meso -in script`):
a deck runs to its thermo lines, and a malformed one exits non-zero with the reference's error
text, the process never aborting."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "usermeso-2.0-mdpd_b200")
LMP = os.path.join(PKG, "lmp_mdpd")

DECK = """units lj
atom_style mdpd/atomic/meso 6.05
neighbor 0.3 bin
region box block 0 8 0 8 0 8 units box
create_box 1 box
create_atoms 1 random 3098 4321 box
mass 1 1.0
velocity all create 1.0 5678 dist gaussian
pair_style mdpd/meso 1.0 1.0 2468
pair_coeff 1 1 -40 25 4.5 {cut} 0.75
fix BC all aboundary/rho/meso cut_rho 0.75
fix NVE all nve/meso
timestep 0.01
run_style mvv/meso
thermo 10
run 40
"""


@pytest.fixture(scope="module")
def lmp():
    if not os.path.exists(LMP):  # the command-line program is built beside libmdpd.so
        sys.path.insert(0, PKG)
        import build
        build.build(verbose=False)
    return LMP


def test_cli_runs_a_deck(lmp, tmp_path):
    deck = tmp_path / "in.mdpd"
    deck.write_text(DECK.format(cut=1.0))
    r = subprocess.run([lmp, "-in", str(deck)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    head = [k for k, l in enumerate(lines) if l.split()[:2] == ["Step", "Temp"]]
    assert head, r.stdout
    rows = [l.split() for l in lines[head[-1] + 1:] if l.split() and l.split()[0].isdigit()]
    assert [int(x[0]) for x in rows] == [0, 10, 20, 30, 40]
    assert all(float(x[1]) > 0 for x in rows)


def test_cli_reports_a_malformed_deck(lmp, tmp_path):
    deck = tmp_path / "in.bad"
    deck.write_text(DECK.format(cut=0.5))  # cutA < cutB
    r = subprocess.run([lmp, "-in", str(deck)], capture_output=True, text=True, timeout=300)
    assert r.returncode != 0
    assert "cutA should be larger than cutB" in r.stderr
