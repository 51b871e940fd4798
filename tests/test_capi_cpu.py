"""C-ABI library: loads, exports every declared symbol, parses scripts (no GPU calls)."""
import ctypes
import os
import re
import subprocess

import pytest

import mdpd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    with open(os.path.join(ROOT, "include", "mdpd.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char \*)\s*\*?(mdpd_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    names = declared()
    assert len(names) >= 30
    L = mdpd.lib()
    for n in names:
        assert hasattr(L, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", mdpd.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (mdpd_\w+)", out))
    assert set(names) <= exported


def test_cli_binary_built():
    exe = os.path.join(os.path.dirname(mdpd.LIB_PATH), "lmp_mdpd")
    assert os.access(exe, os.X_OK)


def test_script_variables_and_parse_errors():
    L = mdpd.Lammps(device=0)
    L.commands("""
variable cut_att equal 1.00
variable skin equal 0.3*${cut_att}
variable n equal round(100.0)
units lj
dimension 3
boundary p p p
neighbor ${skin} bin
neigh_modify every 1 delay 0 check yes
""")
    with pytest.raises(mdpd.MdpdError) as e:
        L.command("atom_style mdpd/atomic/meso")
    assert e.value.code == mdpd.ERR_PARSE and "estimation" in str(e.value)
    L.command("atom_style mdpd/atomic/meso 6")
    L.command("region box block 0 10 0 10 0 10 units box")
    L.command("create_box 1 box")
    L.command("create_atoms 1 random 600 4321 box")
    assert L.natoms() == 600
    L.command("mass 1 1.0")
    L.command("pair_style mdpd/meso 1.0 1.0 123456")
    with pytest.raises(mdpd.MdpdError) as e:
        L.command("pair_coeff 1 1 -40 25 4.5 0.5 0.75")
    assert "cutA should be larger than cutB" in str(e.value)
    L.command("pair_coeff * * -40 25 4.5 1.0 0.75")
    with pytest.raises(mdpd.MdpdError) as e:
        L.command("fix BC all aboundary/rho/meso")
    assert "not set properly" in str(e.value)
    # fix aboundary/meso: the reference's errors (fix_aboundary_meso.cu:46-77)
    L.command("group fluid type 1")
    with pytest.raises(mdpd.MdpdError) as e:
        L.command("fix W fluid aboundary/meso wall nosuch rc 1.0 rho 8.0")
    assert "Undefined wall group id in fix aboundary/meso" in str(e.value)
    with pytest.raises(mdpd.MdpdError) as e:
        L.command("fix W fluid aboundary/meso wall all rc 1.0")
    assert "Fix aboundary/meso usage: aboundary/meso <wall groupid> <rc double> <rho double>" in str(e.value)
    L.command("fix W fluid aboundary/meso wall all rho 8.0 sigma 0.1 rc 1.0 frac 0.3")  # keywords in any order
    assert "overlapped" not in L.log  # the reference compares the two groups' bits
    L.command("fix W fluid aboundary/meso wall fluid rho 8.0 rc 1.0")
    assert "mobile and wall group overlapped" in L.log
    L.command("unfix W")
    with pytest.raises(mdpd.MdpdError) as e:
        L.command("frobnicate 1 2 3")
    assert e.value.code == mdpd.ERR_PARSE
    with pytest.raises(mdpd.MdpdError) as e:
        L.command("run_style verlet")
    assert e.value.code == mdpd.ERR_PARSE
    L.close()


def test_create_atoms_random_matches_lammps_park_generator():
    # CreateAtoms::add_random draws x,y,z from RanPark(seed) inside the box bounds
    L = mdpd.Lammps()
    L.commands("""
units lj
atom_style dpd/atomic/meso
region box block 0 10 0 10 0 10 units box
create_box 1 box
create_atoms 1 random 5 574856 box
""")
    x, v, tag, typ = L.state()
    seed = 574856
    def park():
        nonlocal seed
        k = seed // 127773
        seed = 16807 * (seed - k * 127773) - 2836 * k
        if seed < 0:
            seed += 2147483647
        return seed / 2147483647.0
    for i in range(5):
        ref = [10.0 * park() for _ in range(3)]
        assert abs(x[i] - ref).max() < 1e-12
    L.close()


def test_lattice_fcc_count():
    L = mdpd.Lammps()
    L.commands("""
units lj
atom_style mdpd/atomic/meso 4
lattice fcc 4.0
region box block 0 10 0 10 0 10
create_box 1 box
region slab block 4 6 0 10 0 10
create_atoms 1 region slab
""")
    # fcc at reduced density 4 has a = 1; a 2x10x10 slab (faces included on x) holds ~ 4*200 sites
    assert 800 <= L.natoms() <= 1000
    L.close()
