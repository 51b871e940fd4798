"""The reference's example decks run unchanged through the script surface (mdpd_file), and the
data/dump I/O round trips (needs a B200).

Decks (examples/v2.5, copied verbatim to tests/golden/decks by tests/golden/make_golden.py):
  box_10x10x10/in.test           7,000 mDPD particles, two fluid types, fix aboundary/rho/meso
                                 with empty wall groups, 10,000 steps: every thermo line is
                                 written, the run ends clean, T within 2% of kT over its second half
  liquid_vacuum_interface/in.gpu.water
                                 an fcc-lattice slab of 820,000 particles, skin 1.0 checked every
                                 4 steps, fix density/meso profiles along x, 10,000 steps: the
                                 profiles are written, the liquid stays a slab with vacuum beside it
  static_contact_angle_.../in.gpu.static_contact
                                 run verbatim (its A_SL = -20): the fluid's y density profile
                                 against the reference's own out.profile.a_-20; with the one
                                 A_att_12 line changed to -35 (as the reference's authors ran it)
                                 against out.profile.a_-35; bulk bins within 2%, wall-adjacent
                                 within 4%; its dump custom id type xs ys zs is read back
I/O: write_data -> read_data reproduces positions, velocities and types bit for bit.
The quasi-2D pore deck needs init_solids_fluids.dat, which the reference tree does not hold.
"""
import gzip
import json
import os
import shutil

import numpy as np
import pytest

import mdpd

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def deck_text(name):
    with open(os.path.join(GOLDEN, "decks", name)) as f:
        return f.read()


def run_deck(tmp_path, monkeypatch, name, text=None):
    (tmp_path / name).write_text(text if text is not None else deck_text(name))
    monkeypatch.chdir(tmp_path)
    lam = mdpd.Lammps()
    lam.file(name)
    return lam


def thermo_rows(log):
    """numeric thermo rows (Step Temp E_pair E_mol TotEng Press) of a LAMMPS log"""
    rows = []
    for line in log.splitlines():
        t = line.split()
        if len(t) == 6:
            try:
                rows.append([float(x) for x in t])
            except ValueError:
                pass
    return np.array(rows)


def test_box_deck_runs_verbatim(tmp_path, monkeypatch):
    lam = run_deck(tmp_path, monkeypatch, "in.test")
    t = lam.thermo()
    rows = thermo_rows(lam.log)
    lam.close()
    assert t.status == 0 and t.natoms == 7000 and t.step == 10000
    assert np.array_equal(rows[:, 0], np.arange(0, 10001, 100))  # thermo 100
    temp = rows[len(rows) // 2:, 1]
    assert abs(temp.mean() - 1.0) < 0.02, temp.mean()
    assert np.max(np.abs(t.momentum)) < 1e-6 * t.natoms


def test_water_slab_deck_runs_verbatim(tmp_path, monkeypatch):
    lam = run_deck(tmp_path, monkeypatch, "in.gpu.water")
    t = lam.thermo()
    rows = thermo_rows(lam.log)
    lam.close()  # the density fix writes its open window at destruction
    assert t.status == 0 and t.natoms == 820000 and t.step == 10000
    assert np.array_equal(rows[:, 0], np.arange(0, 10001, 100))
    files = sorted((p for p in os.listdir(tmp_path) if p.startswith("out.profile.")),
                   key=lambda p: int(p.rsplit(".", 1)[1]))
    assert len(files) >= 9, files
    prof = np.loadtxt(tmp_path / files[-1])
    assert prof.shape == (50, 2)
    # particles per bin along x (the window's mean): every particle is counted, and they form a
    # liquid slab near the middle with vacuum far from it
    cnt = prof[:, 1]
    assert abs(cnt.sum() - 820000) < 1.0
    assert np.all(cnt[:10] < 1e-3 * cnt.max()) and np.all(cnt[-10:] < 1e-3 * cnt.max()), cnt
    assert abs(rows[len(rows) // 2:, 1].mean() - 1.0) < 0.02


def static_contact(tmp_path, monkeypatch, a_sl):
    with gzip.open(os.path.join(GOLDEN, "static_contact_init.dat.gz"), "rb") as f, \
            open(tmp_path / "LAMMPS_init_noimage.dat", "wb") as g:
        shutil.copyfileobj(f, g)
    text = deck_text("in.gpu.static_contact")
    if a_sl != -20:  # the deck's own value; the reference's other runs changed this one line
        line = next(l for l in text.splitlines() if l.split()[:2] == ["variable", "A_att_12"])
        text = text.replace(line, line.replace("-20", str(a_sl)))
    lam = run_deck(tmp_path, monkeypatch, "in.gpu.static_contact", text)
    t = lam.thermo()
    lam.close()
    assert t.status == 0 and t.step == 100000
    files = sorted(p for p in os.listdir(tmp_path) if p.startswith("out.profile."))
    assert files, os.listdir(tmp_path)
    prof = np.loadtxt(tmp_path / files[-1])
    ref = np.array(json.load(open(os.path.join(GOLDEN, "static_contact_profiles.json")))["gpu"][str(a_sl)])
    assert np.allclose(prof[:, 0], ref[:, 0])
    assert abs(prof[:, 1].sum() - 4000) < 1.0
    bulk = slice(2, 8)
    rel = np.abs(prof[bulk, 1] - ref[bulk, 1]) / ref[bulk, 1]
    assert np.all(rel < 0.02), (prof[:, 1], ref[:, 1])
    assert np.all(np.abs(prof[[1, 8], 1] - ref[[1, 8], 1]) / ref[[1, 8], 1] < 0.04), (prof[:, 1], ref[:, 1])
    return tmp_path


def read_dump_frames(path):
    frames = []
    with open(path) as f:
        lines = f.read().splitlines()
    k = 0
    while k < len(lines):
        assert lines[k] == "ITEM: TIMESTEP"
        step = int(lines[k + 1])
        assert lines[k + 2] == "ITEM: NUMBER OF ATOMS"
        n = int(lines[k + 3])
        assert lines[k + 4].startswith("ITEM: BOX BOUNDS pp pp pp")
        bounds = np.array([[float(x) for x in lines[k + 5 + d].split()] for d in range(3)])
        assert lines[k + 8] == "ITEM: ATOMS id type xs ys zs"
        atoms = np.array([[float(x) for x in l.split()] for l in lines[k + 9:k + 9 + n]])
        frames.append((step, bounds, atoms))
        k += 9 + n
    return frames


def test_static_contact_deck_verbatim_a20_and_its_dump(tmp_path, monkeypatch):
    d = static_contact(tmp_path, monkeypatch, -20)
    frames = read_dump_frames(d / "out.lammpstrj")
    assert [f[0] for f in frames] == list(range(0, 100001, 1000))  # dump every 1000 after the reset
    step, bounds, atoms = frames[-1]
    assert np.allclose(bounds, [[-30, 30], [-5, 5], [-2.5, 2.5]])
    assert np.array_equal(np.sort(atoms[:, 0]), np.arange(1, 9281))
    assert set(np.unique(atoms[:, 1])) == {1.0, 2.0}
    assert atoms[:, 2:].min() > -0.05 and atoms[:, 2:].max() < 1.05  # scaled coordinates


def test_static_contact_deck_a35(tmp_path, monkeypatch):
    static_contact(tmp_path, monkeypatch, -35)


def test_write_data_read_data_round_trip(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    setup = """
units lj
atom_style mdpd/atomic/meso 6.05
neighbor 0.3 bin
{box}
mass 1 1.0
mass 2 1.0
pair_style mdpd/meso 1.0 1.0 4242
pair_coeff 1 1 -40 25 4.5 1.0 0.75
pair_coeff 1 2 -35 25 4.5 1.0 0.75
pair_coeff 2 2 -45 25 4.5 1.0 0.75
fix BC all aboundary/rho/meso cut_rho 0.75
fix NVE all nve/meso
timestep 0.01
run_style mvv/meso
"""
    a = mdpd.Lammps()
    a.commands(setup.format(box="region box block 0 8 0 8 0 8 units box\ncreate_box 2 box\n"
                                "create_atoms 1 random 2000 11 box\ncreate_atoms 2 random 1000 12 box\n"
                                "velocity all create 1.0 13 dist gaussian"))
    a.run(50)
    a.command("write_data snap.data")
    xa, va, _, ta = a.state()
    a.close()
    b = mdpd.Lammps()
    b.commands(setup.format(box="read_data snap.data"))
    xb, vb, _, tb = b.state()
    b.close()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb) and np.array_equal(ta, tb)
