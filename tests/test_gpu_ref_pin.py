"""The CUDA path against the reference's own device kernels (needs a B200).

The fixtures tests/golden/ref_<case>.npz hold what the reference's kernels computed for four seeded
boxes (oracle/ref_harness.cu; tests/golden/make_ref_golden.py).  Here the same boxes go through
the library's script surface (read_data of the same particles, the same styles and
coefficients, reset_timestep to the same step) and its setup pass -- rebuild, density, forces --
is compared with them:

  sort permutation (tags in internal order), packed FP32 positions (x, y, z and the type byte
  of w; the library packs its own wall flags above it), TEA signatures                bit-exact
  neighbour rows of every particle as (count, order-free hash of the neighbour tags): the
  reference's full rows on boxes that keep the full list, its rows reduced by the pair-once
  rule (owned entries and those within r_d + skin + 1e-3) otherwise                   bit-exact
  rho: the same FP32 terms (hardware rsqrt); summed in FP32 here, in FP64 by the reference
                                                                  |d rho_i| <= 2e-6 * mean rho
  force (FP32 pair arithmetic, exact FP64 gaussian, against the reference's FP64 arithmetic on
  the same FP32 inputs and its own rho): |dF_i| <= 1e-5 * max(|F_i|, F_rms), F_rms the RMS of
  |F_i| over the box; the per-particle relative error is printed (pytest -s)
"""
import json
import os
import sys

import numpy as np
import pytest

import mdpd

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLDEN)
import make_ref_golden as G  # noqa: E402

CASES = [c for c in G.CASES if os.path.exists(os.path.join(GOLDEN, f"ref_{c}.npz"))]


def write_data(c, path):
    with open(path, "w") as f:
        f.write("seeded case of tests/golden/make_ref_golden.py\n\n")
        f.write(f"{c['n']} atoms\n{c['ntype']} atom types\n\n")
        for d, ax in enumerate("xyz"):
            f.write(f"{float(c['lo'][d])!r} {float(c['hi'][d])!r} {ax}lo {ax}hi\n")
        f.write("\nMasses\n\n")
        for t in range(c["ntype"]):
            f.write(f"{t + 1} {c['mass'][t]!r}\n")
        f.write("\nAtoms\n\n")
        for i in range(c["n"]):
            x = c["x"][i]
            f.write(f"{c['tag'][i]} {c['type'][i]} {float(x[0])!r} {float(x[1])!r} {float(x[2])!r}\n")
        f.write("\nVelocities\n\n")
        for i in range(c["n"]):
            v = c["v"][i]
            f.write(f"{c['tag'][i]} {float(v[0])!r} {float(v[1])!r} {float(v[2])!r}\n")


def box_of(c, tmp_path):
    data = tmp_path / f"{c['name']}.data"
    write_data(c, data)
    lam = mdpd.Lammps()
    lines = [
        "units lj", "dimension 3", "boundary p p p",
        f"atom_style mdpd/atomic/meso {c['rho_est']}",
        f"neighbor {c['skin']} bin", "neigh_modify every 1 delay 0 check yes",
        f"read_data {data}",
    ]
    if c["arb_bc"]:
        lines += ["group fluid type 1", "group wall type 2",
                  f"pair_style mdpd/meso {c['kT']} {c['cutforce']} {c['seed']} fluid wall"]
    else:
        lines += [f"pair_style mdpd/meso {c['kT']} {c['cutforce']} {c['seed']}"]
    for (a, b), (A, B, g, rc, rd) in c["pair"].items():
        lines.append(f"pair_coeff {a} {b} {A} {B} {g} {rc} {rd}")
    lines.append("pair_modify rng exact")
    if c["arb_bc"]:
        lines.append(f"fix BC all aboundary/rho/meso cut_rho {c['cut_rho']} phi_c {c['phi_c']} cut_phi {c['cut_phi']} "
                     f"rho_wall {c['rho_wall']} wall wall mobile fluid")
        lines.append("fix NVE fluid nve/meso")
    else:
        lines.append(f"fix BC all aboundary/rho/meso cut_rho {c['cut_rho']}")
        lines.append("fix NVE all nve/meso")
    lines += [f"timestep {c['dt']}", f"reset_timestep {c['step']}", "run_style mvv/meso"]
    lam.commands("\n".join(lines))
    return lam


def rows_by_tag(n, ti, tj):
    """(count, hash) of each tag's row from the (tag_i, tag_j) pairs of a build."""
    o = np.argsort(ti, kind="stable")
    ti, tj = ti[o], tj[o]
    count = np.bincount(ti - 1, minlength=n)
    return count, G.row_hash(count, tj)


@pytest.fixture(scope="module", params=CASES)
def setup_case(request, tmp_path_factory):
    c = G.make_case(request.param)
    F = np.load(os.path.join(GOLDEN, f"ref_{request.param}.npz"))
    assert json.loads(str(F["meta"]))["input_sha256"] == G.input_sha(c)
    lam = box_of(c, tmp_path_factory.mktemp(request.param))
    lam.setup()
    yield c, F, lam
    lam.close()


def test_permutation_bit_exact(setup_case):
    c, F, lam = setup_case
    assert np.array_equal(lam.field("tag"), F["perm_tags"])


def test_rows_bit_exact(setup_case):
    c, F, lam = setup_case
    ti, tj = lam.pairs()
    count, h = rows_by_tag(c["n"], ti, tj)
    full = bool(c["arb_bc"])  # wall-coupled boxes keep the full list; pair-once boxes reduce it
    want_c, want_h = (F["full_count"], F["full_hash"]) if full else (F["red_count"], F["red_hash"])
    assert np.array_equal(count, want_c)
    assert np.array_equal(h, want_h)


def test_packed_positions_and_signatures_bit_exact(setup_case):
    c, F, lam = setup_case
    if "pos_bits" not in F:
        pytest.skip("large case: packed bits not stored")
    n = c["n"]
    order = np.argsort(lam.field("tag"))
    bits = lam.field("pos4")[:n].view(np.uint32)[order].copy()
    bits[:, 3] &= 0xFF  # type - 1; bits 8 and up hold the library's mobile/wall flags
    assert np.array_equal(bits, F["pos_bits"])
    assert np.array_equal(lam.field("vel4")[:n, 3].view(np.uint32)[order], F["sig"])


def test_density_matches_reference(setup_case):
    c, F, lam = setup_case
    order = np.argsort(lam.field("tag"))
    rho = lam.field("rho")[:c["n"]].astype(np.float64)[order]
    err = np.abs(rho - F["rho"])
    print(f"\n{c['name']}: rho max |d| / mean = {err.max() / F['rho'].mean():.2e}, "
          f"max rel = {(err / np.maximum(F['rho'], 1e-30)).max():.2e}")
    assert err.max() <= 2e-6 * F["rho"].mean()


def test_force_matches_reference(setup_case):
    c, F, lam = setup_case
    if c["arb_bc"]:
        pytest.skip("wall-coupled forces need the wall fraction of a step (tests/test_gpu_walls.py)")
    order = np.argsort(lam.field("tag"))
    f = lam.field("force")[:c["n"], :3].astype(np.float64)[order][F["sample_tags"] - 1]
    fr = F["force"]
    mag = np.linalg.norm(fr, axis=1)
    err = np.linalg.norm(f - fr, axis=1)
    frms = np.sqrt(np.mean(mag ** 2))
    rel = err / mag
    print(f"\n{c['name']}: force |dF_i|/|F_i| median {np.median(rel):.2e} p99 {np.quantile(rel, 0.99):.2e} "
          f"p99.9 {np.quantile(rel, 0.999):.2e} max {rel.max():.2e}; max |dF_i|/F_rms {err.max() / frms:.2e}")
    assert np.all(err <= 1e-5 * np.maximum(mag, frms))
