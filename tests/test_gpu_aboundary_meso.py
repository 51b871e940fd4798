"""fix aboundary/meso (the Gaussian-density wall of fix_aboundary_meso.cu) against the oracle.

A periodic 8 x 8 x 8 box holds a frozen wall slab (z < 2, density 8) and an mDPD fluid above it
(density 6.05, its lowest layer started inside the slab's top so that one step reaches the wall
density threshold) moving into the wall. Two decks differ only in the fix. One step of each (no
neighbour rebuild in it) gives the state before the fix (the deck without it) and after it (the
deck with it); the oracle applies its restatement of the fix to the first, over the reference's
whole rows (oracle rebuild of the same start: the row length the reference passes is core plus
skin after its list join), and must give the second.

Tolerances: positions bit-identical (the fix changes v and f only); the set of reflected particles
identical up to 2 whose wall density lies within FP32 rounding of rho0/2 (CUDA's expf against the
host's); reflected v and f within 1e-4 of (|v| + 1) and (|f| + 1), the magnitudes before the fix.
The wall normal is an FP32 sum of Gaussian-weighted offsets that the device takes in its list's
order and the oracle in the reference's core-then-skin order; its lateral terms largely cancel, so
its direction carries a few 1e-5 of relative rounding (a reflection changes v by O(|v|)).
"""
import numpy as np
import pytest

import mdpd
import oracle

pytestmark = pytest.mark.gpu

L = 8.0
WALL_TOP = 2.0


def slab(seed=77, fluid_bottom=WALL_TOP):
    rng = np.random.default_rng(seed)
    nw = int(8.0 * L * L * WALL_TOP)
    nf = int(6.05 * L * L * (L - fluid_bottom))
    xw = rng.uniform((0, 0, 0), (L, L, WALL_TOP), (nw, 3))
    xf = rng.uniform((0, 0, fluid_bottom), (L, L, L), (nf, 3))
    v = np.concatenate([rng.normal(0, 1, (nf, 3)), np.zeros((nw, 3))])
    v[:nf, 2] -= 1.5  # towards the wall below
    return nf, nw, np.concatenate([xf, xw]), v


def deck(nf, nw, x, v, extra="", delay=5, body=""):
    lam = mdpd.Lammps()
    lam.commands(f"""
units lj
boundary p p p
neighbor 0.3 bin
neigh_modify every 1 delay {delay} check yes
atom_style mdpd/atomic/meso 8
region box block 0 {L} 0 {L} 0 {L} units box
create_box 2 box
create_atoms 1 random {nf} 11 box
create_atoms 2 random {nw} 12 box
group fluid type 1
group solid type 2
mass * 1
pair_style mdpd/meso 1.0 1.0 4321
pair_coeff * * -40 25 4.5 1.0 0.75
fix BC all aboundary/rho/meso cut_rho 0.75
fix NVE fluid nve/meso
{body}
{extra}
timestep 0.01
run_style mvv/meso
""")
    lam.set_state(x, v)  # tags 1..nf are the fluid (type 1)
    return lam


def fix_line(rho0):
    return f"fix W fluid aboundary/meso wall solid rc 1.0 rho {rho0}"


def one_step_parity(nf, nw, x, v, fz=0.0, rho0=8.0):
    """one step of the decks without and with the fix from (x, v), with a body force fz along z
    on the fluid; the fix against the oracle on the total force (the force field reports it, body
    force included, as the reference's f holds it)"""
    body = f"fix F fluid addforce/meso 0.0 0.0 {fz}" if fz else ""
    plain = deck(nf, nw, x, v, body=body)
    walled = deck(nf, nw, x, v, fix_line(rho0), body=body)
    x0, _, _, typ0 = plain.state()
    ref = oracle.rebuild(x0, typ0, (0, 0, 0), (L, L, L), 1.0, 0.3, 8.0)
    plain.run(1)
    walled.run(1)
    n = plain.natoms()
    tags = plain.field("tag")
    assert np.array_equal(tags, ref["tags"]) and np.array_equal(walled.field("tag"), tags)
    assert plain.thermo().nbuild == 1 and walled.thermo().nbuild == 1  # the setup build's rows
    assert np.array_equal(walled.field("x").view(np.uint64), plain.field("x").view(np.uint64))
    # the state before the fix (internal order), with the oracle's ghosts mapped onto the device's
    pos = plain.field("pos4")
    mask = plain.field("mask")
    src, img = plain.field("ghost_src"), plain.field("ghost_img")
    mask_all = np.concatenate([mask, mask[src]])
    ours = {(int(s), int(c)): n + g for g, (s, c) in enumerate(zip(src, img))}
    gmap = np.array([ours[(int(s), int(c))] for s, c in zip(ref["gsrc"], ref["gimg"])], np.int64)
    table = ref["table"].astype(np.int64)
    table = np.where(table >= n, gmap[np.clip(table - n, 0, None)], table).astype(np.int32)
    _, vt, _, _ = plain.state()
    v_pre = vt[tags - 1]
    f_pre = plain.field("force")[:, :3].astype(np.float64)  # the total force, body force included
    sigma = 1.0 / 4.0 / np.pi  # the default rc^2 / (4 pi)
    v_ref, f_ref = oracle.aboundary_meso(pos, mask_all, ref["count"], table, 2, 4, rho0, sigma, 0.01, v_pre, f_pre)
    _, vw, _, _ = walled.state()
    v_gpu = vw[tags - 1]
    f_gpu = walled.field("force")[:, :3].astype(np.float64)
    # reflected: v or f changed (a particle leaving the wall keeps its v, not its force into it)
    hit_ref = np.any(v_ref != v_pre, 1) | np.any(f_ref != f_pre, 1)
    hit_gpu = np.any(v_gpu != v_pre, 1) | np.any(f_gpu != f_pre, 1)
    assert np.sum(hit_ref != hit_gpu) <= 2, (hit_ref.sum(), hit_gpu.sum())
    both = hit_ref & hit_gpu
    vs = np.linalg.norm(v_pre[both], axis=1)[:, None] + 1
    fs = np.linalg.norm(f_pre[both], axis=1)[:, None] + 1
    assert np.all(np.abs(v_gpu[both] - v_ref[both]) <= 1e-4 * vs)
    assert np.all(np.abs(f_gpu[both] - f_ref[both]) <= 1e-4 * fs)
    rest = ~hit_ref & ~hit_gpu
    assert np.array_equal(v_gpu[rest], v_pre[rest])
    assert np.array_equal(f_gpu[rest], f_pre[rest])
    assert np.all((mask[hit_gpu] & 4) == 0)  # only the fix's group is touched
    return int(hit_ref.sum())


def test_aboundary_meso_one_step_matches_oracle():
    nf, nw, x, v = slab(fluid_bottom=1.0)
    assert one_step_parity(nf, nw, x, v) > 20  # the wall is reached


def test_aboundary_meso_after_a_run_with_rebuilds():
    # 200 steps with the fix, a body force into the wall and rebuilds whenever due; then the
    # one-step parity from the relaxed state (fluid layered against the wall surface). The
    # wall's own repulsion keeps the relaxed fluid ~0.5 off its surface, where the Gaussian wall
    # density is below 8/2; rho0 = 1 moves the fix's threshold out to ~0.4 from the surface.
    nf, nw, x, v = slab(seed=5)
    lam = deck(nf, nw, x, v, fix_line(1.0), delay=0, body="fix F fluid addforce/meso 0.0 0.0 -0.5")
    lam.run(200)
    t = lam.thermo()
    assert t.status == 0 and t.nbuild > 5 and np.isfinite(t.temp)
    x1, v1, _, _ = lam.state()
    assert one_step_parity(nf, nw, x1, v1, fz=-0.5, rho0=1.0) > 20
