"""mDPD liquid-vapour slab (the 60x30x30 slab geometry scaled down, and at full size): temperature, the liquid
density plateau and the surface tension gamma = (Lx/2)(Pxx - (Pyy+Pzz)/2), with the FP32
random-number transform (default) against the bit-exact FP64 transform (pair_modify rng exact).

Tolerances: T within 2% of kT in each mode for the small slab (it carries a ~1% bias at
dt = 0.01), within 1% at full size (108,900 particles, 18,000 sampled steps), and the two modes'
mean T within 0.5% or 3 combined standard errors of each other;
gamma > 0 and the two RNG modes agree within 2% of gamma or 3 combined standard errors (block
averages), whichever is larger; liquid plateau density within 2%.

A slab small enough for the FP64 oracle engine (6,050 particles) runs from the same start through
both: T within 1% of the oracle's, the liquid plateau density within 2%, the surface tension
within 2% of the oracle's or 3 combined standard errors, whichever is larger.
"""
import numpy as np
import pytest

import mdpd
import oracle

pytestmark = pytest.mark.gpu


def slab(rng_mode, seed):
    Lx, Ly, Lz, half = 30.0, 12.0, 12.0, 5.0
    n = int(round(2 * half * Ly * Lz * 6.05))
    lam = mdpd.Lammps()
    lam.commands(f"""
units lj
atom_style mdpd/atomic/meso 6.05
neighbor 0.3 bin
neigh_modify every 1 delay 0 check yes
region box block 0 {Lx} 0 {Ly} 0 {Lz} units box
create_box 1 box
region liq block {Lx / 2 - half} {Lx / 2 + half} 0 {Ly} 0 {Lz} units box
create_atoms 1 random {n} {seed} liq
mass 1 1.0
velocity all create 1.0 {seed + 1} dist gaussian
pair_style mdpd/meso 1.0 1.0 {seed + 2}
pair_coeff 1 1 -40 25 4.5 1.0 0.75
pair_modify rng {rng_mode}
fix BC all aboundary/rho/meso cut_rho 0.75
fix NVE all nve/meso
timestep 0.01
run_style mvv/meso
""")
    lam.run(3000)
    gam, tem, prof = [], [], []
    for _ in range(40):
        lam.run(100)
        t = lam.thermo()
        gam.append(t.surface_tension)
        tem.append(t.temp)
        x, _, _, _ = lam.state()
        xc = x[:, 0] - np.average(x[:, 0], weights=None)  # slab stays near the middle
        h, _ = np.histogram(np.mod(x[:, 0], Lx), bins=30, range=(0, Lx))
        prof.append(h / (Ly * Lz * 1.0))
    lam.close()
    return np.array(gam), np.array(tem), np.mean(prof, 0)


def block_se(a, nb=8):
    b = np.array([c.mean() for c in np.array_split(a, nb)])
    return b.std(ddof=1) / np.sqrt(nb)


def test_slab_surface_tension_and_temperature():
    gf, tf, pf = slab("fast", 1111)
    ge, te, pe = slab("exact", 1111)
    for t in (tf, te):
        assert abs(t.mean() - 1.0) < 0.02, (tf.mean(), te.mean())
    assert abs(tf.mean() - te.mean()) < max(0.005, 3 * np.hypot(block_se(tf), block_se(te))), (tf.mean(), te.mean())
    assert gf.mean() > 0 and ge.mean() > 0
    tol = max(0.02 * abs(ge.mean()), 3 * np.hypot(block_se(gf), block_se(ge)))
    assert abs(gf.mean() - ge.mean()) < tol, (gf.mean(), ge.mean(), tol)
    # liquid plateau: the densest third of the profile, same in both modes
    top_f = np.sort(pf)[-8:].mean(); top_e = np.sort(pe)[-8:].mean()
    assert abs(top_f - top_e) / top_e < 0.02, (top_f, top_e)
    assert 5.0 < top_f < 8.0


def slab_full_size(rng_mode, seed, steps=20000, discard=2000, every=100):
    """The 60x30x30 liquid-vapour slab at full size: box [-30,30]x[-15,15]x[-15,15], liquid |x| < 10 at
    density 6.05 (108,900 particles), A=-40, B=25, r_c=1, r_d=0.75, gamma=4.5, kT=1, dt=0.01."""
    lam = mdpd.Lammps()
    lam.commands(f"""
units lj
atom_style mdpd/atomic/meso 6.05
neighbor 0.3 bin
neigh_modify every 1 delay 0 check yes
region box block -30 30 -15 15 -15 15 units box
create_box 1 box
region liq block -10 10 -15 15 -15 15 units box
create_atoms 1 random 108900 {seed} liq
mass 1 1.0
velocity all create 1.0 {seed + 1} dist gaussian
pair_style mdpd/meso 1.0 1.0 {seed + 2}
pair_coeff 1 1 -40 25 4.5 1.0 0.75
pair_modify rng {rng_mode}
fix BC all aboundary/rho/meso cut_rho 0.75
fix NVE all nve/meso
timestep 0.01
run_style mvv/meso
""")
    lam.run(discard)
    gam, tem, prof = [], [], []
    for _ in range((steps - discard) // every):
        lam.run(every)
        t = lam.thermo()
        gam.append(t.surface_tension)
        tem.append(t.temp)
    x, _, _, _ = lam.state()
    h, _ = np.histogram(np.mod(x[:, 0] + 30.0, 60.0), bins=60, range=(0, 60))
    prof = h / (30.0 * 30.0)
    lam.close()
    return np.array(gam), np.array(tem), prof


def test_slab_60x30x30_full_size():
    # 20,000 steps, the first 2,000 discarded; block averages of 180 samples
    gf, tf, pf = slab_full_size("fast", 2024)
    ge, te, pe = slab_full_size("exact", 2024)
    for t in (tf, te):  # the spec's bar at full size (the small slab above carries a ~1% bias)
        assert abs(t.mean() - 1.0) < 0.01, (tf.mean(), te.mean())
    assert abs(tf.mean() - te.mean()) < max(0.005, 3 * np.hypot(block_se(tf), block_se(te))), (tf.mean(), te.mean())
    assert gf.mean() > 0 and ge.mean() > 0
    tol = max(0.02 * abs(ge.mean()), 3 * np.hypot(block_se(gf), block_se(ge)))
    assert abs(gf.mean() - ge.mean()) < tol, (gf.mean(), ge.mean(), tol)
    # liquid plateau (the 14 central 1-wide bins of the 20-wide slab), both modes, within 2%
    top_f = np.sort(pf)[-14:].mean(); top_e = np.sort(pe)[-14:].mean()
    assert abs(top_f - top_e) / top_e < 0.02, (top_f, top_e)
    assert 5.5 < top_f < 7.5


def test_small_slab_against_oracle_engine():
    # box [-12,12] x [-5,5]^2, liquid |x| < 5 at rho 6.05 (6,050 particles), A -40, B 25, r_d 0.75,
    # gamma 4.5, kT 1, dt 0.01; the same positions and velocities through the GPU path and the
    # FP64 oracle engine: 1,000 relaxation steps, then 4,000 steps sampled every 20
    rng = np.random.default_rng(77)
    lo, L = np.array([-12.0, -5.0, -5.0]), np.array([24.0, 10.0, 10.0])
    n = int(round(6.05 * 10.0 * 10.0 * 10.0))
    x = np.column_stack([rng.uniform(-5, 5, n), rng.uniform(-5, 5, n), rng.uniform(-5, 5, n)])
    v = rng.normal(0, 1, (n, 3)); v -= v.mean(0)
    b = mdpd.Batch([mdpd.box_spec(n, L, lo=lo, x=x, v=v, seed=31337)])
    b.setup()
    sim = oracle.Sim(x, v, tuple(lo), tuple(lo + L), seed=31337)
    sim.setup()
    b.step(1000); sim.run(1000)
    tg, to, gg, go = [], [], [], []
    hg, ho = np.zeros(24), np.zeros(24)
    for _ in range(200):
        b.step(20); sim.run(20)
        t = b.thermo(0); o = sim.thermo()
        tg.append(t.temp); to.append(o["temp"]); gg.append(t.surface_tension); go.append(o["surface_tension"])
        xg, _ = b.state(0); xo = sim.state()[0]
        hg += np.histogram(np.mod(xg[:, 0] + 12.0, 24.0), bins=24, range=(0, 24))[0]
        ho += np.histogram(np.mod(xo[:, 0] + 12.0, 24.0), bins=24, range=(0, 24))[0]
    sim.close()
    b.close()
    tg, to, gg, go = map(np.array, (tg, to, gg, go))
    assert abs(tg.mean() - to.mean()) < 0.01 * to.mean(), (tg.mean(), to.mean())
    # the slab drifts as a whole along x: the plateau is the densest 6 one-wide bins
    plat_g = np.sort(hg)[-6:].mean() / (200 * 100.0)
    plat_o = np.sort(ho)[-6:].mean() / (200 * 100.0)
    assert abs(plat_g - plat_o) < 0.02 * plat_o, (plat_g, plat_o)
    assert gg.mean() > 0 and go.mean() > 0
    tol = max(0.02 * abs(go.mean()), 3 * np.hypot(block_se(gg), block_se(go)))
    assert abs(gg.mean() - go.mean()) < tol, (gg.mean(), go.mean(), tol)
    print(f"\nsmall slab: T {tg.mean():.4f} vs oracle {to.mean():.4f}; plateau {plat_g:.3f} vs {plat_o:.3f}; "
          f"gamma {gg.mean():.3f} +- {block_se(gg):.3f} vs {go.mean():.3f} +- {block_se(go):.3f}")
