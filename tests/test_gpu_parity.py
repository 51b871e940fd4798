"""Parity of the CUDA path with the oracle on the same seeded inputs (needs a B200).

Tolerances (stated per result):
  sort permutation, ghost images, pair sets, packed FP32 positions, RNG words: bit-exact
  FP64 gaussian (parity mode): bit-exact;  FP32 gaussian: |err| <= 3e-6 (absolute)
  density rho (FP32 pass with the hardware rsqrt, as the reference, vs FP64 oracle): <= 5e-6 relative
  conservative forces at sigma = 0 (FP32 pass vs FP64 oracle), per particle:
  |dF_i| <= 1e-5 * max(|F_i|, F_rms), F_rms the RMS of |F_i| over the box (relative where the
  net force is not tiny; 1e-5 of the typical force where the pair forces nearly cancel); the
  per-particle |dF_i|/|F_i| percentiles are printed (pytest -s)
  full forces with the random term (exact RNG): same bound
  one velocity-Verlet step (FP64 x, v from the same FP32 forces): bit-exact
"""
import os

import numpy as np
import pytest

import mdpd
import oracle

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def mdpd_box(n=6000, L=10.0, seed=4321, vseed=4928, kT=1.0, gamma=4.5, A=-40.0, B=25.0, rho_est=6.05,
             exact=False, skin=0.3, extra=""):
    lam = mdpd.Lammps()
    lam.commands(f"""
units lj
dimension 3
boundary p p p
atom_style mdpd/atomic/meso {rho_est}
neighbor {skin} bin
neigh_modify every 1 delay 0 check yes
region box block 0 {L} 0 {L} 0 {L} units box
create_box 1 box
create_atoms 1 random {n} {seed} box
mass 1 1.0
velocity all create 1.0 {vseed} dist gaussian
pair_style mdpd/meso {kT} 1.0 123456
pair_coeff 1 1 {A} {B} {gamma} 1.0 0.75
pair_modify rng {'exact' if exact else 'fast'}
fix BC all aboundary/rho/meso cut_rho 0.75
fix NVE all nve/meso
timestep 0.01
run_style mvv/meso
{extra}
""")
    return lam


def dpd_box(n=3000, L=10.0, seed=777, vseed=999, exact=True):
    lam = mdpd.Lammps()
    lam.commands(f"""
units lj
atom_style dpd/atomic/meso
neighbor 0.3 bin
region box block 0 {L} 0 {L} 0 {L} units box
create_box 1 box
create_atoms 1 random {n} {seed} box
mass 1 1.0
velocity all create 1.0 {vseed}
pair_style dpd/meso 1.0 5678
pair_coeff 1 1 25.0 4.5 3.0 1.0
pair_modify rng {'exact' if exact else 'fast'}
fix NVE all nve/meso
timestep 0.01
run_style mvv/meso
""")
    return lam


def oracle_rebuild(lam, L=10.0, rho_est=6.05):
    x0, v0, tag0, typ0 = lam.state()  # tag order, before the device rebuild
    return oracle.rebuild(x0, typ0, (0, 0, 0), (L, L, L), 1.0, 0.3, rho_est), x0, v0


def test_sort_permutation_bit_exact():
    lam = mdpd_box()
    ref, _, _ = oracle_rebuild(lam)
    lam.setup()
    tags = lam.field("tag")
    assert np.array_equal(tags, ref["tags"])
    # wrapped FP64 positions in the new order are bit-identical
    assert np.array_equal(lam.field("x").view(np.uint64), ref["x"].view(np.uint64))


def test_ghost_images_and_packed_positions_bit_exact():
    lam = mdpd_box()
    ref, _, _ = oracle_rebuild(lam)
    lam.setup()
    g = lam.geometry()
    n = lam.natoms()
    assert g["nghost"] == len(ref["gsrc"])
    tags = lam.field("tag")
    gpu_set = set(zip(tags[lam.field("ghost_src")].tolist(), lam.field("ghost_img").tolist()))
    ref_set = set(zip(ref["tags"][ref["gsrc"]].tolist(), ref["gimg"].tolist()))
    assert gpu_set == ref_set
    pos = lam.field("pos4")
    assert np.array_equal(pos[:n, :3].view(np.uint32), ref["pos4"][:n, :3].view(np.uint32))
    # ghost packed coordinates, matched by (source tag, image)
    gk = {k: i for i, k in enumerate(zip(tags[lam.field("ghost_src")].tolist(), lam.field("ghost_img").tolist()))}
    rk = list(zip(ref["tags"][ref["gsrc"]].tolist(), ref["gimg"].tolist()))
    order = np.array([gk[k] for k in rk])
    assert np.array_equal(pos[n + order, :3].view(np.uint32), ref["pos4"][n:, :3].view(np.uint32))


# density cutoff + skin + 1e-3 (squared, FP32): the reduced rows of a pair-once mDPD box keep
# the pairs within it and the pairs their particle owns
RN2_LIST = np.float32((0.75 + 0.3 + 1e-3) ** 2)


@pytest.mark.parametrize("n,L", [(6000, 10.0), (20000, 15.0)])
def test_pair_sets_bit_exact(n, L):
    # the reference's full list (oracle), reduced by the rule of a pair-once box: the entries
    # owned by the row's particle (a local above it, an upper ghost image) and those within
    # RN2_LIST; the other pairs reach neither the density sum nor the force pass before the
    # next build (the full list itself is checked bit-exact on the DPD box below)
    lam = mdpd_box(n=n, L=L)
    ref, _, _ = oracle_rebuild(lam, L=L)
    lam.setup()
    ti, tj = lam.pairs()
    cnt, tab = oracle.reduce_rows(ref["count"], ref["table"], ref["pos4"], ref["gimg"], RN2_LIST)
    assert 0.7 * ref["count"].sum() < cnt.sum() < 0.85 * ref["count"].sum()
    ri, rj = oracle.pairs_from_rows(cnt, tab, ref["tags"], ref["gsrc"])
    a = np.sort(ti.astype(np.int64) * (1 << 32) + tj)
    b = np.sort(ri.astype(np.int64) * (1 << 32) + rj)
    assert len(a) == len(b)
    assert np.array_equal(a, b)
    assert len(np.unique(a)) == len(a)  # no duplicate images


def test_rng_signatures_and_gaussian_bit_exact():
    lam = mdpd_box()
    lam.setup()
    tags = lam.field("tag")
    vel = lam.field("vel4")
    sn = oracle.seed_now(123456, 0)
    n = lam.natoms()
    assert np.array_equal(vel[:n, 3].view(np.uint32), oracle.sig_mdpd(tags, sn))
    rng = np.random.default_rng(11)
    si = rng.integers(0, 2**32, 1 << 20, dtype=np.uint64).astype(np.uint32)
    sj = rng.integers(0, 2**32, 1 << 20, dtype=np.uint64).astype(np.uint32)
    si[:3] = [0, 0xFFFFFFFF, 1]; sj[:3] = [0, 0xFFFFFFFF, 0]
    e, f = mdpd.gaussian(si, sj)
    ref = oracle.gaussian(si, sj)
    assert np.array_equal(e.view(np.uint64), ref.view(np.uint64))
    assert np.max(np.abs(f.astype(np.float64) - ref)) <= 3e-6


def test_gaussian_matches_reference_golden_when_present():
    path = os.path.join(GOLDEN, "ref_device.json")
    if not os.path.exists(path):
        pytest.skip("no reference device vectors yet")
    import json
    g = json.load(open(path))
    u = np.array(g["u"], np.uint32); v = np.array(g["v"], np.uint32)
    ref = np.array([int(h, 16) for h in g["gauss"]], np.uint64)
    e, _ = mdpd.gaussian(u, v)
    assert np.array_equal(e.view(np.uint64), ref)


def gpu_rows(lam):
    cnt, rows = lam.list_rows()
    return cnt, np.where(rows < 0, 0, rows).astype(np.int32)


def test_density_matches_oracle():
    # over the reference's full rows (oracle), so that a neighbour missing from the device's
    # rows would show
    lam = mdpd_box()
    ref_rb, _, _ = oracle_rebuild(lam)
    lam.setup()
    n = lam.natoms()
    pos = lam.field("pos4")
    rho = lam.field("rho")
    ref = oracle.density(ref_rb["pos4"], ref_rb["count"], ref_rb["table"], np.ones(n, np.int32), 1, 0.75,
                         np.ones(8))
    assert np.max(np.abs(rho[:n] - ref) / ref) < 5e-6


def assert_force_bar(f, ref, label, mask=None):
    """|dF_i| <= 1e-5 * max(|F_i|, F_rms) for every particle; prints the relative-error percentiles"""
    if mask is not None:
        f, ref = f[mask], ref[mask]
    mag = np.linalg.norm(ref, axis=1)
    err = np.linalg.norm(f - ref, axis=1)
    frms = np.sqrt(np.mean(mag ** 2))
    rel = err / np.maximum(mag, 1e-30)
    print(f"\n{label}: |dF_i|/|F_i| median {np.median(rel):.2e} p99.9 {np.quantile(rel, 0.999):.2e} "
          f"max {rel.max():.2e}; max |dF_i|/F_rms {err.max() / frms:.2e}")
    assert np.all(err <= 1e-5 * np.maximum(mag, frms)), (err / np.maximum(mag, frms)).max()


@pytest.mark.parametrize("exact", [False, True])
def test_conservative_force_sigma0(exact):
    lam = mdpd_box(kT=0.0, gamma=0.0, exact=exact)
    lam.setup()
    n = lam.natoms()
    cnt, rows = gpu_rows(lam)
    pos, vel, rho = lam.field("pos4"), lam.field("vel4"), lam.field("rho").astype(np.float64)
    f = lam.field("force")[:, :3].astype(np.float64)
    coeffs = {(0, 0): (1.0, 0.75, -40.0, 25.0, 0.0, 0.0)}
    ref = oracle.force_mdpd(pos, vel, rho, cnt, rows, coeffs, 0.01)
    assert_force_bar(f[:n], ref, f"sigma=0 forces ({'exact' if exact else 'fast'} rng)")


def test_full_force_with_exact_rng():
    lam = mdpd_box(exact=True)
    lam.setup()
    n = lam.natoms()
    cnt, rows = gpu_rows(lam)
    pos, vel, rho = lam.field("pos4"), lam.field("vel4"), lam.field("rho").astype(np.float64)
    f = lam.field("force")[:, :3].astype(np.float64)
    sigma = np.sqrt(2 * 1.0 * 4.5)
    coeffs = {(0, 0): (1.0, 0.75, -40.0, 25.0, 4.5, sigma)}
    ref = oracle.force_mdpd(pos, vel, rho, cnt, rows, coeffs, 0.01)
    assert_force_bar(f[:n], ref, "full forces (exact rng)")


def test_velocity_verlet_step_bit_exact():
    # x1 = x0 + dt * (v0 + dtfm * f0) in FP64 with the reference's FMA order; a rebuild in
    # the step may reorder particles and wrap them by one period, so match by tag
    lam = mdpd_box()
    lam.setup()
    x0 = lam.field("x"); tags = lam.field("tag")
    f0 = lam.field("force")[:, :3].astype(np.float64)
    _, v0s, _, _ = lam.state()  # tag order
    v0 = v0s[tags - 1]
    lam.step(1)
    x1 = lam.field("x"); tags1 = lam.field("tag")
    x1 = x1[np.argsort(tags1)][tags - 1]  # back to the setup order
    fma = oracle.lib().orc_fma
    dtfm = 0.5 * 0.01 * oracle.lib().orc_rcp(1.0)
    L = 10.0
    for i in range(0, len(x0), 31):
        for d in range(3):
            e = fma(0.01, fma(dtfm, f0[i, d], v0[i, d]), x0[i, d])
            assert x1[i, d] in (e, e + L, e - L), (i, d, x1[i, d], e)


def test_dpd_pairs_signatures_and_forces():
    lam = dpd_box()
    x0, _, _, typ0 = lam.state()
    ref = oracle.rebuild(x0, typ0, (0, 0, 0), (10, 10, 10), 1.0, 0.3, 0.0)
    lam.setup()
    assert np.array_equal(lam.field("tag"), ref["tags"])
    ti, tj = lam.pairs()
    ri, rj = oracle.pairs_from_rows(ref["count"], ref["table"], ref["tags"], ref["gsrc"])
    assert np.array_equal(np.sort(ti.astype(np.int64) * (1 << 32) + tj), np.sort(ri.astype(np.int64) * (1 << 32) + rj))
    n = lam.natoms()
    vel = lam.field("vel4")
    sn = oracle.seed_now(5678, 0)
    assert np.array_equal(vel[:n, 3].view(np.uint32), oracle.sig_dpd(lam.field("tag"), vel[:n], sn))
    cnt, rows = gpu_rows(lam)
    pos = lam.field("pos4")
    f = lam.field("force")[:, :3].astype(np.float64)
    reff = oracle.force_dpd(pos, vel, cnt, rows, {(0, 0): (1.0, 25.0, 4.5, 3.0, 1.0)}, 0.01)
    assert_force_bar(f[:n], reff, "classic DPD forces")


def test_list_overflow_reported_not_crashed():
    # a density estimate far below the real density gives too short rows (n_col = 32):
    # the build stops inserting at the row end and the call returns MDPD_ERR_OVERFLOW
    lam = mdpd_box(rho_est=0.1)
    with pytest.raises(mdpd.MdpdError) as e:
        lam.setup()
    assert e.value.code == mdpd.ERR_OVERFLOW


def test_deterministic_replay():
    out = []
    for _ in range(2):
        lam = mdpd_box(n=4000)
        lam.setup()
        lam.step(50)
        x, v, _, _ = lam.state()
        out.append((x, v))
        lam.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_density_shapes_give_the_same_bits():
    # the density pass's neighbour gathers in flight (pair_modify gather 4 | 6 | 8, the shapes the
    # autotuner picks from) change only how many loads a lane has in flight: rho sums each row in
    # entry order, so rho, forces and 50 steps of trajectory are bitwise the same
    out = []
    for g in (4, 6, 8):
        lam = mdpd_box(n=4000, extra=f"pair_modify gather {g}")
        lam.setup()
        rho, f = lam.field("rho"), lam.field("force")
        lam.step(50)
        x, v, _, _ = lam.state()
        out.append((rho, f, x, v))
        lam.close()
    for o in out[1:]:
        for a, b in zip(out[0], o):
            assert np.array_equal(a, b)
    lam = mdpd.Lammps()
    with pytest.raises(mdpd.MdpdError):
        lam.command("pair_modify gather 5")
    lam.close()


def test_staged_and_table_force_entries_give_the_same_bits():
    # the pair-once force pass stages each warp's compact rows in shared memory (pair_modify stage
    # yes, the default) or reads each entry from the table in the pair loop (stage no, also the
    # path of a warp whose rows exceed the staging capacity): the same pairs in the same per-lane
    # order, so forces and 50 steps of trajectory are bitwise the same
    out = []
    for st in ("yes", "no"):
        lam = mdpd_box(n=4000, extra=f"pair_modify stage {st}")
        lam.setup()
        f = lam.field("force")
        lam.step(50)
        x, v, _, _ = lam.state()
        out.append((f, x, v))
        lam.close()
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
    lam = mdpd.Lammps()
    with pytest.raises(mdpd.MdpdError):
        lam.command("pair_modify stage maybe")
    lam.close()


def test_two_type_pair_once_force_and_density_match_oracle():
    # the pair-once passes with two atom types (coefficients looked up per type pair, masses per
    # type in the density): sigma = 0 forces and the density against the FP64 oracle
    lam = mdpd.Lammps()
    lam.commands("""
units lj
atom_style mdpd/atomic/meso 6.05
neighbor 0.3 bin
region box block 0 10 0 10 0 10 units box
create_box 2 box
create_atoms 1 random 4000 2468 box
create_atoms 2 random 2000 1357 box
mass 1 1.0
mass 2 1.5
velocity all create 1.0 97531 dist gaussian
pair_style mdpd/meso 0.0 1.0 123456
pair_coeff 1 1 -40 25 0.0 1.0 0.75
pair_coeff 1 2 -30 20 0.0 1.0 0.70
pair_coeff 2 2 -50 30 0.0 0.9 0.75
fix BC all aboundary/rho/meso cut_rho 0.75
fix NVE all nve/meso
timestep 0.01
run_style mvv/meso
""")
    lam.setup()
    n = lam.natoms()
    cnt, rows = gpu_rows(lam)
    pos, vel = lam.field("pos4"), lam.field("vel4")
    rho = lam.field("rho").astype(np.float64)
    mass = np.zeros(8); mass[0], mass[1] = 1.0, 1.5
    ref_rho = oracle.density(pos, cnt, rows, np.ones(n, np.int32), 1, 0.75, mass)
    assert np.max(np.abs(rho[:n] - ref_rho) / ref_rho) < 5e-6
    f = lam.field("force")[:, :3].astype(np.float64)
    coeffs = {(0, 0): (1.0, 0.75, -40.0, 25.0, 0.0, 0.0), (0, 1): (1.0, 0.70, -30.0, 20.0, 0.0, 0.0),
              (1, 0): (1.0, 0.70, -30.0, 20.0, 0.0, 0.0), (1, 1): (0.9, 0.75, -50.0, 30.0, 0.0, 0.0)}
    ref = oracle.force_mdpd(pos, vel, rho, cnt, rows, coeffs, 0.01)
    assert_force_bar(f[:n], ref, "two-type sigma=0 forces")


@pytest.mark.parametrize("A", [float("inf"), -1e12, -2e8])
def test_nonfinite_or_out_of_range_force_reported(A):
    # injected on the host through the coefficients: an infinite A gives non-finite forces;
    # A = -1e12 gives single pair terms beyond the fixed-point range; A = -2e8 gives pair terms
    # of ~1e8, each inside the int64 range of 2^-32 units but ~25 of them add past 2^31, where a
    # particle's sum would wrap -- the per-pair bound 2^31 / (n_col + 1) catches them.  All come
    # back as MDPD_ERR_NAN from the call and the context stays usable
    lam = mdpd_box(A=A)
    with pytest.raises(mdpd.MdpdError) as e:
        lam.setup()
    assert e.value.code == mdpd.ERR_NAN
    lam.close()
    ok = mdpd_box()
    ok.setup()
    ok.step(2)
    assert ok.thermo().status == 0


def test_virial_and_pair_energy_match_oracle():
    # thermo's virial tensor and pair energy (compute pressure/meso, pe/meso) after setup,
    # against the oracle's per-atom sums over full rows (each pair twice at half weight; the
    # pair-once pass adds each pair once at full weight); exact RNG, FP32 pair terms vs FP64
    lam = mdpd_box(exact=True)
    lam.setup()
    t = lam.thermo()
    cnt, rows = gpu_rows(lam)
    pos, vel, rho = lam.field("pos4"), lam.field("vel4"), lam.field("rho").astype(np.float64)
    sigma = np.sqrt(2 * 1.0 * 4.5)
    coeffs = {(0, 0): (1.0, 0.75, -40.0, 25.0, 4.5, sigma)}
    _, vir, ep = oracle.force_mdpd(pos, vel, rho, cnt, rows, coeffs, 0.01, ev=True)
    vsum, vabs = vir.sum(0), np.abs(vir).sum(0)
    assert np.all(np.abs(np.array(t.virial) - vsum) <= 1e-5 * vabs + 1e-6), (np.array(t.virial), vsum)
    assert abs(t.pe - ep.sum()) <= 1e-5 * np.abs(ep).sum(), (t.pe, ep.sum())
    # the scalar pressure from them (compute_pressure_meso.cu:121-150)
    n = lam.natoms()
    ke = t.ke
    p_ref = (2 * ke + vsum[:3].sum()) / 3.0 / 1000.0
    assert abs(t.press - p_ref) <= 1e-5 * (2 * ke + vabs[:3].sum()) / 3.0 / 1000.0 + 1e-9, (t.press, p_ref)


def test_body_force_adds_momentum_exactly():
    # fix addforce/meso fx fy fz on the nve group: the pair forces cancel exactly in the
    # fixed-point sums, so after t time units the mean velocity has grown by (fx, fy, fz) t / m
    # up to the FP32 rounding of each particle's f + b (forces ~1e2 after equilibration: a
    # random walk of ~1e-9 in the mean over 200 half-kicks)
    lam = mdpd_box(extra="fix F all addforce/meso 0.02 -0.01 0.005")
    lam.setup()
    lam.step(300)  # past the random start's large forces, where FP32 f + b loses digits of b
    _, v0, _, _ = lam.state()
    lam.step(100)
    _, v1, _, _ = lam.state()
    dv = v1.mean(0) - v0.mean(0)
    print("body force: mean dv - b t =", dv - np.array([0.02, -0.01, 0.005]))
    assert np.allclose(dv, np.array([0.02, -0.01, 0.005]) * 100 * 0.01, rtol=0, atol=2e-8), dv
