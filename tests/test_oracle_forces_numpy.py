"""The oracle's FP64 density and pair-force passes against independent numpy restatements of the
reference kernels, on a list the oracle built (its pair sets are checked in
test_oracle_rebuild_numpy).  These oracle functions are what the GPU force, density, virial and
energy tolerances are measured against.  No GPU.

- density: gpu_compute_rho (fix_aboundary_rho_meso.cu:119-165), factor 15/(2 pi r_d^5) (:90),
  the mass of i, not of j, on every term;
- mDPD: gpu_mdpd (pair_mdpd_meso.cu:139-225): F = [A w_c + B (rho_i + rho_j) w_d - gamma w_c^2
  (r.v)/r + sigma w_c xi/sqrt(dt)] r/r, energy 1/2 A r_c w_c^2 + 1/2 B r_d (rho_i + rho_j) w_d^2 and
  the virial, each halved per particle;
- classic DPD: gpu_dpd (pair_dpd_meso.cu:91-205) with w_r = w_c^expw.

xi is the pinned pairwise gaussian (test_oracle_pins).  The force passes form the coordinate and
velocity differences in FP32 and everything after in FP64, as the reference does, on both sides:
agreement to 1e-12 of the summed magnitudes.  The reference's density pass is FP32 throughout
with the hardware rsqrt; the oracle follows its FP32 steps and this numpy restatement stays FP64,
so the two agree to 2e-6 of rho (tests/test_oracle_ref_pin.py pins the oracle to the reference's
own output at 1e-6 of the mean density).
"""
import numpy as np

import oracle

L = 6.0


def setup(seed, ntype=2):
    rng = np.random.default_rng(seed)
    n = int(6.05 * L ** 3)
    typ = rng.integers(1, ntype + 1, n).astype(np.int32)
    ref = oracle.rebuild(rng.uniform(0, L, (n, 3)), typ, (0, 0, 0), (L, L, L), 1.0, 0.3, 6.05)
    src = np.concatenate([np.arange(n), ref["gsrc"]])
    sig = oracle.sig_mdpd(ref["tags"], oracle.seed_now(4242, 17))
    vel = rng.normal(0, 1, (n, 3)).astype(np.float32)
    vel4 = np.zeros((len(src), 4), np.float32)
    vel4[:, :3] = vel[src]
    vel4[:, 3] = sig[src].view(np.float32)
    rho = rng.uniform(4, 9, n)[src]
    I = np.repeat(np.arange(n), ref["count"])
    J = np.concatenate([ref["table"][i, :ref["count"][i]] for i in range(n)])
    return ref, n, src, vel4, rho, I, J


def pair_geometry(pos4, vel4, I, J):
    # r64 dx = coord1.x - coord2.x with FP32 members: the difference is rounded to FP32
    d = (pos4[I, :3] - pos4[J, :3]).astype(np.float64)
    dv = (vel4[I, :3] - vel4[J, :3]).astype(np.float64)
    rsq = np.einsum("ij,ij->i", d, d)
    dot = np.einsum("ij,ij->i", d, dv)
    return d, rsq, dot


def sum_rows(n, I, vals):
    out = np.zeros((n,) + vals.shape[1:])
    np.add.at(out, I, vals)
    return out


def test_density_matches_numpy():
    ref, n, src, vel4, _, I, J = setup(3)
    pos4 = ref["pos4"]
    ptype = pos4[:, 3].view(np.int32) & 0xFF
    mass_type = np.array([1.0, 2.5] + [1.0] * 6)
    h = 0.75
    mask = np.ones(len(pos4), np.int32)
    mask[::7] = 2  # not in the group: not written (stays 0 in the oracle's output)
    rho = oracle.density(pos4, ref["count"], ref["table"], mask, 1, h, mass_type)
    d, rsq, _ = pair_geometry(pos4, vel4, I, J)
    ok = (rsq < h * h) & (rsq >= 1e-20)
    w = np.where(ok, (h - np.sqrt(rsq)) ** 2, 0.0) * mass_type[ptype[I]] * 15.0 / (2 * np.pi * h ** 5)
    want = sum_rows(n, I, w)
    want[mask[:n] & 1 == 0] = 0.0
    assert np.all(np.abs(rho - want) <= 2e-6 * (np.abs(want) + 1))
    assert (want > 0).sum() > 0.8 * n


def test_mdpd_force_energy_virial_match_numpy():
    ref, n, src, vel4, rho, I, J = setup(5)
    pos4 = ref["pos4"]
    ptype = pos4[:, 3].view(np.int32) & 0xFF
    dt = 0.01
    # type pair -> (cut, cut_r, A, B, gamma, sigma), symmetric
    cf = {(0, 0): (1.0, 0.75, -40.0, 25.0, 4.5, 3.0), (1, 1): (1.0, 0.7, -30.0, 22.0, 6.0, 3.46),
          (0, 1): (0.9, 0.8, -50.0, 28.0, 5.0, 3.16)}
    cf[(1, 0)] = cf[(0, 1)]
    f, vir, ep = oracle.force_mdpd(pos4, vel4, rho, ref["count"], ref["table"], cf, dt, ev=True)
    tab = np.array([[cf[(a, b)] for b in range(2)] for a in range(2)])[ptype[I], ptype[J]]
    cut, cut_r, A, B, gam, sig = tab.T
    d, rsq, dot = pair_geometry(pos4, vel4, I, J)
    ok = (rsq < cut * cut) & (rsq >= 1e-20)
    r = np.sqrt(rsq)
    wc = 1 - r / cut
    wd = np.maximum(1 - r / cut_r, 0)
    xi = oracle.gaussian(vel4[I, 3].view(np.uint32), vel4[J, 3].view(np.uint32))
    rr = rho[I] + rho[J]
    fp = np.where(ok, (A * wc + B * rr * wd - gam * wc * wc * dot / r + sig * wc * xi / np.sqrt(dt)) / r, 0.0)
    Fij = d * fp[:, None]
    want = sum_rows(n, I, Fij)
    scale = sum_rows(n, I, np.abs(Fij)).sum(1) + 1e-30
    assert np.all(np.abs(f - want).max(1) <= 1e-12 * scale)
    en = np.where(ok, 0.5 * A * cut * wc ** 2 + 0.5 * B * cut_r * rr * wd ** 2, 0.0)
    assert np.allclose(ep, 0.5 * sum_rows(n, I, en), rtol=1e-12, atol=1e-12)
    comps = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    vw = np.stack([d[:, a] * d[:, b] * fp for a, b in comps], 1)
    assert np.allclose(vir, 0.5 * sum_rows(n, I, vw), rtol=1e-11, atol=1e-9)
    # the full list holds every pair from both ends with the same xi: total momentum change 0
    assert np.abs(f.sum(0)).max() <= 1e-10 * np.abs(f).sum()


def test_dpd_force_matches_numpy_with_power_weight():
    ref, n, src, vel4, _, I, J = setup(9, ntype=1)
    pos4 = ref["pos4"]
    dt = 0.02
    for expw in (1.0, 0.5):
        cut, a0, gam, sig = 1.0, 25.0, 4.5, 3.0
        f, vir, ep = oracle.force_dpd(pos4, vel4, ref["count"], ref["table"], {(0, 0): (cut, a0, gam, sig, expw)}, dt,
                                      ev=True)
        d, rsq, dot = pair_geometry(pos4, vel4, I, J)
        ok = (rsq < cut * cut) & (rsq >= 1e-20)
        r = np.sqrt(rsq)
        wc = 1 - r / cut
        wr = np.where(ok, np.abs(wc) ** expw, 0.0)
        xi = oracle.gaussian(vel4[I, 3].view(np.uint32), vel4[J, 3].view(np.uint32))
        fp = np.where(ok, (a0 * wc - gam * wr * wr * dot / r + sig * wr * xi / np.sqrt(dt)) / r, 0.0)
        Fij = d * fp[:, None]
        want = sum_rows(n, I, Fij)
        scale = sum_rows(n, I, np.abs(Fij)).sum(1) + 1e-30
        assert np.all(np.abs(f - want).max(1) <= 1e-12 * scale), expw
        assert np.allclose(ep, 0.5 * sum_rows(n, I, np.where(ok, 0.5 * a0 * cut * wc ** 2, 0.0)), rtol=1e-12, atol=1e-12)
