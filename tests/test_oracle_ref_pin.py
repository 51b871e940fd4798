"""The oracle against the reference's own device kernels (no GPU here).

tests/golden/ref_<case>.npz hold what the reference's kernels produced on a B200 for four seeded
boxes (oracle/ref_harness.cu, compiled unmodified from the reference's sources; fixtures made by
tests/golden/make_ref_golden.py).  Each result of the oracle's restatement is compared with them:

  reorder keys, sort permutation, borderness, ghost images, full and reduced list rows,
  packed FP32 positions, TEA signatures                                        bit-exact
  rho (the reference computes it in FP32 with the hardware rsqrt; the oracle follows the
  FP32 steps with a correctly rounded 1/sqrtf)                  |d rho_i| <= 1e-6 * mean rho
  force, virial, e_pair from the reference's rho (FP64 pair arithmetic on FP32 inputs, both
  sides; the FP64 gaussian is bit-exact)                       |dF_i| <= 1e-12 * |F_i| + 1e-10
  wall volume fraction phi (mixed FP32/FP64 in the reference)               |d phi| <= 1e-5
  bounce-back: the same particles reflected, their x and v                     |d| <= 1e-5
"""
import json
import os
import sys

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLDEN)
import make_ref_golden as G  # noqa: E402

CASES = [c for c in G.CASES if os.path.exists(os.path.join(GOLDEN, f"ref_{c}.npz"))]


def coeffs_of(c):
    out = {}
    for (a, b), (A, B, g, rc, rd) in c["pair"].items():
        out[(a - 1, b - 1)] = out[(b - 1, a - 1)] = (rc, rd, A, B, g, np.sqrt(2.0 * c["kT"] * g))
    return out


class Run:
    """The oracle's rebuild of one case, with the arrays the comparisons need."""

    def __init__(self, name, skin=None):
        self.c = c = G.make_case(name)
        self.F = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
        self.meta = json.loads(str(self.F["meta"]))
        skin = c["skin"] if skin is None else skin
        self.r = r = oracle.rebuild(c["x"], c["type"], c["lo"], c["hi"], c["cutforce"], skin, c["rho_est"])
        self.n = n = c["n"]
        self.tags = t = r["tags"]
        self.order = np.argsort(t)                       # tag order -> internal index
        self.alltags = np.concatenate([t, t[r["gsrc"]]])
        self.src = np.concatenate([np.arange(n), r["gsrc"]])
        self.mask_all = c["mask"][t[self.src] - 1]

    def rows(self, count, table):
        flat = np.concatenate([table[i, :count[i]] for i in range(self.n)])
        return count[self.order], G.row_hash(count, self.alltags[flat])[self.order]

    def vel4(self):
        c = self.c
        v = np.zeros((len(self.alltags), 4), np.float32)
        v[:, :3] = c["v"][self.alltags - 1].astype(np.float32)
        v[:, 3] = oracle.sig_mdpd(self.alltags, oracle.seed_now(c["seed"], c["step"])).view(np.float32)
        return v


@pytest.fixture(scope="module", params=CASES)
def run(request):
    return Run(request.param)


def test_inputs_are_the_ones_the_reference_ran(run):
    assert run.meta["input_sha256"] == G.input_sha(run.c)


def test_sort_permutation_and_keys_bit_exact(run):
    F = run.F
    assert np.array_equal(run.tags, F["perm_tags"])
    assert run.r["n_bulk"] == run.meta["n_bulk"]
    assert np.array_equal(run.r["key"][F["perm_tags"] - 1] >> np.uint64(run.r["nbits"] - 1) & np.uint64(1),
                          (F["border"][F["perm_tags"] - 1] > 0).astype(np.uint64))
    if "key" in F:
        assert np.array_equal(run.r["key"].view(np.int64), F["key"])


def test_ghost_images_bit_exact(run):
    g = np.sort(run.tags[run.r["gsrc"]].astype(np.int64) * 27 + run.r["gimg"])
    assert np.array_equal(g, run.F["ghosts"])


def test_full_list_rows_bit_exact(run):
    cnt, h = run.rows(run.r["count"], run.r["table"])
    assert np.array_equal(cnt, run.F["full_count"])
    assert np.array_equal(h, run.F["full_hash"])


def test_reduced_rows_bit_exact(run):
    rd = max(v[4] for v in run.c["pair"].values())
    oc, ot = oracle.reduce_rows(run.r["count"], run.r["table"], run.r["pos4"], run.r["gimg"],
                                np.float32((rd + run.c["skin"] + 1e-3) ** 2))
    cnt, h = run.rows(oc, ot)
    assert np.array_equal(cnt, run.F["red_count"])
    assert np.array_equal(h, run.F["red_hash"])


def test_packed_positions_and_signatures_bit_exact(run):
    F = run.F
    if "pos_bits" not in F:
        pytest.skip("large case: packed bits not stored")
    assert np.array_equal(run.r["pos4"][:run.n].view(np.uint32)[run.order], F["pos_bits"])
    assert np.array_equal(run.vel4()[:run.n, 3].view(np.uint32)[run.order], F["sig"])


def test_density_matches_reference(run):
    c = run.c
    rho = oracle.density(run.r["pos4"], run.r["count"], run.r["table"], run.mask_all, c["rho_bit"], c["cut_rho"],
                         np.ones(8))
    ref = run.F["rho"]
    assert np.abs(rho[run.order] - ref).max() <= 1e-6 * ref.mean()


def test_force_virial_energy_match_reference(run):
    c, F = run.c, run.F
    rho_int = F["rho"][run.tags - 1]
    rho_all = rho_int[run.src]
    phi = None
    if c["arb_bc"]:
        mob = (c["mask"] & c["mobile_bit"]) != 0
        pt = np.zeros(run.n)
        pt[mob] = F["phi_mobile"]
        phi = np.zeros(len(run.alltags))
        phi[:run.n] = pt[run.tags - 1]
    f, vir, ep = oracle.force_mdpd(run.r["pos4"], run.vel4(), rho_all, run.r["count"], run.r["table"], coeffs_of(c),
                                   c["dt"], phi=phi, mask=run.mask_all,
                                   arb=(c["arb_bc"], c["mobile_bit"], c["wall_bit"]), ev=True)
    si = run.order[F["sample_tags"] - 1]
    fr = F["force"]
    err = np.abs(f[si] - fr).max(axis=1)
    assert np.all(err <= 1e-12 * np.linalg.norm(fr, axis=1) + 1e-10)
    sv = si[:len(F["e_pair"])]
    assert np.abs(vir[sv] - F["virial"]).max() <= 1e-12 * np.abs(F["virial"]).max()
    assert np.abs(ep[sv] - F["e_pair"]).max() <= 1e-12 * np.abs(F["e_pair"]).max()


def test_wall_fraction_and_bounce_back_match_reference():
    if "wall_8k" not in CASES:
        pytest.skip("no wall fixture")
    run = Run("wall_8k")
    c, F, r = run.c, run.F, run.r
    L = np.array(c["hi"]) - np.array(c["lo"])
    sh = np.stack([r["gimg"] % 3 - 1, (r["gimg"] // 3) % 3 - 1, r["gimg"] // 9 - 1], 1) * L
    xall = np.concatenate([r["x"], r["x"][r["gsrc"]] + sh])
    xin, vin = c["x"][run.tags - 1], c["v"][run.tags - 1]
    xo, vo, phi = oracle.aboundary(xin, vin, xall, run.mask_all, r["count"], r["table"], c["mobile_bit"],
                                   c["wall_bit"], c["cut_phi"], c["rho_wall"], c["phi_c"], c["dt"], np.ones(8),
                                   c["type"][run.tags - 1])
    mob = (c["mask"] & c["mobile_bit"]) != 0
    assert np.abs(phi[run.order][mob] - F["phi_mobile"]).max() <= 1e-5
    state = np.concatenate([xo, vo], 1)[run.order]
    moved = np.nonzero(np.any(state != np.concatenate([c["x"], c["v"]], 1), axis=1))[0] + 1
    assert len(F["bounce_tags"]) > 50
    assert np.array_equal(moved, F["bounce_tags"])
    assert np.abs(state[F["bounce_tags"] - 1] - F["bounce_state"]).max() <= 1e-5


def test_a_changed_skin_is_caught():
    # the pins discriminate: the list of a 0.31 skin is not the reference's 0.3 list
    run = Run("liquid_3k", skin=0.31)
    cnt, h = run.rows(run.r["count"], run.r["table"])
    assert not np.array_equal(h, run.F["full_hash"])
