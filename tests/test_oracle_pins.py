"""Pins of the CPU oracle against the reference's own code and fixtures (no GPU)."""
import json
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def test_tea_words_match_reference_header():
    # premix_TEA<16/32/64> of src/USER-MESO/math_meso.h compiled unmodified on the host
    g = load("tea_words.json")
    v0 = np.array(g["v0"], np.uint32); v1 = np.array(g["v1"], np.uint32)
    for rounds in (16, 32, 64):
        got = oracle.tea(v0, v1, rounds)
        assert np.array_equal(got, np.array(g[f"tea{rounds}"], np.uint32)), rounds


def test_morton_matches_bitloop():
    L = oracle.lib()
    rng = np.random.default_rng(3)
    for _ in range(200):
        x, y, z = (int(a) for a in rng.integers(0, 1 << 21, 3))
        ref = 0
        for i in range(21):
            ref |= ((x >> i) & 1) << (3 * i) | ((y >> i) & 1) << (3 * i + 1) | ((z >> i) & 1) << (3 * i + 2)
        assert L.orc_morton3(x, y, z) == ref


def test_brev():
    L = oracle.lib()
    for x in (0, 1, 0x80000000, 0x12345678, 0xFFFFFFFF):
        assert L.orc_brev(x) == int(f"{x:032b}"[::-1], 2)


def test_gaussian_symmetric_bounded_and_normal():
    rng = np.random.default_rng(7)
    si = rng.integers(0, 2**32, 200000, dtype=np.uint64).astype(np.uint32)
    sj = rng.integers(0, 2**32, 200000, dtype=np.uint64).astype(np.uint32)
    g = oracle.gaussian(si, sj)
    assert np.array_equal(g, oracle.gaussian(sj, si))  # symmetric in (i, j): momentum conservation
    assert np.all(np.abs(g) <= 4.0)
    assert abs(g.mean()) < 0.01 and abs(g.std() - 1.0) < 0.01


def test_rcp_is_correctly_rounded_on_masses():
    L = oracle.lib()
    for m in (1.0, 2.0, 0.5, 3.0, 1.7):
        assert abs(L.orc_rcp(m) - 1.0 / m) <= 2.3e-16 / m


device = pytest.mark.skipif(not os.path.exists(os.path.join(GOLDEN, "ref_device.json")),
                            reason="ref_device.json is produced on a GPU by oracle/_ref/ref_pin device")


def _u64(hexes):
    return np.array([int(h, 16) for h in hexes], np.uint64)


@device
def test_gaussian_matches_reference_device_code():
    # gaussian_TEA<4> from the reference header, run on a B200: bit-exact FP64
    g = load("ref_device.json")
    u = np.array(g["u"], np.uint32); v = np.array(g["v"], np.uint32)
    ref = _u64(g["gauss"]).view(np.float64)
    got = oracle.gaussian(u, v)
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))


@device
def test_pair_distance_contraction_matches_nvcc():
    # dx*dx+dy*dy+dz*dz as nvcc emits it == fma(dz,dz, fma(dx,dx, dy*dy))
    g = load("ref_device.json")
    a = _u64(g["dr2_a"]).astype(np.uint32).view(np.float32).reshape(-1, 3)
    b = _u64(g["dr2_b"]).astype(np.uint32).view(np.float32).reshape(-1, 3)
    ref = _u64(g["dr2"]).astype(np.uint32).view(np.float32)
    L = oracle.lib()
    d = (a - b).astype(np.float32)
    got = np.array([L.orc_dr2f(*map(float, r)) for r in d], np.float32)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@device
def test_bin_and_subbin_contraction_matches_nvcc():
    g = load("ref_device.json")
    x = _u64(g["x"]).view(np.float64)
    lo, inv, bs, ci = (_u64([g[k]]).view(np.float64)[0] for k in ("lo", "inv", "bs", "ci"))
    bins = np.array(g["bin"], np.uint32)
    ref_bin = _u64(g["bin_expr"]).view(np.float64)
    ref_sub = _u64(g["sub_expr"]).view(np.float64)
    fma = oracle.lib().orc_fma
    got_bin = np.array([fma(xx - lo, inv, 1.0) for xx in x])
    got_sub = np.array([fma(-float(np.uint32(b - 1)), bs, xx) * ci for xx, b in zip(x, bins)])
    assert np.array_equal(got_bin, ref_bin)
    assert np.array_equal(got_sub, ref_sub)


def test_static_contact_fixture():
    p = load("static_contact_profiles.json")
    for a in ("-20", "-30", "-35"):
        gpu = np.array(p["gpu"][a]); cpu = np.array(p["cpu"][a])
        assert len(gpu) == 10 and len(cpu) == 10
        assert abs(gpu[:, 1].sum() - 4000) < 5  # 4,000 fluid particles in the deck
        # the reference's own GPU and CPU profiles agree to a few percent in the bulk bins
        assert np.all(np.abs(gpu[2:8, 1] - cpu[2:8, 1]) / cpu[2:8, 1] < 0.06)
