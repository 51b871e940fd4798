"""The oracle's rebuild (oracle.rebuild: pbc wrap, 2-level reorder sort, ghost images, FP32 pack,
full neighbour list) against independent numpy restatements, so the bit-exact GPU parity tests
that compare with it stand on a checked oracle.  No GPU.

1. Sort permutation: the reorder key of gpu_build_reorder_keypair<1> (atom_meso.cu:271-311)
   with MesoAtom::sort_local's widths (atom_meso.cu:346-387), border slabs of MesoComm::borderness
   (comm_meso.cu:195-261), the reference's clamp at [nmin, nmax) and bit-loop Morton code
   (math_meso.h:165-201), then a stable sort of the keys.  nvcc contracts (x - lo) * inv + 1 and
   x - (b - 1) * binsize into FMAs (pinned against nvcc's code by test_oracle_pins); numpy has no
   FP64 fma, so each is evaluated exactly with fractions and rounded once.
2. Pair set: every particle against every periodic image that MesoComm::borders creates
   (images within cutghost of a face, edges and corners included), positions packed to FP32 as
   dp2sp_merged does (atom_vec_mdpd_atomic_meso.cu:140-206), r^2 in FP32 in nvcc's contraction
   fma(dz, dz, fma(dx, dx, dy*dy)) compared with (r_c + skin)^2 (gpu_build_neighbor_list,
   neigh_build_meso.cu:17-127).  fmaf is emulated by an FP64 multiply-add rounded to FP32, which
   can differ from fmaf in a tie, so pairs within 1e-5 (relative) of the cutoff are left out.
"""
from fractions import Fraction

import numpy as np

import oracle


def fma64(a, b, c):
    """a*b + c rounded once to FP64 (exact rational arithmetic)"""
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def clamp(i, nmin, nmax):
    return max(nmin, min(i, nmax - 1))


def morton3(x, y, z):
    r = 0
    for i in range(21):
        r |= ((x >> i) & 1) << (3 * i) | ((y >> i) & 1) << (3 * i + 1) | ((z >> i) & 1) << (3 * i + 2)
    return r


def reorder_perm(x, b):
    """new -> old order of the locals after sort_local"""
    n = len(x)
    max_bin = max(b.mbin[0], b.mbin[1], b.mbin[2])
    l1_width = 3 * int(np.floor(np.log2(max_bin * 2.0)))
    l2_width = 12
    keys = []
    for i in range(n):
        bid, sub, border = [], [], False
        for d in range(3):
            c = float(x[i, d])
            bd = clamp(int(fma64(c - b.lo[d], b.bininv[d], 1.0)), 0, b.mbin[d])
            off = fma64(-float((bd - 1) & 0xFFFFFFFF), b.binsize[d], c)  # uint (bid - 1) widened
            sub.append(clamp(int(off * (16 * b.bininv[d])), 0, 16))
            bid.append(bd)
            border |= c <= b.lo[d] + b.cutghost or c >= b.hi[d] - b.cutghost
        k = morton3(*bid) << l2_width | morton3(*sub)
        if border:
            k |= 1 << (l1_width + l2_width)
        keys.append(k)
    return np.array(sorted(range(n), key=lambda i: (keys[i], i)), np.int32)


def wrap(x, lo, hi):
    """MesoDomain::pbc"""
    x = x.copy()
    prd = hi - lo
    for d in range(3):
        c = x[:, d]
        c[c < lo[d]] += prd[d]
        m = c >= hi[d]
        c[m] -= prd[d]
        c[m] = np.maximum(c[m], lo[d])
    return x


def f32(v):
    return np.asarray(v, np.float64).astype(np.float32)


def fmaf(a, b, c):
    return (np.asarray(a, np.float64) * np.asarray(b, np.float64) + np.asarray(c, np.float64)).astype(np.float32)


def test_reorder_permutation_matches_numpy_restatement():
    rng = np.random.default_rng(41)
    L = np.array([6.5, 5.2, 7.9])
    n = int(6.05 * L.prod())
    x = rng.uniform(-0.2, 1.0, (n, 3)) * L  # some particles outside: wrapped first
    x[:40] = L * np.round(rng.uniform(0, 1, (40, 3)) * 5) / 5  # some on bin and box faces
    ref = oracle.rebuild(x, np.ones(n, np.int32), (0, 0, 0), tuple(L), 1.0, 0.3, 6.05)
    xw = wrap(x, np.zeros(3), L)
    assert np.array_equal(ref["x"], xw[ref["perm"]])
    assert np.array_equal(ref["perm"], reorder_perm(xw, ref["box"]))
    # bulk particles first, then the border ones
    b = ref["box"]
    xs = ref["x"]
    border = np.any((xs <= np.array(b.lo[:]) + b.cutghost) | (xs >= np.array(b.hi[:]) - b.cutghost), axis=1)
    assert not border[:ref["n_bulk"]].any() and border[ref["n_bulk"]:].all()


def test_full_list_matches_brute_force_over_all_images():
    rng = np.random.default_rng(5)
    L = np.array([6.4, 6.1, 6.7])
    n = int(6.05 * L.prod())
    lo, hi = np.zeros(3), L
    ref = oracle.rebuild(rng.uniform(0, 1, (n, 3)) * L, np.ones(n, np.int32), (0, 0, 0), tuple(L), 1.0, 0.3, 6.05)
    b = ref["box"]
    xs, tags = ref["x"], ref["tags"]
    cen = np.array(b.cen[:])
    cg = b.cutghost
    rc2 = np.float32(b.rc2_tail)
    # every image the ghost exchange creates: shift s_d = +1 needs x_d <= lo + cg, -1 needs >= hi - cg
    shifts = np.array([(sx, sy, sz) for sz in (-1, 0, 1) for sy in (-1, 0, 1) for sx in (-1, 0, 1)])
    codes = (shifts[:, 0] + 1) + 3 * (shifts[:, 1] + 1) + 9 * (shifts[:, 2] + 1)
    ok = np.ones((len(shifts), n), bool)
    for d in range(3):
        ok &= np.where(shifts[:, d:d + 1] == 1, xs[None, :, d] <= lo[d] + cg, True)
        ok &= np.where(shifts[:, d:d + 1] == -1, xs[None, :, d] >= hi[d] - cg, True)
    img = f32((xs[None, :, :] + shifts[:, None, :] * L) - cen)  # (27, n, 3) packed FP32
    # ghost images the oracle made: the same set of (source, code)
    made = set(zip(ref["gsrc"].tolist(), ref["gimg"].tolist()))
    want = {(j, int(codes[s])) for s in range(27) for j in np.nonzero(ok[s])[0].tolist() if codes[s] != 13}
    assert made == want
    pos = ref["pos4"][:, :3]
    assert np.array_equal(pos[:n], img[13])
    # oracle rows as (i, source j, image code)
    code_of = np.concatenate([np.full(n, 13), ref["gimg"]])
    src_of = np.concatenate([np.arange(n), ref["gsrc"]])
    checked = 0
    for i in range(n):
        pi = pos[i]
        dx = (pi[0] - img[:, :, 0]).astype(np.float32)
        dy = (pi[1] - img[:, :, 1]).astype(np.float32)
        dz = (pi[2] - img[:, :, 2]).astype(np.float32)
        r2 = fmaf(dz, dz, fmaf(dx, dx, (dy * dy).astype(np.float32)))
        near = np.abs(r2.astype(np.float64) - rc2) <= 1e-5 * rc2
        hit = ok & (r2 <= rc2)
        hit[13, i] = False  # not the particle itself
        s_idx, j_idx = np.nonzero(hit & ~near)
        want_i = set(zip(j_idx.tolist(), codes[s_idx].tolist()))
        row = ref["table"][i, :ref["count"][i]]
        got = set(zip(src_of[row].tolist(), code_of[row].tolist()))
        s_n, j_n = np.nonzero(near & ok)
        skip = set(zip(j_n.tolist(), codes[s_n].tolist()))
        assert want_i == got - skip, (i, tags[i])
        checked += len(got)
    assert checked > 0.99 * n * 4 / 3 * np.pi * 1.3 ** 3 * 6.05 * 0.9
