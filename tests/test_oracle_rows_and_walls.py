"""The oracle's restatements of the pair-once rows (orc_reduce_rows) and of fix aboundary/meso
(orc_aboundary_meso) against independent numpy ones, so the GPU parity tests that lean on them
stand on a checked oracle. No GPU.

numpy has no fused multiply-add: fmaf(a, b, c) is emulated by rounding a*b + c, taken in FP64
(a*b of two FP32 values is exact there), to FP32. That double rounding can differ from fmaf in
a tie, so distances within 1e-5 (relative) of the cutoff are left out of the comparison. The
wall density uses numpy's FP32 exp against the C library's expf: reflected v and f agree to
1e-5 of their magnitudes, and the reflected set to particles whose density is not within 1e-5
of rho0/2.
"""
import numpy as np

import oracle

L = 6.0


def fmaf(a, b, c):
    return (np.asarray(a, np.float64) * np.asarray(b, np.float64) + np.asarray(c, np.float64)).astype(np.float32)


def dist2(dx, dy, dz):
    """fma(dz, dz, fma(dx, dx, dy*dy)) in FP32, as nvcc contracts the sum of squares"""
    return fmaf(dz, dz, fmaf(dx, dx, (np.float32(dy) * np.float32(dy)).astype(np.float32)))


def dot(a, b):
    """a.x*b.x + a.y*b.y + a.z*b.z in FP32, contracted in the form of dist2"""
    return fmaf(a[2], b[2], fmaf(a[0], b[0], (np.float32(a[1]) * np.float32(b[1])).astype(np.float32)))


def rebuild(x, typ):
    return oracle.rebuild(x, typ, (0, 0, 0), (L, L, L), 1.0, 0.3, 8.0)


def test_reduce_rows_keeps_owned_and_density_range_pairs():
    rng = np.random.default_rng(31)
    n = int(6.05 * L ** 3)
    ref = rebuild(rng.uniform(0, L, (n, 3)), np.ones(n, np.int32))
    rn2 = np.float32((0.75 + 0.3 + 1e-3) ** 2)
    cnt, tab = oracle.reduce_rows(ref["count"], ref["table"], ref["pos4"], ref["gimg"], rn2)
    pos = ref["pos4"]
    checked = 0
    for i in range(n):
        row = ref["table"][i, :ref["count"][i]]
        d = pos[i, :3] - pos[row, :3]
        r2 = dist2(d[:, 0], d[:, 1], d[:, 2])
        if np.any(np.abs(r2 - rn2) <= 1e-5 * rn2):
            continue  # a tie of the emulated fma could go either way
        owned = np.where(row < n, row > i, ref["gimg"][np.clip(row - n, 0, None)] > 13)
        want = row[owned | (r2 <= rn2)]
        assert cnt[i] == len(want) and np.array_equal(tab[i, :cnt[i]], want), i
        checked += 1
    assert checked > 0.99 * n
    # each pair within the density range is in both rows; each other pair in its owner's only
    assert 0.7 * ref["count"].sum() < cnt.sum() < 0.85 * ref["count"].sum()


def aboundary_numpy(pos, mask_all, count, table, mobile_bit, wall_bit, rho0, sigma, dt, v, f):
    """fix aboundary/meso (gpu_aboundary_v2, fix_aboundary_meso.cu:186-246) in FP32 numpy, over
    whole rows: the reference's dev_pair_count_core is core plus skin after the list join"""
    n = len(count)
    v, f = v.copy(), f.copy()
    sg, r0, dtf = np.float32(sigma), np.float32(rho0), np.float32(dt)
    nf = np.float32(1.0 / np.sqrt((2 * np.pi) ** 3 * sigma ** 3))
    hs = np.float32(0.5 * np.float64(dtf))
    ex = np.float32(np.float32(-0.5) / sg)
    density = np.zeros(n, np.float32)
    for i in range(n):
        if not mask_all[i] & mobile_bit:
            continue
        v0, f0 = v[i].astype(np.float32), f[i].astype(np.float32)
        c1 = fmaf(dtf, fmaf(hs, f0, v0), pos[i, :3])
        rho = np.float32(0)
        g = np.zeros(3, np.float32)
        for j in table[i, :count[i]]:
            if not mask_all[j] & wall_bit:
                continue
            d = (c1 - pos[j, :3]).astype(np.float32)
            w = np.float32(nf * np.exp(np.float32(ex * dist2(d[0], d[1], d[2]))))
            rho = np.float32(rho + w)
            g = fmaf(d, np.float32(w / sg), g)
        density[i] = rho
        if rho > np.float32(0.5) * r0:
            e = -(g * np.float32(1.0 / np.sqrt(np.float64(dist2(g[0], g[1], g[2])))))
            e = e.astype(np.float32)
            vd = np.float32(max(0.0, dot(v0, e)))
            fd = np.float32(max(0.0, dot(f0, e)))
            v[i] -= (np.float32(2.0) * vd * e).astype(np.float64)
            f[i] -= (np.float32(2.0) * fd * e).astype(np.float64)
    return v, f, density


def test_aboundary_meso_oracle_matches_numpy():
    rng = np.random.default_rng(8)
    nw, nf = int(8 * L * L * 1.5), int(6.05 * L * L * (L - 1.0))
    x = np.concatenate([rng.uniform((0, 0, 1.0), (L, L, L), (nf, 3)), rng.uniform((0, 0, 0), (L, L, 1.5), (nw, 3))])
    ref = rebuild(x, np.ones(nf + nw, np.int32))
    n = nf + nw
    mobile = np.isin(ref["tags"], np.arange(1, nf + 1))  # tags 1..nf are the fluid
    mask = np.where(mobile, 3, 5).astype(np.int32)
    mask_all = np.concatenate([mask, mask[ref["gsrc"]]])
    v = rng.normal(0, 1, (n, 3)) - np.array([0, 0, 1.5])
    f = rng.normal(0, 30, (n, 3))
    sigma = 1.0 / 4.0 / np.pi
    v_c, f_c = oracle.aboundary_meso(ref["pos4"], mask_all, ref["count"], ref["table"], 2, 4, 8.0, sigma, 0.01, v, f)
    v_n, f_n, rho = aboundary_numpy(ref["pos4"], mask_all, ref["count"], ref["table"], 2, 4, 8.0, sigma, 0.01, v, f)
    hit_c = np.any(v_c != v, 1) | np.any(f_c != f, 1)
    hit_n = np.any(v_n != v, 1) | np.any(f_n != f, 1)
    borderline = np.abs(rho - 4.0) <= 1e-5 * 4.0
    assert hit_c.sum() > 20
    assert np.array_equal(hit_c[~borderline], hit_n[~borderline])
    both = hit_c & hit_n
    vs = np.linalg.norm(v[both], axis=1)[:, None] + 1
    fs = np.linalg.norm(f[both], axis=1)[:, None] + 1
    assert np.all(np.abs(v_c[both] - v_n[both]) <= 1e-5 * vs)
    assert np.all(np.abs(f_c[both] - f_n[both]) <= 1e-5 * fs)
