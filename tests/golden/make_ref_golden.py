"""Golden vectors from the reference's own device kernels (oracle/ref_harness.cu).

    python tests/golden/make_ref_golden.py cases            # write oracle/_ref/cases/<case>.bin
    oracle/_ref/ref_harness <case>.bin <case>.out          # on a machine with a GPU, per case
    python tests/golden/make_ref_golden.py collect <dir>   # <dir>/<case>.out -> ref_<case>.npz

The cases are seeded and regenerated bit for bit by make_case(), so the fixtures hold only what
the reference computed, keyed by particle tag:
  perm_tags     tags in the order of the reference's reorder sort (MesoAtom::sort_local)
  key           the reorder key of each tag (gpu_build_reorder_keypair<1>), small cases
  border        slabs holding each tag (MesoComm::borderness)
  ghosts        sorted source_tag * 27 + image code of the periodic ghost images
  full_count, full_hash   each tag's full-list row (gpu_build_neighbor_list<32,5> + join) as
                its length and an order-free hash of its neighbours' tags (row_hash below)
  red_count, red_hash     the same rows reduced as a pair-once mDPD box keeps them (the owned
                entries and those within r_d + skin + 1e-3; the library's own rule, applied
                to the reference's rows)
  pos_bits, sig small cases: the FP32 packed position and the TEA signature
                (gpu_merge_xvt_mdpd) of each tag
  rho           gpu_compute_rho of every tag
  sample_tags   tags whose force is stored (every tag of a case of up to 4096); the first 1024
                of them also keep virial and e_pair
  force, virial, e_pair  gpu_mdpd<1> at those tags
  sums          totals over all particles: rho, force (3), virial (6), e_pair
  phi, bounce_* wall cases: gpu_aboundary's wall fraction of every mobile tag, and position and
                velocity of the tags it reflected
Nothing here runs on a GPU; the harness does.
"""
import hashlib
import json
import os
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CASE_DIR = os.path.join(ROOT, "oracle", "_ref", "cases")
SMALL = 10000   # cases up to this size keep per-particle keys, packed positions and signatures
NSAMPLE = 4096  # tags whose forces are kept (every tag of a smaller case)
NVIRIAL = 1024  # of those, the tags whose virial and energy are kept

CASES = ("liquid_3k", "liquid_40k", "two_types_6k", "wall_8k")


def _maxwell(rng, n, kT=1.0):
    v = rng.normal(0.0, np.sqrt(kT), (n, 3))
    return v - v.mean(0)


def make_case(name):
    """The seeded input of one case: box, parameters and tag-ordered arrays (tags 1..n)."""
    base = dict(cutforce=1.0, skin=0.3, rho_est=6.05, dt=0.01, cut_phi=1.0, rho_wall=8.0, phi_c=0.5, arb_bc=0,
                rho_bit=1, mobile_bit=0, wall_bit=0, kT=1.0)
    if name == "liquid_3k":
        L, n = 8.0, 3098
        rng = np.random.default_rng(11)
        x = rng.uniform(0.0, L, (n, 3))
        c = dict(base, name=name, lo=(0.0,) * 3, hi=(L,) * 3, seed=4242, step=0, cut_rho=0.75, ntype=1,
                 pair={(1, 1): (-40.0, 25.0, 4.5, 1.0, 0.75)}, x=x, v=_maxwell(rng, n), type=np.ones(n, np.int32),
                 mask=np.ones(n, np.int32))
    elif name == "liquid_40k":
        n = 40000
        L = (n / 6.05) ** (1 / 3)
        rng = np.random.default_rng(12)
        x = rng.uniform(0.0, L, (n, 3))
        c = dict(base, name=name, lo=(0.0,) * 3, hi=(L,) * 3, seed=987654, step=1234, cut_rho=0.74, ntype=1,
                 pair={(1, 1): (-45.3, 27.1, 4.5, 1.0, 0.74)}, x=x, v=_maxwell(rng, n), type=np.ones(n, np.int32),
                 mask=np.ones(n, np.int32))
    elif name == "two_types_6k":
        L, n = 10.0, 6000
        rng = np.random.default_rng(13)
        x = rng.uniform(0.0, L, (n, 3))
        t = (rng.random(n) < 0.5).astype(np.int32) + 1
        c = dict(base, name=name, lo=(0.0,) * 3, hi=(L,) * 3, seed=31337, step=7, cut_rho=0.75, ntype=2,
                 pair={(1, 1): (-40.0, 25.0, 4.5, 1.0, 0.75), (1, 2): (-30.0, 25.0, 4.5, 1.0, 0.75),
                       (2, 2): (-50.0, 25.0, 4.5, 1.0, 0.75)},
                 x=x, v=_maxwell(rng, n), type=t, mask=np.ones(n, np.int32))
    elif name == "wall_8k":
        # frozen wall slab (type 2, rho 8) at z < 1.5 in a periodic 10^3 box, fluid (type 1,
        # rho 6.05) above it; 40 fluid particles start inside the wall's top half, so the
        # bounce-back has work.  Groups: all = 1, fluid (mobile) = 2, wall = 4.
        L = 10.0
        rng = np.random.default_rng(14)
        nw = int(round(8.0 * L * L * 1.5))
        nf = int(round(6.05 * L * L * 8.5))
        xw = np.column_stack([rng.uniform(0, L, nw), rng.uniform(0, L, nw), rng.uniform(0, 1.5, nw)])
        xf = np.column_stack([rng.uniform(0, L, nf), rng.uniform(0, L, nf), rng.uniform(1.5, L, nf)])
        xf[:40, 2] = rng.uniform(0.8, 1.5, 40)
        x = np.concatenate([xf, xw])
        n = len(x)
        t = np.concatenate([np.ones(nf, np.int32), np.full(nw, 2, np.int32)])
        v = _maxwell(rng, n)
        v[nf:] = 0.0
        mask = np.where(t == 1, 1 | 2, 1 | 4).astype(np.int32)
        c = dict(base, name=name, lo=(0.0,) * 3, hi=(L,) * 3, seed=2718, step=3, cut_rho=0.75, ntype=2,
                 pair={(1, 1): (-40.0, 25.0, 4.5, 1.0, 0.75), (1, 2): (-30.0, 25.0, 4.5, 1.0, 0.75),
                       (2, 2): (-40.0, 25.0, 4.5, 1.0, 0.75)},
                 x=x, v=v, type=t, mask=mask, arb_bc=1, mobile_bit=2, wall_bit=4)
    else:
        raise KeyError(name)
    c["n"] = len(c["x"])
    c["tag"] = np.arange(1, c["n"] + 1, dtype=np.int32)
    c["mass"] = [1.0] * 8
    return c


def coeff_table(c):
    """ntype*ntype*6 doubles {cut, cut_r, A, B, gamma, sigma} (MesoPairMDPD::prepare_coeff,
    pair_mdpd_meso.cu:70-91), sigma = sqrt(2 kT gamma) (pair_mdpd_meso.cu:387)."""
    nt = c["ntype"]
    tab = np.zeros((nt, nt, 6))
    for (a, b), (A, B, g, rc, rd) in c["pair"].items():
        row = (rc, rd, A, B, g, np.sqrt(2.0 * c["kT"] * g))
        tab[a - 1, b - 1] = row
        tab[b - 1, a - 1] = row
    return tab


def input_sha(c):
    h = hashlib.sha256()
    for k in ("x", "v", "type", "mask"):
        h.update(np.ascontiguousarray(c[k]).tobytes())
    return h.hexdigest()


def write_case(c, path):
    with open(path, "wb") as f:
        f.write(b"MDPDCASE")
        f.write(struct.pack("<4i", c["n"], c["ntype"], c["arb_bc"], 0))
        f.write(struct.pack("<6d", *c["lo"], *c["hi"]))
        f.write(struct.pack("<4d", c["cutforce"], c["skin"], c["rho_est"], c["dt"]))
        f.write(struct.pack("<4d", c["cut_rho"], c["cut_phi"], c["rho_wall"], c["phi_c"]))
        f.write(struct.pack("<Iiq", c["seed"], 0, c["step"]))
        f.write(struct.pack("<4i", c["rho_bit"], c["mobile_bit"], c["wall_bit"], 0))
        f.write(struct.pack("<8d", *c["mass"]))
        f.write(coeff_table(c).astype("<f8").tobytes())
        for d in range(3):
            f.write(np.ascontiguousarray(c["x"][:, d], "<f8").tobytes())
        for d in range(3):
            f.write(np.ascontiguousarray(c["v"][:, d], "<f8").tobytes())
        for k in ("tag", "type", "mask"):
            f.write(np.ascontiguousarray(c[k], "<i4").tobytes())


def read_out(path):
    """The harness's records: name[32], dtype[8], count (int64), data."""
    out = {}
    with open(path, "rb") as f:
        while True:
            h = f.read(48)
            if len(h) < 48:
                break
            name = h[:32].rstrip(b"\0").decode()
            dt = h[32:40].rstrip(b"\0").decode()
            (cnt,) = struct.unpack("<q", h[40:48])
            dtype = {"f8": "<f8", "f4": "<f4", "i4": "<i4", "u8": "<u8"}[dt]
            out[name] = np.frombuffer(f.read(cnt * np.dtype(dtype).itemsize), dtype).copy()
    return out


def fmix32(h):
    h = np.asarray(h, np.uint32).copy()
    h ^= h >> np.uint32(16)
    h *= np.uint32(0x85EBCA6B)
    h ^= h >> np.uint32(13)
    h *= np.uint32(0xC2B2AE35)
    h ^= h >> np.uint32(16)
    return h


def row_hash(count, tag_j):
    """Order-free hash of each row's neighbour tags: the sum (mod 2^32) of fmix32(tag) over the
    row's entries; rows given by their lengths and the entries' tags concatenated."""
    count = np.asarray(count, np.int64)
    mixed = fmix32(np.asarray(tag_j, np.uint32)).astype(np.uint64)
    ends = np.cumsum(count)
    cs = np.zeros(len(mixed) + 1, np.uint64)
    cs[1:] = np.cumsum(mixed, dtype=np.uint64)
    return ((cs[ends] - cs[ends - count]) & np.uint64(0xFFFFFFFF)).astype(np.uint32)


def reduce_rows_flat(count, rows, pos4, nlocal, gimg, rn2):
    """A pair-once mDPD box's rows from full rows (concatenated): entries owned by the row --
    a local j > i or a ghost image shifted in the positive direction (image code > 13) -- and
    those within rn2 (FP32 distance with the list test's contraction, evaluated by the oracle)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    n = len(count)
    ncol = int(count.max()) if n else 1
    table = np.zeros((n, max(ncol, 1)), np.int32)
    off = np.concatenate([[0], np.cumsum(count)])
    for i in range(n):
        table[i, :count[i]] = rows[off[i]:off[i + 1]]
    oc, ot = oracle.reduce_rows(count, table, pos4, gimg, np.float32(rn2))
    flat = np.concatenate([ot[i, :oc[i]] for i in range(n)]) if n else np.zeros(0, np.int32)
    return oc, flat


def collect(c, o):
    """Fixture arrays from one harness output, keyed by tag."""
    n = c["n"]
    perm = o["perm"]
    tags_sorted = c["tag"][perm]                  # internal (sorted) order -> tag
    order = np.argsort(tags_sorted)               # tag order -> internal index
    tag_all = o["tag_all"]
    assert np.array_equal(tag_all[:n], tags_sorted)
    cnt = o["list_count"]
    rows = o["list_rows"]
    gsrc, gimg = o["ghost_src"], o["ghost_img"]
    pos4 = o["coord_merged"].reshape(-1, 4)
    vel4 = o["veloc_merged"].reshape(-1, 4)
    full_hash = row_hash(cnt, tag_all[rows])
    rd = max(r for (_, _, _, _, r) in c["pair"].values())
    rn2 = np.float32((rd + c["skin"] + 1e-3) ** 2)
    rcnt, rrows = reduce_rows_flat(cnt, rows, pos4, n, gimg, rn2)
    red_hash = row_hash(rcnt, tag_all[rrows])
    geo = o["geometry_i"]
    fx = np.stack([o["force_x"], o["force_y"], o["force_z"]], 1)
    vir = np.stack([o[k] for k in ("virial_xx", "virial_yy", "virial_zz", "virial_xy", "virial_xz", "virial_yz")], 1)
    small = n <= SMALL
    if n <= NSAMPLE:
        sample = np.arange(1, n + 1, dtype=np.int32)
    else:
        sample = np.unique(np.random.default_rng(7).choice(np.arange(1, n + 1), NSAMPLE, replace=False)).astype(np.int32)
    si = order[sample - 1]
    sv = si[:NVIRIAL]
    meta = {k: (list(v) if isinstance(v, tuple) else v) for k, v in c.items()
            if k in ("name", "n", "lo", "hi", "seed", "step", "cut_rho", "ntype", "cutforce", "skin", "rho_est",
                     "dt", "arb_bc", "cut_phi", "rho_wall", "phi_c", "kT")}
    meta["pair"] = {f"{a} {b}": list(v) for (a, b), v in c["pair"].items()}
    meta["input_sha256"] = input_sha(c)
    meta["n_col"], meta["n_bulk"], meta["nghost"] = int(geo[3]), int(geo[4]), int(geo[5])
    meta["mbin"] = [int(g) for g in geo[:3]]
    fix = dict(
        meta=np.array(json.dumps(meta)),
        perm_tags=tags_sorted.astype(np.int32),
        border=o["border"].astype(np.int8),
        ghosts=np.sort(tag_all[gsrc].astype(np.int64) * 27 + gimg).astype(np.int32),
        full_count=cnt[order].astype(np.int16), full_hash=full_hash[order],
        red_count=rcnt[order].astype(np.int16), red_hash=red_hash[order],
        sample_tags=sample,
        rho=o["rho"][order], force=fx[si], virial=vir[sv], e_pair=o["e_pair"][sv],
        sums=np.concatenate([[o["rho"].sum()], fx.sum(0), vir.sum(0), [o["e_pair"].sum()]]),
    )
    if small:
        fix["key"] = o["reorder_key"].view(np.int64)
        fix["pos_bits"] = pos4[:n].view(np.uint32)[order]
        fix["sig"] = vel4[:n, 3].view(np.uint32)[order]
    if c["arb_bc"]:
        phi = o["phi"][order]
        mob = (c["mask"] & c["mobile_bit"]) != 0
        fix["phi_mobile"] = phi[mob]
        b = np.stack([o["bounce_" + k] for k in ("x", "y", "z", "vx", "vy", "vz")], 1)[order]
        xs = np.concatenate([c["x"], c["v"]], 1)
        moved = np.nonzero(np.any(b != xs, axis=1))[0]
        fix["bounce_tags"] = (moved + 1).astype(np.int32)
        fix["bounce_state"] = b[moved]
    return fix


def main(argv):
    if len(argv) < 2 or argv[1] not in ("cases", "collect"):
        print(__doc__)
        return 2
    if argv[1] == "cases":
        os.makedirs(CASE_DIR, exist_ok=True)
        for name in CASES:
            write_case(make_case(name), os.path.join(CASE_DIR, name + ".bin"))
            print("wrote", os.path.join(CASE_DIR, name + ".bin"))
        return 0
    src = argv[2]
    for name in CASES:
        p = os.path.join(src, name + ".out")
        if not os.path.exists(p):
            print("missing", p)
            continue
        c = make_case(name)
        fix = collect(c, read_out(p))
        dst = os.path.join(HERE, f"ref_{name}.npz")
        np.savez_compressed(dst, **fix)
        print("wrote", dst, os.path.getsize(dst), "bytes")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
