"""ctypes front of the CPU oracle (liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU baseline legs as the oracle
and as the timed CPU restatement; never by the product library.  Each helper runs the
reference's algorithm for one hot-path function (see mdpd_oracle.h for file:line).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

u32p, i32p, dp, fp, u64p = (C.POINTER(C.c_uint32), C.POINTER(C.c_int32), C.POINTER(C.c_double),
                            C.POINTER(C.c_float), C.POINTER(C.c_uint64))


class Box(C.Structure):
    _fields_ = [("lo", C.c_double * 3), ("hi", C.c_double * 3), ("prd", C.c_double * 3), ("cen", C.c_double * 3),
                ("skin", C.c_double), ("cutneighmax", C.c_double), ("cutghost", C.c_double),
                ("binsize", C.c_double * 3), ("bininv", C.c_double * 3), ("mbin", C.c_int * 3),
                ("n_col", C.c_int), ("rc2_core", C.c_float), ("rc2_tail", C.c_float),
                ("expected_neigh_count", C.c_double)]


class MdpdCoeff(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("cut", "cut_r", "A", "B", "gamma", "sigma")]


class DpdCoeff(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("cut", "cutsq", "cutinv", "expw", "a0", "gamma", "sigma")]


class SimParams(C.Structure):
    _fields_ = [("style", C.c_int), ("ntype", C.c_int), ("lo", C.c_double * 3), ("hi", C.c_double * 3),
                ("skin", C.c_double), ("dt", C.c_double), ("kT", C.c_double), ("seed", C.c_uint32),
                ("rho_est", C.c_double), ("cut_rho", C.c_double), ("mass_type", C.c_double * 8),
                ("mcoeff", MdpdCoeff * 64), ("dcoeff", DpdCoeff * 64), ("nve_groupbit", C.c_int),
                ("rho_groupbit", C.c_int), ("body_force", C.c_double * 3), ("body_groupbit", C.c_int),
                ("arb_bc", C.c_int), ("mobile_bit", C.c_int), ("wall_bit", C.c_int), ("cut_phi", C.c_double),
                ("rho_wall", C.c_double), ("phi_c", C.c_double), ("nthreads", C.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.check_call(["make", "-C", HERE, "liboracle.so"], stdout=subprocess.DEVNULL)
        L = C.CDLL(LIB)
        L.orc_premix_tea.restype = C.c_uint32
        L.orc_premix_tea.argtypes = [C.c_uint32, C.c_uint32, C.c_int]
        L.orc_seed_now.restype = C.c_uint32
        L.orc_seed_now.argtypes = [C.c_uint32, C.c_int64]
        L.orc_brev.restype = C.c_uint32
        L.orc_brev.argtypes = [C.c_uint32]
        L.orc_gaussian_tea4.restype = C.c_double
        L.orc_gaussian_tea4.argtypes = [C.c_uint32, C.c_uint32]
        L.orc_rcp.restype = C.c_double
        L.orc_rcp.argtypes = [C.c_double]
        L.orc_morton3.restype = C.c_uint64
        L.orc_morton3.argtypes = [C.c_uint32] * 3
        L.orc_fma.restype = C.c_double
        L.orc_fma.argtypes = [C.c_double] * 3
        L.orc_dr2f.restype = C.c_float
        L.orc_dr2f.argtypes = [C.c_float] * 3
        L.orc_sim_create.restype = C.c_void_p
        L.orc_sim_create.argtypes = [C.POINTER(SimParams), C.c_int, dp, dp, i32p, i32p, i32p]
        L.orc_sim_destroy.argtypes = [C.c_void_p]
        L.orc_sim_setup.argtypes = [C.c_void_p]
        L.orc_sim_run.argtypes = [C.c_void_p, C.c_int64]
        L.orc_sim_get.argtypes = [C.c_void_p, dp, dp, dp, dp]
        L.orc_sim_thermo.argtypes = [C.c_void_p, dp]
        L.orc_sim_nbuild.restype = C.c_int64
        L.orc_sim_nbuild.argtypes = [C.c_void_p]
        _lib = L
    return _lib


def P(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def tea(v0, v1, rounds):
    return np.array([lib().orc_premix_tea(int(a), int(b), rounds) for a, b in zip(v0, v1)], np.uint32)


def gaussian(si, sj):
    si = np.ascontiguousarray(si, np.uint32); sj = np.ascontiguousarray(sj, np.uint32)
    out = np.zeros(len(si))
    lib().orc_gaussian_batch(len(si), P(si, C.c_uint32), P(sj, C.c_uint32), P(out, C.c_double))
    return out


def seed_now(seed, step):
    return lib().orc_seed_now(seed, step)


def sig_mdpd(tags, sn):
    tags = np.ascontiguousarray(tags, np.int32)
    out = np.zeros(len(tags), np.uint32)
    lib().orc_sig_mdpd(len(tags), P(tags, C.c_int32), C.c_uint32(sn), P(out, C.c_uint32))
    return out


def sig_dpd(tags, vel4, sn):
    tags = np.ascontiguousarray(tags, np.int32); vel4 = np.ascontiguousarray(vel4, np.float32)
    out = np.zeros(len(tags), np.uint32)
    lib().orc_sig_dpd(len(tags), P(tags, C.c_int32), P(vel4, C.c_float), C.c_uint32(sn), P(out, C.c_uint32))
    return out


def box(lo, hi, cutforce, skin, rho_est, n):
    b = Box()
    lo = (C.c_double * 3)(*lo); hi = (C.c_double * 3)(*hi)
    lib().orc_box_setup(C.byref(b), lo, hi, C.c_double(cutforce), C.c_double(skin), C.c_double(rho_est), n)
    return b


def rebuild(x, typ, lo, hi, cutforce, skin, rho_est):
    """Reference rebuild for locals given in tag order: pbc wrap, 2-level reorder sort,
    ghost images, FP32 pack, full list.  Returns a dict of arrays in the new order."""
    L = lib()
    n = len(x)
    b = box(lo, hi, cutforce, skin, rho_est, n)
    xs = np.ascontiguousarray(x[:, 0], np.float64).copy()
    ys = np.ascontiguousarray(x[:, 1], np.float64).copy()
    zs = np.ascontiguousarray(x[:, 2], np.float64).copy()
    L.orc_pbc(C.byref(b), n, P(xs, C.c_double), P(ys, C.c_double), P(zs, C.c_double))
    key = np.zeros(n, np.uint64)
    nbits = C.c_int()
    L.orc_reorder_keys(C.byref(b), n, P(xs, C.c_double), P(ys, C.c_double), P(zs, C.c_double),
                       P(key, C.c_uint64), C.byref(nbits))
    perm = np.zeros(n, np.int32)
    L.orc_stable_sort_u64(n, P(key, C.c_uint64), P(perm, C.c_int32))
    key_in = key.copy()  # reorder key of each particle, input (tag) order
    xs, ys, zs, key = xs[perm].copy(), ys[perm].copy(), zs[perm].copy(), key[perm]
    tags = (perm + 1).astype(np.int32)
    typ = np.ascontiguousarray(np.asarray(typ, np.int32)[perm])
    border = (key >> np.uint64(nbits.value - 1)) & np.uint64(1)
    nb = np.nonzero(border)[0]
    n_bulk = int(nb[0]) if len(nb) else n
    cap = 8 * n + 4096
    gsrc = np.zeros(cap, np.int32); gimg = np.zeros(cap, np.int32)
    ng = L.orc_ghosts(C.byref(b), n, n_bulk, P(xs, C.c_double), P(ys, C.c_double), P(zs, C.c_double), cap,
                      P(gsrc, C.c_int32), P(gimg, C.c_int32))
    assert ng >= 0
    gsrc, gimg = gsrc[:ng].copy(), gimg[:ng].copy()
    pos4 = np.zeros((n + ng, 4), np.float32)
    L.orc_pack_pos(C.byref(b), n, ng, P(xs, C.c_double), P(ys, C.c_double), P(zs, C.c_double),
                   P(typ, C.c_int32), P(gsrc, C.c_int32), P(gimg, C.c_int32), P(pos4, C.c_float))
    sx = (gimg % 3 - 1); sy = (gimg // 3) % 3 - 1; sz = gimg // 9 - 1
    xa = np.concatenate([xs, xs[gsrc] + sx * b.prd[0]])
    ya = np.concatenate([ys, ys[gsrc] + sy * b.prd[1]])
    za = np.concatenate([zs, zs[gsrc] + sz * b.prd[2]])
    cnt = np.zeros(n, np.int32); core = np.zeros(n, np.int32)
    table = np.zeros(n * b.n_col, np.int32)
    ovf = L.orc_build_list(C.byref(b), n, n + ng, P(xa, C.c_double), P(ya, C.c_double), P(za, C.c_double),
                           P(pos4, C.c_float), P(cnt, C.c_int32), P(core, C.c_int32), P(table, C.c_int32))
    table = table.reshape(n, b.n_col)
    return dict(box=b, perm=perm, tags=tags, key=key_in, x=np.stack([xs, ys, zs], 1), n_bulk=n_bulk, gsrc=gsrc,
                gimg=gimg,
                pos4=pos4, count=cnt, count_core=core, table=table, overflow=ovf, nbits=nbits.value)


def pairs_from_rows(count, table, tags_local, gsrc):
    """(tag_i, tag_j) of a row-major list over locals then ghosts."""
    n = len(count)
    ti, tj = [], []
    alltags = np.concatenate([tags_local, tags_local[gsrc]])
    for i in range(n):
        r = table[i, :count[i]]
        ti.append(np.full(count[i], tags_local[i], np.int32))
        tj.append(alltags[r])
    return np.concatenate(ti) if ti else np.zeros(0, np.int32), np.concatenate(tj) if tj else np.zeros(0, np.int32)


def reduce_rows(count, table, pos4, gimg, rn2):
    """Rows of a pair-once box: entries owned by the row's particle or within rn2 (FP32)."""
    n, ncol = table.shape
    count = np.ascontiguousarray(count, np.int32)
    table = np.ascontiguousarray(table, np.int32)
    pos4 = np.ascontiguousarray(pos4, np.float32)
    gimg = np.ascontiguousarray(gimg, np.int32) if len(gimg) else np.zeros(1, np.int32)
    oc = np.zeros(n, np.int32)
    ot = np.zeros((n, ncol), np.int32)
    lib().orc_reduce_rows(n, ncol, P(count, C.c_int32), P(table, C.c_int32), P(pos4, C.c_float),
                          P(gimg, C.c_int32), C.c_float(rn2), P(oc, C.c_int32), P(ot, C.c_int32))
    return oc, ot


def aboundary_meso(pos4, mask_all, count, table, mobile_bit, wall_bit, rho0, sigma, dt, v, f):
    """fix aboundary/meso at the end of a step over whole rows (count[i] entries): returns (v, f)
    after the wall reflection."""
    n, ncol = table.shape
    pos4 = np.ascontiguousarray(pos4, np.float32)
    mask_all = np.ascontiguousarray(mask_all, np.int32)
    cc = np.ascontiguousarray(count, np.int32)
    table = np.ascontiguousarray(table, np.int32)
    vv = [np.ascontiguousarray(v[:, d], np.float64).copy() for d in range(3)]
    ff = [np.ascontiguousarray(f[:, d], np.float64).copy() for d in range(3)]
    lib().orc_aboundary_meso(n, P(pos4, C.c_float), P(mask_all, C.c_int32), P(cc, C.c_int32), P(table, C.c_int32),
                             ncol, mobile_bit, wall_bit, C.c_double(rho0), C.c_double(sigma), C.c_double(dt),
                             *[P(a, C.c_double) for a in vv + ff])
    return np.stack(vv, 1), np.stack(ff, 1)


def density(pos4, count, table, mask, groupbit, cut_rho, mass_type):
    n = len(count)
    ncol = table.shape[1]
    pos4 = np.ascontiguousarray(pos4, np.float32); count = np.ascontiguousarray(count, np.int32)
    table = np.ascontiguousarray(table, np.int32); mask = np.ascontiguousarray(mask, np.int32)
    mt = np.ascontiguousarray(mass_type, np.float64)
    rho = np.zeros(n)
    lib().orc_density(n, P(pos4, C.c_float), P(count, C.c_int32), P(table, C.c_int32), ncol, P(mask, C.c_int32),
                      groupbit, C.c_double(cut_rho), P(mt, C.c_double), P(rho, C.c_double))
    return rho


def force_mdpd(pos4, vel4, rho, count, table, coeffs, dt, phi=None, mask=None, arb=(0, 0, 0), ev=False):
    """coeffs: dict (ti,tj) 0-based -> (cut, cut_r, A, B, gamma, sigma); rho/phi/mask over locals+ghosts."""
    n = len(count)
    ntype = max(max(k) for k in coeffs) + 1
    arr = (MdpdCoeff * 64)()
    for (a, b), c in coeffs.items():
        arr[a * ntype + b] = MdpdCoeff(*c)
    ncol = table.shape[1]
    na = len(pos4)
    pos4 = np.ascontiguousarray(pos4, np.float32); vel4 = np.ascontiguousarray(vel4, np.float32)
    rho = np.ascontiguousarray(rho, np.float64)
    phi = np.zeros(na) if phi is None else np.ascontiguousarray(phi, np.float64)
    mask = np.ones(na, np.int32) if mask is None else np.ascontiguousarray(mask, np.int32)
    count = np.ascontiguousarray(count, np.int32); table = np.ascontiguousarray(table, np.int32)
    f = np.zeros((n, 3)); vir = np.zeros((n, 6)) if ev else None; ep = np.zeros(n) if ev else None
    lib().orc_force_mdpd(n, P(pos4, C.c_float), P(vel4, C.c_float), P(rho, C.c_double), P(phi, C.c_double),
                         P(mask, C.c_int32), P(count, C.c_int32), P(table, C.c_int32), ncol, ntype, arr,
                         C.c_double(dt), arb[0], arb[1], arb[2], P(f, C.c_double),
                         P(vir, C.c_double) if ev else None, P(ep, C.c_double) if ev else None)
    return (f, vir, ep) if ev else f


def force_dpd(pos4, vel4, count, table, coeffs, dt, ev=False):
    """coeffs: dict (ti,tj) -> (cut, a0, gamma, sigma, expw)."""
    n = len(count)
    ntype = max(max(k) for k in coeffs) + 1
    arr = (DpdCoeff * 64)()
    for (a, b), (cut, a0, gam, sig, expw) in coeffs.items():
        arr[a * ntype + b] = DpdCoeff(cut, cut * cut, 1.0 / cut, expw, a0, gam, sig)
    ncol = table.shape[1]
    pos4 = np.ascontiguousarray(pos4, np.float32); vel4 = np.ascontiguousarray(vel4, np.float32)
    count = np.ascontiguousarray(count, np.int32); table = np.ascontiguousarray(table, np.int32)
    f = np.zeros((n, 3)); vir = np.zeros((n, 6)) if ev else None; ep = np.zeros(n) if ev else None
    lib().orc_force_dpd(n, P(pos4, C.c_float), P(vel4, C.c_float), P(count, C.c_int32), P(table, C.c_int32),
                        ncol, ntype, arr, C.c_double(dt), P(f, C.c_double),
                        P(vir, C.c_double) if ev else None, P(ep, C.c_double) if ev else None)
    return (f, vir, ep) if ev else f


def aboundary(x, v, xa, mask_all, count, table, mobile_bit, wall_bit, cut_phi, rho_wall, phi_c, dt,
              mass_type, types):
    """Wall volume fraction + bounce-back of mobile locals (gpu_aboundary); returns x, v, phi."""
    n = len(count)
    xs = [np.ascontiguousarray(x[:, d]).copy() for d in range(3)]
    vs = [np.ascontiguousarray(v[:, d]).copy() for d in range(3)]
    xas = [np.ascontiguousarray(xa[:, d], np.float64) for d in range(3)]
    mask_all = np.ascontiguousarray(mask_all, np.int32); count = np.ascontiguousarray(count, np.int32)
    table = np.ascontiguousarray(table, np.int32); types = np.ascontiguousarray(types, np.int32)
    mt = np.ascontiguousarray(mass_type, np.float64)
    phi = np.zeros(n)
    lib().orc_aboundary(n, *[P(a, C.c_double) for a in xs], *[P(a, C.c_double) for a in vs],
                        *[P(a, C.c_double) for a in xas], P(mask_all, C.c_int32), P(count, C.c_int32),
                        P(table, C.c_int32), table.shape[1], mobile_bit, wall_bit, C.c_double(cut_phi),
                        C.c_double(rho_wall), C.c_double(phi_c), C.c_double(0.5 * dt), C.c_double(dt),
                        P(mt, C.c_double), P(types, C.c_int32), P(phi, C.c_double))
    return np.stack(xs, 1), np.stack(vs, 1), phi


class Sim:
    """The oracle's full single-box engine (the CPU restatement timed as a baseline)."""

    def __init__(self, x, v, lo, hi, style=0, A=-40.0, B=25.0, gamma=4.5, kT=1.0, cut=1.0, cut_r=0.75,
                 cut_rho=0.75, sigma=3.0, a0=25.0, dt=0.01, skin=0.3, seed=1234, rho_est=6.05, nthreads=0,
                 types=None, mask=None, body=(0, 0, 0), body_bit=0):
        p = SimParams()
        p.style, p.ntype = style, 1
        p.lo[:] = list(lo); p.hi[:] = list(hi)
        p.skin, p.dt, p.kT, p.seed, p.rho_est, p.cut_rho = skin, dt, kT, seed, rho_est, cut_rho
        for t in range(8):
            p.mass_type[t] = 1.0
        p.mcoeff[0] = MdpdCoeff(cut, cut_r, A, B, gamma, np.sqrt(2 * kT * gamma))
        p.dcoeff[0] = DpdCoeff(cut, cut * cut, 1.0 / cut, 1.0, a0, gamma, sigma)
        p.nve_groupbit, p.rho_groupbit = 1, 1
        p.body_force[:] = list(body); p.body_groupbit = body_bit
        p.nthreads = nthreads
        n = len(x)
        x = np.ascontiguousarray(x, np.float64); v = np.ascontiguousarray(v, np.float64)
        tag = np.arange(1, n + 1, dtype=np.int32)
        typ = np.ones(n, np.int32) if types is None else np.ascontiguousarray(types, np.int32)
        msk = np.ones(n, np.int32) if mask is None else np.ascontiguousarray(mask, np.int32)
        self.n = n
        self.p = p
        self.h = lib().orc_sim_create(C.byref(p), n, P(x, C.c_double), P(v, C.c_double), P(tag, C.c_int32),
                                      P(typ, C.c_int32), P(msk, C.c_int32))

    def setup(self):
        return lib().orc_sim_setup(self.h)

    def run(self, n):
        return lib().orc_sim_run(self.h, int(n))

    def state(self):
        x = np.zeros((self.n, 3)); v = np.zeros((self.n, 3)); f = np.zeros((self.n, 3)); r = np.zeros(self.n)
        lib().orc_sim_get(self.h, P(x, C.c_double), P(v, C.c_double), P(f, C.c_double), P(r, C.c_double))
        return x, v, f, r

    def thermo(self):
        o = np.zeros(14)
        lib().orc_sim_thermo(self.h, P(o, C.c_double))
        vol = float(np.prod(np.array(self.p.hi[:]) - np.array(self.p.lo[:])))
        ptensor = o[8:14] / vol
        lx = self.p.hi[0] - self.p.lo[0]
        return dict(temp=o[0], virial=o[1], pe=o[2], momentum=o[3:6], nbuild=o[6], step=o[7], ptensor=ptensor,
                    surface_tension=0.5 * lx * (ptensor[0] - 0.5 * (ptensor[1] + ptensor[2])))

    def close(self):
        if self.h:
            lib().orc_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
