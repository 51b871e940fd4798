"""mdpd_kinetic_sums_noalloc: kinetic sums over caller-owned device arrays, allocating nothing.

Some callers cannot let the library allocate device memory: a host code that calls in from
inside its own timestep on arrays it already owns (a LAMMPS fix on its USER-MESO device
arrays, an application whose caching allocator or fixed arena holds the GPU), because
cudaMalloc/cudaFree synchronise the whole device and fail when the caller's pool holds the
memory. This entry point keeps its scratch in a fixed device array instead. Here its sums are
checked, through the C ABI, against the existing thermo entry point (mdpd_thermo) of the same
state, on two calls in a row of different sizes (the second call reuses the scratch the first
one filled). Tolerances: kinetic energy and temperatures 1e-12 relative, momentum 1e-12 of
sum |m v| (both sides are FP64 sums in a fixed order, only the grouping differs).

This file runs last (pytest collects files by name), so that a stop at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import mdpd

pytestmark = pytest.mark.gpu

MAX_N = 1 << 24


def two_type_box(n1, n2, L, seed):
    lam = mdpd.Lammps()
    lam.commands(f"""
units lj
atom_style mdpd/atomic/meso 6.05
neighbor 0.3 bin
region box block 0 {L} 0 {L} 0 {L} units box
create_box 2 box
create_atoms 1 random {n1} {seed} box
create_atoms 2 random {n2} {seed + 1} box
mass 1 1.0
mass 2 1.5
group fluid type 1
velocity all create 1.0 {seed + 2} dist gaussian
pair_style mdpd/meso 1.0 1.0 {seed + 3}
pair_coeff * * -40 25 4.5 1.0 0.75
fix BC all aboundary/rho/meso cut_rho 0.75
fix NVE fluid nve/meso
timestep 0.01
run_style mvv/meso
""")
    lam.run(20)
    return lam


def fn():
    f = mdpd.lib().mdpd_kinetic_sums_noalloc
    d = C.POINTER(C.c_double)
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int64,
                  C.c_void_p, d, C.c_char_p, C.c_int64]
    f.restype = C.c_int
    return f


def call(vx, vy, vz, mass, mask, groupbit, n):
    sums = np.zeros(11)
    err = C.create_string_buffer(256)
    rc = fn()(vx, vy, vz, mass, mask, groupbit, n, None, sums.ctypes.data_as(C.POINTER(C.c_double)), err, 256)
    return rc, sums, err.value.decode()


def device_sums(lam, groupbit):
    import torch
    n = lam.natoms()
    v = lam.field("v").reshape(n, 3)
    typ = lam.field("type")
    mask = lam.field("mask").astype(np.int32)
    mass = np.array([1.0, 1.5])[typ - 1]
    dev = [torch.tensor(np.ascontiguousarray(a), device="cuda:0") for a in (v[:, 0], v[:, 1], v[:, 2], mass, mask)]
    torch.cuda.synchronize()
    rc, sums, err = call(*[t.data_ptr() for t in dev], groupbit, n)
    assert rc == 0, err
    return sums, v, mass, mask


def check_against_thermo(lam):
    n = lam.natoms()
    t = lam.thermo()
    s_all, v, mass, mask = device_sums(lam, 1)          # group all
    s_fl, _, _, _ = device_sums(lam, 2)                 # group fluid (the nve group)
    assert s_all[10] == n
    assert abs(0.5 * s_all[0] - t.ke) <= 1e-12 * t.ke
    assert abs(s_all[0] / (3 * n - 3) - t.temp) <= 1e-12 * t.temp
    scale = np.sum(mass[:, None] * np.abs(v))
    assert np.all(np.abs(s_all[1:4] - np.array(t.momentum)) <= 1e-12 * scale)
    assert abs(s_all[4] + s_all[5] + s_all[6] - s_all[0]) <= 1e-12 * s_all[0]
    ng = int(np.count_nonzero(mask & 2))
    assert s_fl[10] == ng and 0 < ng < n
    assert abs(s_fl[0] / (3 * ng - 3) - t.temp_group) <= 1e-12 * t.temp_group


def test_noalloc_kinetic_sums_match_thermo_twice_in_a_row():
    big = two_type_box(9000, 3000, 12.6, 1234)
    small = two_type_box(1500, 500, 7.0, 4321)
    check_against_thermo(big)     # fills many scratch rows
    check_against_thermo(small)   # fewer rows: stale rows of the first call must not be read
    big.run(10)
    check_against_thermo(big)


def test_noalloc_rejects_oversize_and_host_arrays():
    import torch
    d = torch.zeros(4, dtype=torch.float64, device="cuda:0")
    p = d.data_ptr()
    rc, sums, err = call(p, p, p, p, None, 1, MAX_N + 1)
    assert rc == 7 and "exceeds" in err            # MDPD_ERR_ARG, nothing launched
    host = np.zeros(4)
    h = host.ctypes.data
    rc, sums, err = call(h, h, h, h, None, 1, 4)
    assert rc == 7 and "device memory" in err
    rc, sums, err = call(p, p, p, p, None, 1, 0)
    assert rc == 0 and not sums.any()
