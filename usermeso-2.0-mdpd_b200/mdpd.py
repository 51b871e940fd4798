"""ctypes bindings of libmdpd.so (include/mdpd.h) with the reference's call shapes.

The script surface mirrors LAMMPS' Python/library interface for this path:
``Lammps().command("pair_style mdpd/meso 1.0 1.0 123456")``, ``.file(path)``,
``.run(n)`` -- the same commands, arguments and errors as the USER-MESO styles.  Errors
raise :class:`MdpdError` carrying the MDPD_* status.  Nothing here computes: every call
goes to the CUDA library, and loading fails loudly when the library is missing.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("MDPD_LIB", os.path.join(HERE, "libmdpd.so"))

OK, ERR_PARSE, ERR_OOM, ERR_OVERFLOW, ERR_NAN, ERR_TIMEOUT, ERR_CUDA, ERR_ARG, ERR_STATE, ERR_BUDGET = range(10)


class MdpdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Opts(C.Structure):
    _fields_ = [("device", C.c_int), ("verbose", C.c_int)]


class Thermo(C.Structure):
    _fields_ = [("step", C.c_int64), ("natoms", C.c_int64), ("nbuild", C.c_int64),
                ("temp", C.c_double), ("press", C.c_double), ("pe", C.c_double), ("ke", C.c_double),
                ("virial", C.c_double * 6), ("momentum", C.c_double * 3), ("temp_group", C.c_double),
                ("ptensor", C.c_double * 6), ("surface_tension", C.c_double),
                ("status", C.c_int32), ("pad", C.c_int32)]


class BoxSpec(C.Structure):
    _fields_ = [("style", C.c_int32), ("n", C.c_int32), ("lo", C.c_double * 3), ("hi", C.c_double * 3),
                ("A", C.c_double), ("B", C.c_double), ("gamma", C.c_double), ("kT", C.c_double),
                ("cut", C.c_double), ("cut_r", C.c_double), ("cut_rho", C.c_double), ("sigma", C.c_double),
                ("dt", C.c_double), ("skin", C.c_double), ("rho_est", C.c_double), ("mass", C.c_double),
                ("seed", C.c_uint32), ("every", C.c_int32), ("delay", C.c_int32), ("check", C.c_int32),
                ("exact_rng", C.c_int32),
                ("x", C.POINTER(C.c_double)), ("v", C.POINTER(C.c_double)), ("init_seed", C.c_uint64),
                ("fill_lo", C.c_double * 3), ("fill_hi", C.c_double * 3), ("start_step", C.c_int64)]


class JobSpec(C.Structure):
    _fields_ = [("box", BoxSpec), ("nsteps", C.c_int64), ("keep_state", C.c_int32), ("pad", C.c_int32)]


class JobResult(C.Structure):
    _fields_ = [("state", C.c_int32), ("error", C.c_int32), ("steps_done", C.c_int64),
                ("submit_s", C.c_double), ("start_s", C.c_double), ("end_s", C.c_double),
                ("step_ms_p50", C.c_double), ("step_ms_p99", C.c_double), ("thermo", Thermo)]


_lib = None


def lib():
    """Load libmdpd.so once; raise if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libmdpd.so not built at {LIB_PATH}; run usermeso-2.0-mdpd_b200/build.py")
        L = C.CDLL(LIB_PATH)
        vp, i64, i32, cp = C.c_void_p, C.c_int64, C.c_int32, C.c_char_p
        dp, fp, u32p, i32p = (C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_uint32),
                              C.POINTER(C.c_int32))
        sig = {
            "mdpd_create": ([C.POINTER(vp), C.POINTER(Opts)], C.c_int),
            "mdpd_command": ([vp, cp], C.c_int), "mdpd_file": ([vp, cp], C.c_int),
            "mdpd_run": ([vp, i64], C.c_int), "mdpd_setup": ([vp], C.c_int), "mdpd_step": ([vp, i64], C.c_int),
            "mdpd_natoms": ([vp, C.POINTER(i64)], C.c_int),
            "mdpd_get_state": ([vp, dp, dp, i32p, i32p, i64], C.c_int),
            "mdpd_set_state": ([vp, dp, dp, i64], C.c_int),
            "mdpd_thermo": ([vp, C.POINTER(Thermo)], C.c_int),
            "mdpd_log": ([vp], cp), "mdpd_last_error": ([vp], cp), "mdpd_destroy": ([vp], None),
            "mdpd_field_size": ([vp, cp, C.POINTER(i64)], C.c_int),
            "mdpd_get_field": ([vp, cp, vp, i64], C.c_int),
            "mdpd_geometry": ([vp, dp], C.c_int),
            "mdpd_get_pairs": ([vp, i32p, i32p, i64, C.POINTER(i64)], C.c_int),
            "mdpd_gaussian": ([u32p, u32p, dp, fp, i64], C.c_int),
            "mdpd_index_checks": ([], C.c_int),
            "mdpd_jobs_validate": ([cp, i32p, C.POINTER(C.c_uint64)], C.c_int),
            "mdpd_run_jobs": ([cp, cp, C.POINTER(Opts)], C.c_int),
            "mdpd_batch_create": ([C.POINTER(vp), C.POINTER(BoxSpec), i32, C.POINTER(Opts)], C.c_int),
            "mdpd_batch_setup": ([vp], C.c_int), "mdpd_batch_step": ([vp, i64], C.c_int),
            "mdpd_batch_thermo": ([vp, i32, C.POINTER(Thermo)], C.c_int),
            "mdpd_batch_get_state": ([vp, i32, dp, dp, i64], C.c_int),
            "mdpd_batch_get_states": ([vp, C.POINTER(dp), C.POINTER(dp), i32], C.c_int),
            "mdpd_batch_tune": ([vp, i32p, i32p], C.c_int),
            "mdpd_batch_tune_cached": ([vp, cp, i32p, i32p, i32p], C.c_int),
            "mdpd_batch_set_shapes": ([vp, i32, i32], C.c_int),
            "mdpd_batch_time": ([vp, i64, dp], C.c_int),
            "mdpd_batch_profile": ([vp, i64, dp], C.c_int),
            "mdpd_batch_rebuild_steps": ([vp, C.POINTER(i64)], C.c_int),
            "mdpd_batch_last_error": ([vp], cp), "mdpd_batch_destroy": ([vp], None),
            "mdpd_box_bytes": ([C.POINTER(BoxSpec), C.POINTER(C.c_uint64)], C.c_int),
            "mdpd_server_start": ([C.POINTER(vp), C.c_uint64, C.POINTER(Opts)], C.c_int),
            "mdpd_server_submit": ([vp, C.POINTER(JobSpec), C.POINTER(i64)], C.c_int),
            "mdpd_server_poll": ([vp, i64, C.POINTER(JobResult)], C.c_int),
            "mdpd_server_get_state": ([vp, i64, dp, dp, i64], C.c_int),
            "mdpd_server_cancel": ([vp, i64], C.c_int),
            "mdpd_server_drain": ([vp, C.c_double], C.c_int),
            "mdpd_server_stats": ([vp, dp], C.c_int),
            "mdpd_batch_run_thermo": ([vp, i64, C.POINTER(Thermo), C.POINTER(i64)], C.c_int),
            "mdpd_server_set_step_particles": ([vp, C.c_int64], C.c_int),
            "mdpd_server_timing": ([vp, dp], C.c_int),
            "mdpd_server_stop": ([vp], None),
            "mdpd_place": ([C.POINTER(BoxSpec), C.POINTER(C.c_int64), i32, i32, C.POINTER(C.c_uint64), i32p, dp],
                           C.c_int),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t)) if a is not None else None


class Lammps:
    """One box driven by LAMMPS script commands (the reference's input surface)."""

    def __init__(self, device=0, verbose=0):
        L = lib()
        h = C.c_void_p()
        rc = L.mdpd_create(C.byref(h), C.byref(Opts(device, verbose)))
        if rc:
            raise MdpdError(rc, L.mdpd_last_error(None).decode())
        self.h = h

    def _check(self, rc):
        if rc:
            raise MdpdError(rc, lib().mdpd_last_error(self.h).decode())

    def command(self, line):
        self._check(lib().mdpd_command(self.h, line.encode()))

    def commands(self, text):
        for line in text.splitlines():
            self.command(line)

    def file(self, path):
        self._check(lib().mdpd_file(self.h, path.encode()))

    def run(self, n):
        self._check(lib().mdpd_run(self.h, int(n)))

    def setup(self):
        self._check(lib().mdpd_setup(self.h))

    def step(self, n):
        self._check(lib().mdpd_step(self.h, int(n)))

    def natoms(self):
        n = C.c_int64()
        self._check(lib().mdpd_natoms(self.h, C.byref(n)))
        return n.value

    def state(self):
        n = self.natoms()
        x = np.zeros((n, 3)); v = np.zeros((n, 3))
        tag = np.zeros(n, np.int32); typ = np.zeros(n, np.int32)
        self._check(lib().mdpd_get_state(self.h, _ptr(x, C.c_double), _ptr(v, C.c_double),
                                         _ptr(tag, C.c_int32), _ptr(typ, C.c_int32), n))
        return x, v, tag, typ

    def set_state(self, x, v):
        x = np.ascontiguousarray(x, np.float64); v = np.ascontiguousarray(v, np.float64)
        self._check(lib().mdpd_set_state(self.h, _ptr(x, C.c_double), _ptr(v, C.c_double), len(x)))

    def thermo(self):
        t = Thermo()
        self._check(lib().mdpd_thermo(self.h, C.byref(t)))
        return t

    @property
    def log(self):
        return lib().mdpd_log(self.h).decode()

    def field(self, name):
        n = C.c_int64()
        self._check(lib().mdpd_field_size(self.h, name.encode(), C.byref(n)))
        dt = {"pos4": np.float32, "vel4": np.float32, "rho": np.float32, "force": np.float32, "phi": np.float32,
              "x": np.float64, "v": np.float64}.get(name, np.int32)
        out = np.zeros(max(n.value, 1), dt)
        self._check(lib().mdpd_get_field(self.h, name.encode(), out.ctypes.data_as(C.c_void_p), out.nbytes))
        out = out[:n.value]
        if name in ("pos4", "vel4", "force"):
            out = out.reshape(-1, 4)
        if name in ("x", "v"):
            out = out.reshape(-1, 3)
        return out

    def geometry(self):
        g = np.zeros(15)
        self._check(lib().mdpd_geometry(self.h, _ptr(g, C.c_double)))
        return {"lo": g[0:3], "hi": g[3:6], "cen": g[6:9], "mbin": g[9:12].astype(int),
                "cutghost": g[12], "n_col": int(g[13]), "nghost": int(g[14])}

    def pairs(self):
        n = C.c_int64()
        self._check(lib().mdpd_get_pairs(self.h, None, None, 0, C.byref(n)))
        ti = np.zeros(n.value, np.int32); tj = np.zeros(n.value, np.int32)
        self._check(lib().mdpd_get_pairs(self.h, _ptr(ti, C.c_int32), _ptr(tj, C.c_int32), n.value, C.byref(n)))
        return ti, tj

    def list_rows(self):
        """Neighbour list as row-major (n, n_col) of internal indices, from the transposed table."""
        cnt = self.field("count")
        tab = self.field("list")
        ncol = self.geometry()["n_col"]
        n = len(cnt)
        i = np.arange(n)[:, None]
        k = np.arange(ncol)[None, :]
        addr = (i & ~31) * ncol + 32 * k + (i & 31)
        rows = tab[addr]
        rows[k >= cnt[:, None]] = -1
        return cnt, rows

    def close(self):
        if getattr(self, "h", None):
            lib().mdpd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def validate_jobs(path):
    """check a JSON job spec without touching the device: (number of jobs, summed device bytes)"""
    n, b = C.c_int32(), C.c_uint64()
    rc = lib().mdpd_jobs_validate(os.fsencode(path), C.byref(n), C.byref(b))
    if rc:
        raise MdpdError(rc, lib().mdpd_last_error(None).decode())
    return n.value, b.value


def run_jobs(path, out_path, device=0):
    """run a JSON job spec on the serving loop; the result lines (one dict per job, then the
    summary) are written to out_path and returned.  A job that did not finish raises MdpdError
    after the lines are written."""
    import json
    o = Opts(device, 0)
    rc = lib().mdpd_run_jobs(os.fsencode(path), os.fsencode(out_path), C.byref(o))
    if rc and not os.path.exists(out_path):
        raise MdpdError(rc, lib().mdpd_last_error(None).decode())
    with open(out_path) as f:
        lines = [json.loads(t) for t in f if t.strip()]
    if rc:
        raise MdpdError(rc, lib().mdpd_last_error(None).decode() + "\n" + "\n".join(map(str, lines)))
    return lines


def index_checks():
    """True when the loaded library is the index-check build (libmdpd_check.so, MDPD_LIB)."""
    return lib().mdpd_index_checks() == 1


def gaussian(si, sj, exact=True, fast=True):
    si = np.ascontiguousarray(si, np.uint32); sj = np.ascontiguousarray(sj, np.uint32)
    e = np.zeros(len(si)) if exact else None
    f = np.zeros(len(si), np.float32) if fast else None
    rc = lib().mdpd_gaussian(_ptr(si, C.c_uint32), _ptr(sj, C.c_uint32), _ptr(e, C.c_double),
                             _ptr(f, C.c_float), len(si))
    if rc:
        raise MdpdError(rc, lib().mdpd_last_error(None).decode())
    return e, f


def box_spec(n, L, style=0, A=-40.0, B=25.0, gamma=4.5, kT=1.0, cut=1.0, cut_r=0.75, cut_rho=0.75,
             sigma=3.0, dt=0.01, skin=0.3, rho_est=6.05, mass=1.0, seed=1234, every=1, delay=0, check=1,
             exact_rng=0, x=None, v=None, init_seed=1, fill_lo=(0, 0, 0), fill_hi=(0, 0, 0), lo=None, start_step=0):
    L = np.broadcast_to(np.asarray(L, float), (3,))
    lo = np.zeros(3) if lo is None else np.asarray(lo, float)
    s = BoxSpec()
    s.style, s.n = style, n
    s.lo[:] = list(lo); s.hi[:] = list(lo + L)
    s.A, s.B, s.gamma, s.kT, s.cut, s.cut_r, s.cut_rho, s.sigma = A, B, gamma, kT, cut, cut_r, cut_rho, sigma
    s.dt, s.skin, s.rho_est, s.mass, s.seed = dt, skin, rho_est, mass, seed
    s.every, s.delay, s.check, s.exact_rng = every, delay, check, exact_rng
    s._keep = []
    if x is not None:
        x = np.ascontiguousarray(x, np.float64); s._keep.append(x); s.x = _ptr(x, C.c_double)
    if v is not None:
        v = np.ascontiguousarray(v, np.float64); s._keep.append(v); s.v = _ptr(v, C.c_double)
    s.init_seed = init_seed
    s.fill_lo[:] = list(fill_lo); s.fill_hi[:] = list(fill_hi)
    s.start_step = int(start_step)
    return s


def place(specs, ndev, budget_bytes, steps=None):
    """device of each box or job (mdpd_place): work n * steps (steps None: n) balanced over ndev
    devices under each device's budget; returns (device_of, work_per_device); a box that fits no
    device gets -1 and raises MdpdError(ERR_BUDGET) unless every box was placed"""
    n = len(specs)
    arr = (BoxSpec * max(n, 1))(*specs)
    st = None if steps is None else np.ascontiguousarray(steps, np.int64)
    bud = np.ascontiguousarray(np.broadcast_to(np.asarray(budget_bytes, np.uint64), (ndev,)))
    dev = np.zeros(max(n, 1), np.int32)
    work = np.zeros(ndev)
    rc = lib().mdpd_place(arr, _ptr(st, C.c_int64) if st is not None else None, n, ndev, _ptr(bud, C.c_uint64),
                          _ptr(dev, C.c_int32), _ptr(work, C.c_double))
    if rc:
        raise MdpdError(rc, "mdpd_place: " + ("a box fits no device's budget" if rc == ERR_BUDGET else "bad argument"))
    return dev[:n], work


def box_bytes(spec):
    b = C.c_uint64()
    rc = lib().mdpd_box_bytes(C.byref(spec), C.byref(b))
    if rc:
        raise MdpdError(rc, "bad box spec")
    return b.value


class Batch:
    """Many independent boxes stepped by one captured graph per step."""

    def __init__(self, specs, device=0):
        L = lib()
        arr = (BoxSpec * len(specs))(*specs)
        h = C.c_void_p()
        rc = L.mdpd_batch_create(C.byref(h), arr, len(specs), C.byref(Opts(device, 0)))
        if rc:
            raise MdpdError(rc, L.mdpd_batch_last_error(None).decode())
        self.h, self.n = h, [s.n for s in specs]

    def _check(self, rc):
        if rc:
            raise MdpdError(rc, lib().mdpd_batch_last_error(self.h).decode())

    def setup(self):
        self._check(lib().mdpd_batch_setup(self.h))

    def step(self, n):
        self._check(lib().mdpd_batch_step(self.h, int(n)))

    def time(self, n):
        ms = C.c_double()
        self._check(lib().mdpd_batch_time(self.h, int(n), C.byref(ms)))
        return ms.value

    def profile(self, n):
        o = np.zeros(5)
        self._check(lib().mdpd_batch_profile(self.h, int(n), _ptr(o, C.c_double)))
        return dict(zip(["integrate_ms", "rebuild_ms", "density_ms", "force_ms", "rebuild_steps"], o.tolist()))

    def rebuild_steps(self):
        n = C.c_int64()
        self._check(lib().mdpd_batch_rebuild_steps(self.h, C.byref(n)))
        return n.value

    def tune(self, cache=None):
        """pair-pass shapes (density, force) picked by timing the batch's pair passes on its
        current state (the boxes do not advance); with cache (a JSON file path) a stored pick for
        this workload class is applied without timing.  With cache the result is
        (density, force, cached)."""
        a, b = C.c_int32(), C.c_int32()
        if cache is None:
            self._check(lib().mdpd_batch_tune(self.h, C.byref(a), C.byref(b)))
            return a.value, b.value
        hit = C.c_int32()
        self._check(lib().mdpd_batch_tune_cached(self.h, os.fsencode(cache), C.byref(a), C.byref(b), C.byref(hit)))
        return a.value, b.value, bool(hit.value)

    def set_shapes(self, density, force=32):
        """pin the pair-pass shapes (the values tune() reports) without timing"""
        self._check(lib().mdpd_batch_set_shapes(self.h, int(density), int(force)))

    def thermo(self, box):
        t = Thermo()
        self._check(lib().mdpd_batch_thermo(self.h, box, C.byref(t)))
        return t

    def run_thermo(self, nsteps):
        """nsteps steps, every step's thermo of every box ((nsteps, nbox) array of Thermo), read
        back while the next step runs; also the device-to-host bytes per step"""
        t = (Thermo * (int(nsteps) * len(self.n)))()
        nb = C.c_int64()
        self._check(lib().mdpd_batch_run_thermo(self.h, int(nsteps), t, C.byref(nb)))
        return [[t[k * len(self.n) + q] for q in range(len(self.n))] for k in range(int(nsteps))], nb.value

    def thermo_all(self):
        """every box's Thermo, batch order, from one pass"""
        t = (Thermo * len(self.n))()
        self._check(lib().mdpd_batch_thermo_all(self.h, t, len(self.n)))
        return list(t)

    def state(self, box, x=None, v=None):
        """Positions and velocities of one box in tag order; x, v: optional preallocated
        C-contiguous float64 (n, 3) arrays to fill (pinned ones make the copy a direct DMA)."""
        n = self.n[box]
        if x is None:
            x = np.empty((n, 3))  # every row is written
        if v is None:
            v = np.empty((n, 3))
        assert x.shape == (n, 3) and v.shape == (n, 3) and x.dtype == np.float64 and v.dtype == np.float64
        assert x.flags.c_contiguous and v.flags.c_contiguous
        self._check(lib().mdpd_batch_get_state(self.h, box, _ptr(x, C.c_double), _ptr(v, C.c_double), n))
        return x, v

    def states(self, xs=None, vs=None):
        """Every box's positions and velocities in tag order with one call (all copies back to back,
        one wait); xs, vs: optional lists of preallocated C-contiguous float64 (n_k, 3) arrays."""
        nb = len(self.n)
        xs = [np.empty((n, 3)) for n in self.n] if xs is None else xs
        vs = [np.empty((n, 3)) for n in self.n] if vs is None else vs
        assert len(xs) == nb and len(vs) == nb
        for a, n in zip(xs + vs, self.n + self.n):
            assert a.shape == (n, 3) and a.dtype == np.float64 and a.flags.c_contiguous
        dpt = C.POINTER(C.c_double)
        px = (dpt * nb)(*[_ptr(a, C.c_double) for a in xs])
        pv = (dpt * nb)(*[_ptr(a, C.c_double) for a in vs])
        self._check(lib().mdpd_batch_get_states(self.h, px, pv, nb))
        return xs, vs

    def close(self):
        if getattr(self, "h", None):
            lib().mdpd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Serving loop: HBM-budget admission, resident state, continuous batching."""

    def __init__(self, budget_bytes, device=0):
        h = C.c_void_p()
        rc = lib().mdpd_server_start(C.byref(h), int(budget_bytes), C.byref(Opts(device, 0)))
        if rc:
            raise MdpdError(rc, "server start failed")
        self.h = h

    def submit(self, spec, nsteps, keep_state=False):
        j = JobSpec()
        j.box = spec
        j.nsteps, j.keep_state = int(nsteps), int(keep_state)
        jid = C.c_int64()
        rc = lib().mdpd_server_submit(self.h, C.byref(j), C.byref(jid))
        if rc:
            raise MdpdError(rc, "submit refused")
        return jid.value

    def poll(self, jid):
        r = JobResult()
        rc = lib().mdpd_server_poll(self.h, jid, C.byref(r))
        if rc:
            raise MdpdError(rc, "poll failed")
        return r

    def state(self, jid, n):
        x = np.zeros((n, 3)); v = np.zeros((n, 3))
        rc = lib().mdpd_server_get_state(self.h, jid, _ptr(x, C.c_double), _ptr(v, C.c_double), n)
        if rc:
            raise MdpdError(rc, "no state")
        return x, v

    def cancel(self, jid):
        lib().mdpd_server_cancel(self.h, jid)

    def timing(self):
        """seconds in box creation, batch formation, setup of new boxes and chunks (host), the
        chunks' device seconds, the number of batches formed, and host seconds waiting with no
        job resident and retiring jobs"""
        o = np.zeros(8)
        rc = lib().mdpd_server_timing(self.h, _ptr(o, C.c_double))
        if rc:
            raise MdpdError(rc, "timing failed")
        return dict(zip(["create_s", "form_s", "setup_s", "chunks_s", "busy_s", "forms", "wait_s", "retire_s"],
                        o.tolist()))

    def set_step_particles(self, n):
        """particles stepped together: the resident jobs with the least remaining work, up to n
        (0: every resident job)"""
        rc = lib().mdpd_server_set_step_particles(self.h, C.c_int64(int(n)))
        if rc:
            raise MdpdError(rc, "bad step-particle cap")

    def preempt(self, jid):
        """checkpoint and release a job (state 5): state(jid, n) then returns its x, v and
        poll(jid).thermo.step the step to resubmit it from (box_spec(..., start_step=...))"""
        rc = lib().mdpd_server_preempt(self.h, jid)
        if rc:
            raise MdpdError(rc, "preempt refused")

    def drain(self, timeout_s=0.0):
        rc = lib().mdpd_server_drain(self.h, float(timeout_s))
        if rc:
            raise MdpdError(rc, "drain timed out")

    def stats(self):
        o = np.zeros(7)
        lib().mdpd_server_stats(self.h, _ptr(o, C.c_double))
        return dict(zip(["particle_steps_per_s", "step_ms_p50", "step_ms_p99", "job_s_p50", "job_s_p99",
                         "jobs_done", "peak_resident_bytes"], o.tolist()))

    def stop(self):
        if getattr(self, "h", None):
            lib().mdpd_server_stop(self.h)
            self.h = None

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass
