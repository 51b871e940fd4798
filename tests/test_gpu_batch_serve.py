"""Batched and served boxes: each box's result is bitwise the same alone and in the mix
(counter-based RNG, per-box deterministic lists and reductions); admission honours the
HBM budget; failures of one job leave the others' results unchanged."""
import json
import time

import numpy as np
import pytest

import mdpd

pytestmark = pytest.mark.gpu


def specs():
    out = []
    for k, (n, A, B, rd) in enumerate([(2200, -40, 25, 0.75), (7000, -45, 22, 0.72), (3300, -32, 28, 0.79),
                                       (12000, -50, 20, 0.70)]):
        L = (n / 6.05) ** (1 / 3)
        out.append(mdpd.box_spec(n, L, A=A, B=B, cut_r=rd, seed=100 + k, init_seed=7 + k))
    return out


def run_alone(spec, steps, gather=0):
    b = mdpd.Batch([spec])
    if gather:
        b.set_shapes(gather)
    b.setup()
    b.step(steps)
    x, v = b.state(0)
    t = b.thermo(0)
    b.close()
    return x, v, t


@pytest.mark.parametrize("gather", [4, 8])
def test_batch_equals_alone_bitwise(gather):
    # two of the density pass's shapes (neighbour gathers in flight per lane)
    sp = specs()
    steps = 120
    b = mdpd.Batch(sp)
    b.set_shapes(gather)
    b.setup()
    b.step(steps)
    for k, s in enumerate(sp):
        xa, va, ta = run_alone(s, steps, gather)
        xb, vb = b.state(k)
        assert np.array_equal(xa, xb) and np.array_equal(va, vb), k
        assert b.thermo(k).nbuild == ta.nbuild
    # every box's thermo in one pass equals the per-box calls (same fixed-order FP64 sums)
    every = b.thermo_all()
    for k in range(len(sp)):
        one = b.thermo(k)
        assert (every[k].step, every[k].natoms, every[k].nbuild) == (one.step, one.natoms, one.nbuild)
        assert (every[k].temp, every[k].pe, every[k].press) == (one.temp, one.pe, one.press)
    b.close()


def test_run_thermo_reads_every_step_as_step_and_thermo_do():
    # the pipelined call (step k's thermo read back while step k+1 runs) gives, for every step and
    # box, exactly what a step followed by a synchronous thermo read gives
    sp = specs()
    a = mdpd.Batch(sp)
    a.setup()
    ref = []
    for _ in range(12):
        a.step(1)
        ref.append([(t.step, t.temp, t.pe, t.press, t.nbuild) for t in a.thermo_all()])
    xa = [a.state(k) for k in range(len(sp))]
    a.close()
    b = mdpd.Batch(sp)
    b.setup()
    th, nbytes = b.run_thermo(12)
    assert nbytes > 0
    got = [[(t.step, t.temp, t.pe, t.press, t.nbuild) for t in row] for row in th]
    assert got == ref
    for k in range(len(sp)):
        xb, vb = b.state(k)
        assert np.array_equal(xa[k][0], xb) and np.array_equal(xa[k][1], vb)
    b.close()


def test_server_continuous_batching_matches_alone():
    sp = specs()
    steps = [90, 150, 60, 120]
    alone = [run_alone(s, n) for s, n in zip(sp, steps)]
    # budget for the two largest boxes: later jobs wait for memory and join mid-run
    foot = sorted(mdpd.box_bytes(s) for s in sp)
    budget = foot[-1] + foot[-2] + 1024
    srv = mdpd.Server(budget_bytes=budget)
    ids = []
    for s, n in zip(sp, steps):
        ids.append(srv.submit(s, n, keep_state=True))
        time.sleep(0.05)
    srv.drain(timeout_s=300)
    for k, jid in enumerate(ids):
        r = srv.poll(jid)
        assert r.state == 2 and r.steps_done == steps[k], (k, r.state, r.error)
        x, v = srv.state(jid, sp[k].n)
        assert np.array_equal(x, alone[k][0]) and np.array_equal(v, alone[k][1]), k
        assert r.step_ms_p99 >= r.step_ms_p50 > 0
    st = srv.stats()
    assert st["jobs_done"] == len(ids)
    assert st["peak_resident_bytes"] <= budget
    tm = srv.timing()  # where the loop's time went: every part counted, batches were formed
    assert all(tm[k] >= 0 for k in tm) and tm["forms"] >= 1 and tm["busy_s"] > 0
    assert tm["chunks_s"] >= tm["busy_s"] * 0.5
    srv.stop()


def test_server_steps_least_remaining_work_first():
    # with a step cap below the long job's size plus the short one's, a short job that arrives
    # while a long one runs steps alone until it is done (least remaining work first), then the
    # long one goes on; a job cancelled while it waits leaves without stepping; every result is
    # bitwise the run alone
    sp = specs()
    long_s, short_s, third = sp[3], sp[0], sp[1]
    alone_long = run_alone(long_s, 3000)
    alone_short = run_alone(short_s, 30)
    srv = mdpd.Server(budget_bytes=int(20e9))
    srv.set_step_particles(8000)
    jl = srv.submit(long_s, 3000, keep_state=True)
    time.sleep(0.2)  # the long job is under way
    js = srv.submit(short_s, 30, keep_state=True)
    jc = srv.submit(third, 100000)
    srv.cancel(jc)
    srv.drain(timeout_s=300)
    rl, rs, rc = srv.poll(jl), srv.poll(js), srv.poll(jc)
    assert rl.state == 2 and rs.state == 2 and rc.state == 4
    assert rs.end_s < rl.end_s
    assert rc.steps_done == 0
    for jid, ref, n in ((jl, alone_long, long_s.n), (js, alone_short, short_s.n)):
        x, v = srv.state(jid, n)
        assert np.array_equal(x, ref[0]) and np.array_equal(v, ref[1])
    with pytest.raises(mdpd.MdpdError):
        srv.set_step_particles(-1)
    srv.stop()


def test_server_refuses_oversized_and_cancels():
    srv = mdpd.Server(budget_bytes=int(5e8))
    big = mdpd.box_spec(2_000_000, (2e6 / 6.05) ** (1 / 3))
    with pytest.raises(mdpd.MdpdError) as e:
        srv.submit(big, 10)
    assert e.value.code == mdpd.ERR_BUDGET
    sp = specs()
    keep = srv.submit(sp[0], 40, keep_state=True)
    gone = srv.submit(sp[1], 100000)
    srv.cancel(gone)
    srv.drain(timeout_s=120)
    assert srv.poll(gone).state == 4
    assert srv.poll(keep).state == 2
    x, v = srv.state(keep, sp[0].n)
    xa, va, _ = run_alone(sp[0], 40)
    assert np.array_equal(x, xa) and np.array_equal(v, va)
    srv.stop()


def test_autotuner_picks_a_shape_and_keeps_the_physics():
    # pair-once mDPD batch: the density pass's gathers in flight; full-list DPD batch: threads
    # per particle. After tuning the batch keeps stepping with conserved momentum and no error.
    b = mdpd.Batch(specs())
    b.setup()
    b.step(20)
    g, f = b.tune()
    assert g in (4, 6, 8) and f in (0, 32)
    assert b.thermo(0).step == 20  # tuning times the pair passes on the state: no steps
    b.step(100)  # relaxation from the random start
    for k in range(4):
        t = b.thermo(k)
        assert t.status == 0 and 0.5 < t.temp < 2.0
        assert np.max(np.abs(t.momentum)) < 1e-6 * t.natoms
    b.close()
    d = mdpd.Batch([mdpd.box_spec(3000, 10.0, style=1, A=25.0, gamma=4.5, sigma=3.0, rho_est=0.0, seed=5,
                                  init_seed=6)])
    d.setup()
    td, tf = d.tune()
    assert td in (1, 2, 4) and tf in (1, 2, 4)
    d.step(20)
    assert d.thermo(0).status == 0
    d.close()


def test_tuning_leaves_the_state_as_it_was():
    # the autotuner evaluates each candidate's pair passes on the current state (no kick): the
    # forces it leaves are the ones the last step computed, so a tuned batch steps on bitwise as
    # a batch pinned to the same shapes without tuning
    sp = specs()
    a = mdpd.Batch(sp)
    a.setup()
    a.step(20)
    d, f = a.tune()
    a.step(30)
    b = mdpd.Batch(sp)
    b.setup()
    b.step(20)
    b.set_shapes(d, f)
    b.step(30)
    for k in range(len(sp)):
        xa, va = a.state(k)
        xb, vb = b.state(k)
        assert np.array_equal(xa, xb) and np.array_equal(va, vb)
    a.close()
    b.close()


def test_batch_states_equal_the_per_box_reads():
    # mdpd_batch_get_states: every box's x, v with one call, the same arrays as one
    # mdpd_batch_get_state per box; a null array is skipped
    b = mdpd.Batch(specs())
    b.setup()
    b.step(25)
    xs, vs = b.states()
    for k in range(len(xs)):
        x, v = b.state(k)
        assert np.array_equal(xs[k], x) and np.array_equal(vs[k], v)
    with pytest.raises(mdpd.MdpdError):
        b._check(mdpd.lib().mdpd_batch_get_states(b.h, None, None, len(xs)))
    b.close()


def test_box_beyond_the_table_limit_is_refused():
    # the list kernels address a box's neighbour table with unsigned 32-bit offsets: a box whose
    # table would pass 2^32 entries (here through a density estimate that makes the rows long)
    # is refused before anything is allocated, never silently wrapped
    L = (100000 / 6.05) ** (1 / 3)
    with pytest.raises(mdpd.MdpdError) as e:
        mdpd.Batch([mdpd.box_spec(100000, L, rho_est=2.0e5, seed=3, init_seed=4)])
    assert e.value.code == mdpd.ERR_ARG and "neighbour-table entries" in str(e.value)


def test_server_preempt_checkpoint_and_resume():
    # a preempted job leaves its x, v and step as a checkpoint, equal bit for bit to the
    # uninterrupted run at that step; the box resubmitted from it (start_step) continues the run
    # with the same random-number steps. As after a LAMMPS restart (x and v stored, forces
    # recomputed at setup), its first forces see v at the full step where the running integrator
    # had the half step, so 10 steps on it is close to the uninterrupted job but not equal; a
    # resume at the wrong step draws other random forces and is far further off.
    n = 20000
    L = (n / 6.05) ** (1 / 3)

    def spec(**kw):
        return mdpd.box_spec(n, L, A=-40.0, B=25.0, seed=77, init_seed=5, **kw)

    srv = mdpd.Server(20 << 30)
    b = srv.submit(spec(), 4000, keep_state=True)
    t0 = time.time()
    while srv.poll(b).steps_done == 0 and time.time() - t0 < 60:
        time.sleep(0.001)
    srv.preempt(b)
    srv.drain(120)
    rb = srv.poll(b)
    d = rb.steps_done
    assert rb.state == 5 and 0 < d < 4000 and rb.thermo.step == d
    xb, vb = srv.state(b, n)
    with pytest.raises(mdpd.MdpdError):
        srv.preempt(b)  # already ended
    c = srv.submit(spec(), d, keep_state=True)
    e = srv.submit(spec(), d + 10, keep_state=True)
    r = srv.submit(spec(x=xb, v=vb, start_step=d), 10, keep_state=True)
    w = srv.submit(spec(x=xb, v=vb), 10, keep_state=True)  # restarted at step 0: wrong RNG steps
    srv.drain(120)
    xc, vc = srv.state(c, n)
    assert np.array_equal(xc, xb) and np.array_equal(vc, vb)  # the checkpoint is the run at step d
    assert srv.poll(r).thermo.step == d + 10
    xe, ve = srv.state(e, n)
    xr, vr = srv.state(r, n)
    _, vw = srv.state(w, n)
    srv.stop()
    dv_r = np.sqrt(np.mean((vr - ve) ** 2))
    dv_w = np.sqrt(np.mean((vw - ve) ** 2))
    assert dv_r < 0.1 * dv_w and dv_w > 0.1, (dv_r, dv_w)
    dx = np.mod(xr - xe + L / 2, L) - L / 2
    assert np.abs(dx).max() < 1e-2



def test_tune_cache_persists_the_pick(tmp_path):
    cache = tmp_path / "tune.json"
    sp = specs()
    b = mdpd.Batch(sp)
    b.setup()
    d, f, hit = b.tune(cache=cache)
    assert not hit and d in (4, 6, 8) and f in (0, 32)
    assert b.thermo(0).step == 0  # the candidates' pair passes are timed on the state: no steps
    doc = json.loads(cache.read_text())
    (key, entry), = doc["entries"].items()
    assert "pair-once" in key and entry["density"] == d and entry["ms_per_step"] > 0
    b.close()
    # a batch of the same workload class takes the stored pick without stepping, and steps as a
    # batch configured by timing does
    b2 = mdpd.Batch(sp)
    b2.setup()
    assert b2.tune(cache=cache) == (d, f, True)
    assert b2.thermo(0).step == 0
    b2.step(30)
    assert b2.thermo(0).status == 0 and b2.thermo(0).step == 30
    b2.close()
    # a stored shape the family does not offer is refused, the file left as it was
    doc["entries"][key]["density"] = 5
    cache.write_text(json.dumps(doc))
    before = cache.read_text()
    b3 = mdpd.Batch(sp)
    b3.setup()
    with pytest.raises(mdpd.MdpdError) as e:
        b3.tune(cache=cache)
    assert e.value.code == mdpd.ERR_PARSE and "does not offer" in str(e.value)
    assert cache.read_text() == before
    b3.close()


def test_json_job_spec_runs_on_the_server(tmp_path):
    spec = {
        "budget_gb": 0.012,  # 12.9 MB: b (9.5 MB) alone, or a + dpd (11.6 MB) by size alone
        "jobs": [
            {"name": "a", "n": 3000, "box": 8.0, "steps": 60, "seed": 3, "init_seed": 5},
            # fits beside a, but a DPD box steps with other kernels: it waits until a has ended
            {"name": "dpd", "style": "dpd", "n": 3000, "box": 8.0, "A": 25, "sigma": 3.0, "steps": 30},
            {"name": "b", "n": 5000, "box": [12, 8, 8], "steps": 40, "seed": 4, "init_seed": 6},
        ],
    }
    p = tmp_path / "jobs.json"
    p.write_text(json.dumps(spec))
    n, foot = mdpd.validate_jobs(p)
    assert n == 3 and foot > 0
    lines = mdpd.run_jobs(p, tmp_path / "out.jsonl")
    jobs, summary = lines[:-1], lines[-1]["summary"]
    assert [j["job"] for j in jobs] == ["a", "dpd", "b"]
    for j, s in zip(jobs, spec["jobs"]):
        assert j["state"] == "done" and j["error"] == 0 and j["status"] == 0, j
        assert j["steps_done"] == s["steps"] and j["n"] == s["n"]
        assert j["nbuild"] > 0 and j["temp"] > 0 and j["particle_steps_per_s"] > 0
        assert j["step_ms_p99"] >= j["step_ms_p50"] > 0
    assert summary["done"] == 3 and summary["jobs"] == 3
    assert 0 < summary["peak_resident_bytes"] <= 0.012 * 2 ** 30
    assert jobs[1]["queue_s"] >= jobs[0]["run_s"] * 0.5  # the DPD job did not join a
    # the same jobs through the Python spec builder, each in a batch of its own, end in the same state
    for k, sp in ((0, mdpd.box_spec(3000, 8.0, seed=3, init_seed=5)),
                  (1, mdpd.box_spec(3000, 8.0, style=1, A=25, sigma=3.0))):
        alone = run_alone(sp, spec["jobs"][k]["steps"])
        assert alone[2].temp == jobs[k]["temp"] and alone[2].nbuild == jobs[k]["nbuild"], k


def test_server_keeps_pass_families_apart():
    # an exact-RNG job and a DPD job submitted beside a default mDPD job: each ends as it does alone
    sp = [mdpd.box_spec(2500, 7.5, seed=11, init_seed=2), mdpd.box_spec(2500, 7.5, seed=12, init_seed=3, exact_rng=1),
          mdpd.box_spec(2500, 7.5, style=1, A=25, seed=13, init_seed=4)]
    alone = [run_alone(s, 40) for s in sp]
    srv = mdpd.Server(budget_bytes=int(2e9))
    ids = [srv.submit(s, 40, keep_state=True) for s in sp]
    srv.drain(timeout_s=300)
    for k, jid in enumerate(ids):
        assert srv.poll(jid).state == 2
        x, v = srv.state(jid, sp[k].n)
        assert np.array_equal(x, alone[k][0]) and np.array_equal(v, alone[k][1]), k
    srv.stop()
    with pytest.raises(mdpd.MdpdError) as e:
        mdpd.Batch(sp[:2])
    assert e.value.code == mdpd.ERR_ARG and "RNG mode" in str(e.value)
