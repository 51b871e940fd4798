#!/usr/bin/env python
"""mDPD particle-steps/s on B200: batched (256 uneven boxes) vs plain single-box, with the
pair-kernel HBM roofline on a 4M-particle box, served p50/p99 latency, the CPU baseline and
the end-to-end number through the C ABI.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --profile-box N [--equil E] [--steps S] [--shape D] [--rebuild]

N > 1 runs under torchrun, one rank per GPU, each rank stepping its own 256-box set (weak
scaling, no collective on the data path); rank 0 prints ONE JSON line.

--profile-box N is the profiling leg (one GPU, for ncu launch lists and captures): one cubic
mDPD box of N particles (rho 6.05, A -40, B 25, r_d 0.75, skin 0.3) stepped E times, then S steps
in profile mode inside the NVTX range "prof" (integrate, rebuild, density and force as separate
launches timed with CUDA events; `ncu --nvtx --nvtx-include "prof/"` selects them) and, with
--rebuild, one forced full rebuild inside the range "rb".  --shape pins the density pass's
neighbour gathers in flight (4, 6 or 8); --exact uses the FP64 bit-exact pair gaussian.  Prints
one JSON line with the per-phase milliseconds and the graph step time.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "usermeso-2.0-mdpd_b200"))

RHO = 6.05
RC, SKIN = 1.0, 0.3
NBAR = RHO * 4.0 / 3.0 * math.pi * (RC + SKIN) ** 3          # list entries per particle, 55.7
B_RHO = 24 + 4 * NBAR                                         # density pass bytes / particle
B_F = 52 + 4 * NBAR                                           # force pass bytes / particle
B_STEP = B_RHO + B_F + 116                                    # + fused integrate (x, v, f, packs)
SERVE_ARRIVE_S, SERVE_WINDOW_S = 10.0, 40.0  # served leg: arrival span and measured window
WORKLOAD = ("batched mDPD: 256 periodic boxes, N log-uniform in [2k,200k], rho 6.05, "
            "A~U[-50,-30], B~U[20,30], r_d~U[0.7,0.8], kT 1, gamma 4.5, dt 0.01, skin 0.3")


def batched_boxes(seed, nbox=256):
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(np.log(2000), np.log(200000), nbox)).astype(int)
    A = rng.uniform(-50, -30, nbox); B = rng.uniform(20, 30, nbox); rd = rng.uniform(0.7, 0.8, nbox)
    return [dict(n=int(n[k]), L=(n[k] / RHO) ** (1 / 3), A=float(A[k]), B=float(B[k]), rd=float(rd[k]),
                 seed=int(1000 + k + 100000 * seed), init_seed=int(7 + k + 100000 * seed)) for k in range(nbox)]


def rank_boxes(rank, world):
    """This rank's boxes of the weak-scaling workload: world x 256 boxes of the batched workload (seeds
    1..world), placed on the ranks by the library's mdpd_place (particles balanced under a 150 GB
    budget per GPU).  Every rank computes the same placement; nothing is exchanged."""
    cfg = sum((batched_boxes(seed=1 + r) for r in range(world)), [])
    if world == 1:
        return cfg
    import mdpd
    dev, _ = mdpd.place(specs_of(cfg), world, int(150e9))
    return [c for c, d in zip(cfg, dev) if d == rank]


def specs_of(cfg):
    import mdpd
    return [mdpd.box_spec(c["n"], c["L"], A=c["A"], B=c["B"], cut_r=c["rd"], seed=c["seed"],
                          init_seed=c["init_seed"]) for c in cfg]


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, dev):
        self.dev, self.lines, self.p = dev, [], None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.p = None
        return self

    def _read(self):
        for line in self.p.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.p:
            time.sleep(0.25)
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0])); mx = float(f[1])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[3 + k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def aggregate(particle_steps, seconds, world, device="cuda"):
    """Whole-job throughput over ranks: particle-steps summed, time = max over ranks."""
    if world == 1:
        return particle_steps / seconds, seconds
    import torch
    import torch.distributed as dist
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    p = torch.tensor([particle_steps], dtype=torch.float64, device=device)
    dist.all_reduce(p, op=dist.ReduceOp.SUM)
    return float(p.item()) / float(t.item()), float(t.item())


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_per_launch():
    """DRAM bytes per step of the density and force passes (ncu capture of a 1M box, scaled
    by particle count to the 4M box) from the committed profile summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "pair_passes_ncu.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def cpu_baseline(cfg, budget_s=15.0, threads=0):
    """The oracle's FP64 engine (OpenMP over all host threads) on a bounded sample of boxes."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    ncores = threads or os.cpu_count() or 1
    order = sorted(range(len(cfg)), key=lambda k: cfg[k]["n"])
    pick = [order[len(order) // 2], order[len(order) // 4], order[(3 * len(order)) // 4]]
    done_ps, spent = 0.0, 0.0
    sample = []
    for k in pick:
        c = cfg[k]
        rng = np.random.default_rng(c["init_seed"])
        x = rng.uniform(0, c["L"], (c["n"], 3)); v = rng.normal(0, 1, (c["n"], 3)); v -= v.mean(0)
        sim = oracle.Sim(x, v, (0, 0, 0), (c["L"],) * 3, A=c["A"], B=c["B"], cut_r=c["rd"], seed=c["seed"],
                         nthreads=ncores)
        sim.setup()
        sim.run(1)
        t0 = time.perf_counter()
        sim.run(2)
        dt = (time.perf_counter() - t0) / 2
        steps = max(1, min(200, int((budget_s / len(pick)) / max(dt, 1e-6))))
        t0 = time.perf_counter()
        sim.run(steps)
        el = time.perf_counter() - t0
        sim.close()
        done_ps += c["n"] * steps
        spent += el
        sample.append(f"box n={c['n']} x {steps} steps")
    return {"value": done_ps / spent, "unit": "particle-steps/s", "cores": ncores, "kind": "port",
            "sample": "oracle FP64 engine (OpenMP) on 3 boxes of the 256-box set: " + "; ".join(sample)}


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU path (the oracle port; the 2013 reference has no
    CPU mDPD style) on the host cores, same workload, bounded sample per step."""
    if rank != 0:
        return
    cfg = batched_boxes(seed=1)
    base = cpu_baseline(cfg, budget_s=max(5.0, 0.3 * (args.steps + args.warmup)))
    line = {"impl": "reference", "metric": "mDPD particle-steps/s (batched 256-box workload)",
            "value": base["value"], "unit": "particle-steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded)", "config": {"workload": WORKLOAD},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def profile_box(args):
    import torch
    import mdpd
    n = args.profile_box
    L = (n / RHO) ** (1 / 3)
    b = mdpd.Batch([mdpd.box_spec(n, L, A=-40.0, B=25.0, seed=4242, init_seed=99, exact_rng=int(args.exact))])
    if args.shape:
        b.set_shapes(args.shape)
    b.setup()
    b.step(args.equil)
    r0 = b.rebuild_steps()
    torch.cuda.nvtx.range_push("prof")
    p = b.profile(args.steps)
    torch.cuda.nvtx.range_pop()
    out = {"particles": n, "shape": args.shape or "default", "rng": "exact" if args.exact else "fast",
           "profile_ms": p,
           "rebuild_steps": b.rebuild_steps() - r0}
    if args.rebuild:
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("rb")
        b.setup()
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
    out["graph_ms_per_step"] = b.time(args.steps)
    b.close()
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours")
    ap.add_argument("--equil", type=int, default=300, help="untimed equilibration steps from the random start")
    ap.add_argument("--no-extras", action="store_true", help="skip plain/served/roofline/cpu legs")
    ap.add_argument("--profile-box", type=int, default=0, help="profiling leg: one cubic box of this many particles")
    ap.add_argument("--shape", type=int, default=0, help="profiling leg: pinned density shape (4, 6, 8)")
    ap.add_argument("--rebuild", action="store_true", help="profiling leg: one forced rebuild in the range rb")
    ap.add_argument("--exact", action="store_true", help="profiling leg: FP64 bit-exact pair gaussian (rng exact)")
    args = ap.parse_args()
    if args.profile_box:
        profile_box(args)
        return
    rank = int(os.environ.get("RANK", "0")); world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    import mdpd

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    # ---- headline: batched 256-box workload (per GPU), resident in HBM -----------------------
    cfg = rank_boxes(rank, world)
    specs = specs_of(cfg)
    ntot = sum(c["n"] for c in cfg)
    b = mdpd.Batch(specs, device=local)
    b.setup()
    b.step(args.equil)  # relax the random start (untimed)
    shape_density, shape_force = b.tune()  # project autotuner (pair passes timed on the current state)
    b.step(args.warmup)
    r0 = b.rebuild_steps()
    barrier()
    with Clocks(local) as clk:
        barrier()
        torch.cuda.nvtx.range_push("timed")  # ncu --nvtx --nvtx-include timed/ selects these launches
        ms = b.time(args.steps)              # CUDA events on the batch stream, K steps
        torch.cuda.nvtx.range_pop()
        barrier()
    r1 = b.rebuild_steps()
    value, t_max = aggregate(ntot * args.steps, ms * args.steps / 1e3, world)
    # a pair-once mDPD step: integrate, density, force, finalize; a rebuilding step adds 17
    gpu_launches = 4 * args.steps + 17 * (r1 - r0)
    eq_states = [b.state(k) for k in range(len(cfg))] if not args.no_extras else None
    b.close()

    line = {"metric": "mDPD particle-steps/s (batched 256-box workload)", "value": value,
            "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 pair / f64 integrate", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "boxes": len(cfg), "particles_per_gpu": ntot,
                       "start": f"uniform random positions, Maxwell velocities, {args.equil} untimed steps, "
                                "then the autotuner (pair passes timed per candidate shape, no steps)",
                       "rebuild_steps_timed": r1 - r0,
                       "l2": "inputs larger than L2: state + lists of ~%d particles (%.1f GB)" % (
                           ntot, ntot * 1.1e-6),
                       "parallelism": f"{world} GPU(s), {256 * world} boxes placed by mdpd_place "
                                      "(no data-path collective)",
                       "tuned": {"density_gathers_in_flight": shape_density,
                                 "force_rows_staged": shape_force == 32}},
            "clocks": clk.summary(), "gpu_launches": gpu_launches}

    if not args.no_extras:
        # ---- e2e through the C ABI on every rank (its own box set): pinned host arrays in,
        # every step's thermo read back, final state into pinned host arrays; creation, upload
        # and setup inside the timing; particle-steps summed, wall time max over ranks ----
        xs = [x for x, _ in eq_states]
        vs = [v for _, v in eq_states]

        def pinned(shape):
            return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()

        xin = [pinned(x.shape) for x in xs]
        vin = [pinned(v.shape) for v in vs]
        xout = [pinned(x.shape) for x in xs]
        vout = [pinned(v.shape) for v in vs]
        for a, b_ in zip(xin + vin, xs + vs):
            a[:] = b_
        barrier()
        t0 = time.perf_counter()
        sp = [mdpd.box_spec(c["n"], c["L"], A=c["A"], B=c["B"], cut_r=c["rd"], seed=c["seed"], x=x, v=v)
              for c, x, v in zip(cfg, xin, vin)]
        be = mdpd.Batch(sp, device=local)
        be.setup()
        t1 = time.perf_counter()
        # K steps; every step's result (every box's thermo, with that step's energy and virial)
        # comes back to the host while the next step runs
        th, thermo_bytes = be.run_thermo(args.steps)
        temps = [[t.temp for t in row] for row in th]
        t2 = time.perf_counter()
        be.states(xout, vout)  # every box's state with one call (mdpd_batch_get_states)
        e2e_s = time.perf_counter() - t0
        split = {"create_upload_setup_s": t1 - t0, "steps_s": t2 - t1, "download_s": e2e_s - (t2 - t0)}
        be.close()
        state_bytes = 48 * ntot
        e2e_value, e2e_max_s = aggregate(ntot * args.steps, e2e_s, world)
        all_state_bytes, _ = aggregate(state_bytes, 1.0, world)  # summed over ranks
        all_thermo_bytes, _ = aggregate(thermo_bytes, 1.0, world)
        line["e2e"] = {"value": e2e_value, "unit": "particle-steps/s",
                       "h2d_bytes_per_step": int(all_state_bytes / args.steps),
                       "d2h_bytes_per_step": int(all_state_bytes / args.steps + all_thermo_bytes),
                       "note": "wall clock of: create of all 256 boxes from pinned host x, v; setup; K steps, "
                               "each followed by a read of every box's thermo (mdpd_batch_run_thermo: step k's "
                               "thermo comes back while step k+1 runs); full state download into pinned host "
                               "arrays (mdpd_batch_get_states: every box with one call)",
                       "split": split}
        del temps, xin, vin, xout, vout

    # per-GPU legs (plain path, pair-pass roofline, served jobs, CPU baseline): one GPU only, so a
    # multi-GPU run holds its GPUs no longer than the timed and end-to-end legs need
    if not args.no_extras and world == 1:
        # ---- plain single-box path on the same boxes (one box per launch sequence) ----------
        plain_ps, plain_s = 0.0, 0.0
        for c, x, v in zip(cfg, xs, vs):
            s = mdpd.box_spec(c["n"], c["L"], A=c["A"], B=c["B"], cut_r=c["rd"], seed=c["seed"], x=x, v=v)
            bb = mdpd.Batch([s], device=local)
            bb.setup()
            bb.step(3)
            msb = bb.time(20)
            plain_ps += c["n"] * 20
            plain_s += msb * 20 / 1e3
            bb.close()
        line["plain"] = {"value": plain_ps / plain_s, "unit": "particle-steps/s",
                         "note": "same 256 boxes, each stepped alone (20 steps, CUDA events)",
                         "batched_over_plain": value / world / (plain_ps / plain_s)}

        # ---- roofline: pair passes of the 4M-particle cubic box -----------------------------
        n4 = 4_000_000
        s4 = mdpd.box_spec(n4, (n4 / RHO) ** (1 / 3), A=-40.0, B=25.0, seed=4242, init_seed=99)
        b4 = mdpd.Batch([s4], device=local)
        b4.setup()
        b4.step(args.equil)
        tuned4 = b4.tune()  # the project autotuner's shape for this box (pair passes timed per candidate)
        b4.step(args.warmup)
        torch.cuda.nvtx.range_push("pair_profile")  # ncu --nvtx-include pair_profile/: the launch list
        prof = b4.profile(max(10, args.steps // 2))
        torch.cuda.nvtx.range_pop()
        ms4 = b4.time(max(10, args.steps // 2))
        b4.close()
        peak, how = peaks()
        t_pair = (prof["density_ms"] + prof["force_ms"]) / 1e3
        achieved = (B_RHO + B_F) * n4 / t_pair / 1e9
        tr = traffic_per_launch()
        line["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "peak_source": how,
                            "traffic": tr.get("pair_bytes_per_step") if tr else None,
                            "kernel": "pair passes (density + force), 4M-particle box",
                            "bytes_per_particle": B_RHO + B_F, "nbar": NBAR,
                            "density_ms": prof["density_ms"], "force_ms": prof["force_ms"],
                            "density_frac": B_RHO * n4 / (prof["density_ms"] / 1e3) / 1e9 / peak,
                            "force_frac": B_F * n4 / (prof["force_ms"] / 1e3) / 1e9 / peak,
                            "integrate_ms": prof["integrate_ms"], "rebuild_ms_avg": prof["rebuild_ms"],
                            "tuned": {"density_gathers_in_flight": tuned4[0], "force_rows_staged": tuned4[1] == 32}}
        line["single_box_4M"] = {"value": n4 / (ms4 / 1e3), "unit": "particle-steps/s", "ms_per_step": ms4,
                                 "step_frac": B_STEP * n4 / (ms4 / 1e3) / 1e9 / peak,
                                 "note": "whole graph step (rebuilds amortised) against the step's algorithmic "
                                         "bytes, pair passes + integrate = %.1f B/particle" % B_STEP}

        # ---- served: Poisson arrivals of droplet/slab jobs over a fixed window -----------------
        # Poisson(20/s) arrivals of droplet/slab jobs for SERVE_ARRIVE_S seconds, N log-uniform in
        # [5k, 2M], 2,000-20,000 steps each, parameters as the batched workload, 150 GB budget; the server
        # runs until SERVE_WINDOW_S after the first arrival.  Throughput is the particle-steps
        # every job completed by then (finished or not) over the window's wall time.
        srv = mdpd.Server(budget_bytes=int(150e9), device=local)
        rng = np.random.default_rng(5)
        t_arr, ta = [], 0.0
        while True:
            ta += rng.exponential(1 / 20.0)
            if ta > SERVE_ARRIVE_S:
                break
            t_arr.append(ta)
        jobs = []
        t0 = time.perf_counter()
        for k, tk in enumerate(t_arr):
            while time.perf_counter() - t0 < tk:
                time.sleep(0.001)
            n = int(np.exp(rng.uniform(np.log(5000), np.log(2_000_000))))
            steps = int(rng.integers(2000, 20001))
            L = (2 * n / RHO) ** (1 / 3)
            slab = rng.random() < 0.5
            sp = mdpd.box_spec(n, L, A=float(rng.uniform(-50, -30)), B=float(rng.uniform(20, 30)),
                               cut_r=float(rng.uniform(0.7, 0.8)), seed=5000 + k, init_seed=900 + k,
                               fill_lo=(0.25 * L, 0, 0) if slab else (0.103 * L,) * 3,
                               fill_hi=(0.75 * L, L, L) if slab else (0.897 * L,) * 3)
            jobs.append((srv.submit(sp, steps), n, steps))
        while time.perf_counter() - t0 < SERVE_WINDOW_S:
            time.sleep(0.05)
        wall = time.perf_counter() - t0
        res = [(srv.poll(j), n, steps) for j, n, steps in jobs]
        st = srv.stats()
        tm = srv.timing()
        for j, _, _ in jobs:
            srv.cancel(j)
        srv.stop()
        done_ps = sum(n * r.steps_done for r, n, _ in res)
        lat = [r.end_s - r.submit_s for r, _, _ in res if r.state == 2]
        line["served"] = {"throughput": done_ps / wall, "unit": "particle-steps/s",
                          "throughput_busy": st["particle_steps_per_s"],
                          "step_ms_p50": st["step_ms_p50"], "step_ms_p99": st["step_ms_p99"],
                          "job_s_p50": float(np.percentile(lat, 50)) if lat else None,
                          "job_s_p99": float(np.percentile(lat, 99)) if lat else None,
                          "jobs_submitted": len(jobs), "jobs_completed": len(lat),
                          "particle_steps_offered": float(sum(n * steps for _, n, steps in jobs)),
                          "window_s": wall,
                          "served_over_plain": done_ps / wall / (plain_ps / plain_s),
                          "loop_s": tm,
                          "sample": f"Poisson(20/s) droplet/slab jobs arriving over {SERVE_ARRIVE_S:.0f} s, N "
                                    "log-uniform 5k-2M, steps U{2000..20000}, 150 GB budget; throughput = "
                                    f"particle-steps done in the first {SERVE_WINDOW_S:.0f} s / wall time; job "
                                    "latency over the jobs that completed in it"}

        # ---- CPU baseline (oracle port on host cores) ---------------------------------------
        line["cpu_baseline"] = cpu_baseline(cfg)

    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
