"""Profiling driver: one cubic mDPD box (rho 6.05, A -40, B 25, r_d 0.75, skin 0.3) with its
kernels launched one by one under NVTX ranges, for ncu launch lists and captures.

    python usermeso-2.0-mdpd_b200/prof_box.py [--n N] [--equil E] [--steps S] [--rebuild]

Ranges: "prof" holds S steps in profile mode (integrate, rebuild kernels, density pass, force
pass as separate launches timed with CUDA events); "rb" holds one forced full rebuild (sort,
ghosts, bins, list) of the equilibrated box when --rebuild is given.  Select them with
`ncu --nvtx --nvtx-include "prof/"` (or "rb/").  Prints the per-phase milliseconds and the
graph step time.
"""
import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--equil", type=int, default=30)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--rebuild", action="store_true")
    a = ap.parse_args()
    import torch
    import mdpd
    L = (a.n / 6.05) ** (1 / 3)
    b = mdpd.Batch([mdpd.box_spec(a.n, L, A=-40.0, B=25.0, seed=4242, init_seed=99)])
    b.setup()
    b.step(a.equil)
    r0 = b.rebuild_steps()
    torch.cuda.nvtx.range_push("prof")
    p = b.profile(a.steps)
    torch.cuda.nvtx.range_pop()
    print("profile", p, "rebuild steps:", b.rebuild_steps() - r0, flush=True)
    if a.rebuild:
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("rb")
        b.setup()
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
    print("graph ms/step", b.time(a.steps), flush=True)
    b.close()


if __name__ == "__main__":
    main()
