"""Build libmdpd.so in-tree for sm_100a (B200).

    python usermeso-2.0-mdpd_b200/build.py [--force] [--debug]

Compiles csrc/*.cu and csrc/*.cpp with nvcc (-gencode arch=compute_100a,code=sm_100a
-lineinfo), one process per translation unit, and links them into
usermeso-2.0-mdpd_b200/libmdpd.so next to this file.  Objects go to _build/ beside it.
Also builds the command-line driver `lmp_mdpd` (LAMMPS-style `-in script`).
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmdpd.so")
EXE = os.path.join(HERE, "lmp_mdpd")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def flags(debug):
    f = ["-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "-I" + os.path.join(HERE, "..", "include"), "--expt-relaxed-constexpr"]
    f += ["-O0", "-g"] if debug else ["-O3"]
    return f + ARCH


def compile_one(src, obj, debug):
    cmd = [NVCC] + flags(debug) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise SystemExit(r.returncode)
    return obj


def newer(src, dst, deps):
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(p) > t for p in [src] + deps)


def build(force=False, debug=False, verbose=True):
    os.makedirs(OBJ, exist_ok=True)
    headers = glob.glob(os.path.join(SRC, "*.h")) + glob.glob(os.path.join(SRC, "*.cuh")) + \
        [os.path.join(HERE, "..", "include", "mdpd.h")]
    srcs = sorted(glob.glob(os.path.join(SRC, "*.cu")) + glob.glob(os.path.join(SRC, "*.cpp")))
    lib_srcs = [s for s in srcs if not s.endswith("main.cpp")]
    jobs = []
    objs = []
    with cf.ThreadPoolExecutor(max_workers=max(2, os.cpu_count() or 2)) as ex:
        for s in srcs:
            o = os.path.join(OBJ, os.path.basename(s) + ".o")
            objs.append(o)
            if force or newer(s, o, headers):
                jobs.append(ex.submit(compile_one, s, o, debug))
        for j in jobs:
            j.result()
    lib_objs = [o for s, o in zip(srcs, objs) if s in lib_srcs]
    if force or jobs or not os.path.exists(LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + lib_objs + ["-lpthread"]
        subprocess.check_call(cmd)
    main_obj = [o for s, o in zip(srcs, objs) if s.endswith("main.cpp")]
    if main_obj and (force or jobs or not os.path.exists(EXE)):
        cmd = [NVCC] + ARCH + ["-o", EXE] + main_obj + ["-L" + HERE, "-lmdpd",
                                                        "-Xlinker", "-rpath=$ORIGIN"]
        subprocess.check_call(cmd)
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--debug", action="store_true")
    a = ap.parse_args()
    build(a.force, a.debug)
