"""Build libmdpd.so in-tree for sm_100a (B200).

    python usermeso-2.0-mdpd_b200/build.py [--force] [--debug] [--check]

Compiles csrc/*.cu and csrc/*.cpp with nvcc (-gencode arch=compute_100a,code=sm_100a
-lineinfo), one process per translation unit, and links them into
usermeso-2.0-mdpd_b200/libmdpd.so next to this file.  Objects go to _build/ beside it.
Also builds the command-line driver `lmp_mdpd` (LAMMPS-style `-in script`).

--check builds libmdpd_check.so instead (objects in _build_check/): the same sources with
-DMDPD_CHECK, which bounds-checks every neighbour, bin, bucket and permutation index the
kernels read or write.  An index outside its array sets status bit 64 of its box and the
access is skipped (no trap), so a run reports the error through the normal status path.  Load
it in place of libmdpd.so with MDPD_LIB=<path>/libmdpd_check.so.
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
CHECK_LIB = os.path.join(HERE, "libmdpd_check.so")
EXE = os.path.join(HERE, "lmp_mdpd")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def flags(debug, check=False):
    f = ["-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "-I" + os.path.join(HERE, "..", "include"), "--expt-relaxed-constexpr"]
    f += ["-O0", "-g"] if debug else ["-O3"]
    if check:
        f += ["-DMDPD_CHECK"]
    return f + ARCH


def compile_one(src, obj, debug, check=False):
    cmd = [NVCC] + flags(debug, check) + ["-c", src, "-o", obj]
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


def build(force=False, debug=False, verbose=True, check=False):
    obj_dir = OBJ + "_check" if check else OBJ
    lib = CHECK_LIB if check else LIB
    os.makedirs(obj_dir, exist_ok=True)
    headers = glob.glob(os.path.join(SRC, "*.h")) + glob.glob(os.path.join(SRC, "*.cuh")) + \
        [os.path.join(HERE, "..", "include", "mdpd.h")]
    srcs = sorted(glob.glob(os.path.join(SRC, "*.cu")) + glob.glob(os.path.join(SRC, "*.cpp")))
    lib_srcs = [s for s in srcs if not s.endswith("main.cpp")]
    jobs = []
    objs = []
    with cf.ThreadPoolExecutor(max_workers=max(2, os.cpu_count() or 2)) as ex:
        for s in srcs:
            if check and s.endswith("main.cpp"):
                continue
            o = os.path.join(obj_dir, os.path.basename(s) + ".o")
            objs.append(o)
            if force or newer(s, o, headers):
                jobs.append(ex.submit(compile_one, s, o, debug, check))
        for j in jobs:
            j.result()
    if check:
        srcs = lib_srcs
    lib_objs = [o for s, o in zip(srcs, objs) if s in lib_srcs]
    if force or jobs or not os.path.exists(lib):
        cmd = [NVCC] + ARCH + ["-shared", "-o", lib] + lib_objs + ["-lpthread"]
        subprocess.check_call(cmd)
    main_obj = [o for s, o in zip(srcs, objs) if s.endswith("main.cpp")]
    if main_obj and (force or jobs or not os.path.exists(EXE)):
        cmd = [NVCC] + ARCH + ["-o", EXE] + main_obj + ["-L" + HERE, "-lmdpd",
                                                        "-Xlinker", "-rpath=$ORIGIN"]
        subprocess.check_call(cmd)
    if verbose:
        print("built", lib)
    return lib


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--debug", action="store_true")
    ap.add_argument("--check", action="store_true")
    a = ap.parse_args()
    build(a.force, a.debug, check=a.check)
