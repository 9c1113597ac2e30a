"""Build the in-tree CUDA library nuosc_b200/libnuosc_b200.so for sm_100a.

    python nuosc_b200/build.py

nvcc cross-compiles without a GPU.  Every .cu/.cpp under csrc/ is compiled
with -gencode arch=compute_100a,code=sm_100a and linked into one shared
library exporting the C ABI of include/nuosc_b200.h.
"""
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libnuosc_b200.so")
OBJ = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _stale(obj, src, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src] + deps)


def build(verbose=False, jobs=8, extra=()):
    os.makedirs(OBJ, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    cc = nvcc()
    procs, objs = [], []
    for src in sources():
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(obj)
        if not _stale(obj, src, headers):
            continue
        cmd = [cc] + ARCH + NVCC_FLAGS + list(extra) + ["-x", "cu", "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        if len(procs) >= jobs:
            _drain(procs)
    _drain(procs)
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [cc] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    build_driver(verbose)
    return LIB


def build_driver(verbose=False):
    """The command-line driver nuosc_b200/nuosc (the reference's main, on the C ABI)."""
    src = os.path.join(HERE, "driver", "nuosc_main.cpp")
    exe = os.path.join(HERE, "nuosc")
    deps = [src, LIB, os.path.join(ROOT, "include", "nuosc_b200.hpp"), os.path.join(ROOT, "include", "nuosc_b200.h")]
    if os.path.exists(exe) and all(os.path.getmtime(exe) >= os.path.getmtime(d) for d in deps):
        return exe
    cxx = next((c for c in ("/usr/bin/g++", shutil.which("g++")) if c and os.path.exists(c)), None)
    if cxx is None:
        raise RuntimeError("g++ not found")
    cmd = [cxx, "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), src, "-L" + HERE, "-lnuosc_b200",
           "-Wl,-rpath,$ORIGIN", "-o", exe]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return exe


def _drain(procs):
    errs = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            errs.append("%s:\n%s" % (src, out.decode(errors="replace")))
        elif out.strip():
            sys.stderr.write(out.decode(errors="replace"))
    procs.clear()
    if errs:
        raise RuntimeError("nvcc failed\n" + "\n".join(errs))


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
