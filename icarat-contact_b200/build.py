"""Build libicarat_b200.so (sm_100a) in-tree.

    python icarat-contact_b200/build.py [--clean] [-j N]

Every .cu / .cpp under csrc/ is compiled by nvcc for
``-gencode arch=compute_100a,code=sm_100a`` into ``_build/`` and linked into
``lib/libicarat_b200.so`` next to this file.  The C++ app drivers under shim/
(ICARAT's apps over the C++ class shim) are linked against it into lib/.
Objects are rebuilt only when their source or any header is newer.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libicarat_b200.so")
SHIM = os.path.join(HERE, "shim")
CXX = shutil.which("g++", path="/usr/bin:" + os.environ.get("PATH", "")) or "g++"
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-O3", "-I" + INCLUDE, "-I" + SRC]
# nvcc drives the host compiler found on PATH; CXX from the environment is not used


def _headers():
    hs = glob.glob(os.path.join(SRC, "*.hpp")) + glob.glob(os.path.join(SRC, "*.cuh"))
    hs += glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src, hdr_time, verbose):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_time):
        return obj, None
    lang = [] if src.endswith(".cu") else ["-x", "cu"]
    cmd = [NVCC] + ARCH + FLAGS + lang + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, (r.stdout + r.stderr)
    if r.stderr.strip() and verbose:
        print(r.stderr, file=sys.stderr)
    return obj, None


def build(jobs=None, verbose=False, clean=False):
    if clean and os.path.isdir(BUILD):
        shutil.rmtree(BUILD)
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(SRC, "*.cu")) + glob.glob(os.path.join(SRC, "*.cpp")))
    ht = _headers()
    jobs = jobs or min(8, os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        res = list(ex.map(lambda s: _compile(s, ht, verbose), srcs))
    errs = [e for _, e in res if e]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    objs = [o for o, _ in res]
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    build_drivers(verbose)
    return LIB


def build_drivers(verbose=False):
    """shim/*_gpu.cpp -> lib/<name> (host C++, rpath to lib/)."""
    hdrs = glob.glob(os.path.join(SHIM, "*.hpp")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    ht = max([os.path.getmtime(h) for h in hdrs] + [os.path.getmtime(LIB)])
    out = []
    for src in sorted(glob.glob(os.path.join(SHIM, "*_gpu.cpp"))):
        exe = os.path.join(LIB_DIR, os.path.basename(src)[:-4])
        out.append(exe)
        if os.path.exists(exe) and os.path.getmtime(exe) >= max(os.path.getmtime(src), ht):
            continue
        cmd = [CXX, "-O2", "-std=c++17", "-Wall", "-I" + INCLUDE, "-I" + SHIM, src, "-o", exe,
               "-L" + LIB_DIR, "-licarat_b200", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("driver build failed:\n" + r.stdout + r.stderr)
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.j, a.v, a.clean))
