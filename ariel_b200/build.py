"""Builds the in-tree CUDA library ariel_b200/_lib/libariel_b200.so for sm_100a.

Every translation unit is compiled with --fmad=false (no contracted multiply-adds, so each
stage reproduces the reference's fp32 expressions bit for bit) and -lineinfo.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(HERE, "_build")
SO = os.path.join(OUT_DIR, "libariel_b200.so")
SOURCES = ["scan.cu", "particles.cu", "grid.cu", "pcg.cu", "host.cu", "server.cu", "noalloc.cu", "mesh.cu", "surface.cu", "sceneload.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def host_compiler():
    # The image's CXX points at a g++ without an OpenMP runtime; the system one is complete.
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    return "g++"


def flags():
    return ARCH + ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-ccbin", host_compiler(),
                   "-Xcompiler", "-fPIC,-ffp-contract=off", "-Xptxas", "-warn-spills",
                   "--expt-relaxed-constexpr", "--extended-lambda"]


def _needs(obj, src):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(HERE, "..", "include", "ariel.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src, extra):
    obj = os.path.join(OBJ_DIR, src.replace(".cu", ".o"))
    path = os.path.join(SRC, src)
    if not _needs(obj, path):
        return obj, ""
    cmd = [nvcc()] + flags() + extra + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stdout + r.stderr))
    return obj, r.stdout + r.stderr


def build(verbose=False, extra=()):
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(lambda s: _compile(s, list(extra)), SOURCES))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log.strip():
                print(log)
    if not os.path.exists(SO) or any(os.path.getmtime(o) > os.path.getmtime(SO) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-ccbin", host_compiler(), "-o", SO] + objs + ["-lcudart", "-lz"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stdout + r.stderr))
    return SO


if __name__ == "__main__":
    v = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else []
    print(build(verbose=v or bool(extra), extra=extra))
