"""Build the sm_100a library in-tree: rbmd_b200/_lib/librbmd_b200.so (and the `rbmd` host binary).

nvcc compiles every translation unit for `-gencode arch=compute_100a,code=sm_100a` only; the
library has no PyTorch dependency (the C ABI is plain C).  Run `python -m rbmd_b200.build`.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
OUT = os.path.join(HERE, "_lib")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "librbmd_b200.so")
BIN = os.path.join(OUT, "rbmd")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills", "-diag-suppress", "128", "-I", os.path.join(ROOT, "include")] + ARCH
CU_SOURCES = ["k_cells.cu", "k_pair.cu", "k_kspace.cu", "k_integrate.cu", "k_baro.cu", "k_diag.cu", "k_observe.cu", "engine.cu"]
CPP_SOURCES = ["capi.cpp", "serve.cpp", "tune.cpp", "observe.cpp", "snapshot.cpp"]


def nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(src_list, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list)


def _compile(src, extra=()):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    deps = [src] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "rbmd_gpu.h"))
    if _newer(deps, obj):
        cmd = [nvcc(), "-c", src, "-o", obj] + NVCC_FLAGS + list(extra)
        if src.endswith(".cpp"):
            cmd += ["-x", "cu"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
        if r.stderr.strip():
            sys.stderr.write(r.stderr)
    return obj


def build(verbose=False, jobs=None):
    os.makedirs(OUT, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in CU_SOURCES + CPP_SOURCES]
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(_compile, srcs))
    if _newer(objs, LIB):
        cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + ["-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    host_srcs = sorted(os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".cpp")) if os.path.isdir(HOST) else []
    host_deps = [os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith((".h", ".hpp"))] if host_srcs else []
    host_deps.append(os.path.join(ROOT, "include", "rbmd_gpu.h"))
    if host_srcs and _newer(host_srcs + [LIB] + host_deps, BIN):
        cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-o", BIN] + host_srcs + \
              ["-L", OUT, "-lrbmd_b200", "-Wl,-rpath,$ORIGIN", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"host build failed:\n{r.stderr}")
    if verbose:
        print(LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
