"""Builds graphic_lab_task_b200/liblrt_b200.so in-tree (nvcc + g++).

    python -m graphic_lab_task_b200.build          # incremental
    python -m graphic_lab_task_b200.build --force

Kernels are compiled for sm_100a only.  trace_exact.cu is built with
-fmad=false and IEEE division/square root so that its arithmetic rounds like
the reference CPU build with -ffp-contract=off; trace_fast.cu lets ptxas
contract multiply-adds.  Host C++ is built with -ffp-contract=off for the
same reason (the derived layouts must hold the reference's exact floats).
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblrt_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "-I" + CSRC,
               "-I" + INCLUDE, "--expt-relaxed-constexpr"] + ARCH
CXX_COMMON = ["-std=c++17", "-O3", "-fPIC", "-fopenmp", "-ffp-contract=off", "-I" + CSRC, "-I" + INCLUDE,
              "-I" + os.path.join(CUDA_HOME, "include")]

SOURCES = {
    "trace_exact.cu": ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"],
    "trace_fast.cu": ["-fmad=true", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"],
    "device.cu": [],
    "batch.cu": [],
    "adjoint.cu": [],
    "wavefront.cu": [],
    "lbvh.cu": [],
    "scene.cpp": None,
    "layout.cpp": None,
    "workloads.cpp": None,
}
HEADERS = ["trace_impl.cuh", "device_layout.h", "lrt_math.h", "scene.h", "layout.h", "trace_api.h", "device_scene.h",
           "lbvh.h"]


def _stale(obj, src):
    if not os.path.exists(obj):
        return True
    deps = [src] + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(name, extra, verbose):
    src = os.path.join(CSRC, name)
    obj = os.path.join(OUT_DIR, name + ".o")
    if extra is None:
        cmd = ["g++"] + CXX_COMMON + ["-c", src, "-o", obj]
    else:
        cmd = [NVCC] + NVCC_COMMON + extra + ["-c", src, "-o", obj]
        if verbose:
            cmd.append("-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return obj, r.stderr


def build(force=False, verbose=False):
    """Compile every CUDA/C++ source for sm_100a and link liblrt_b200.so."""
    if not os.path.exists(NVCC):
        raise RuntimeError("nvcc not found at %s" % NVCC)
    os.makedirs(OUT_DIR, exist_ok=True)
    jobs = {}
    objs = []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for name, extra in SOURCES.items():
            obj = os.path.join(OUT_DIR, name + ".o")
            objs.append(obj)
            if force or _stale(obj, os.path.join(CSRC, name)):
                jobs[ex.submit(_compile, name, extra, verbose)] = name
        logs = []
        for f in cf.as_completed(jobs):
            _, err = f.result()
            if verbose and err:
                logs.append("[%s]\n%s" % (jobs[f], err))
    relink = force or bool(jobs) or not os.path.exists(LIB)
    if relink:
        tmp = LIB + ".tmp"
        cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-Xcompiler", "-fopenmp", "-lgomp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
        shutil.move(tmp, LIB)
    if verbose:
        for l in logs:
            print(l)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true", help="print ptxas register/spill reports")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    sys.exit(main())
