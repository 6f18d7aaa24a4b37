"""Build libfft3d_b200.so (sm_100a) and the CPU test helper, in-tree.

    python opt-fft_b200/build.py [--jobs N] [--force]

nvcc cross-compiles for sm_100a without a GPU.  Outputs:
    opt-fft_b200/libfft3d_b200.so          the product: C ABI + CUDA kernels
    opt-fft_b200/build/libfft3d_hostcheck.so   CPU run of the kernels' pass code (tests only)
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "build")
LIB = os.path.join(HERE, "libfft3d_b200.so")
HOSTCHECK = os.path.join(BUILD, "libfft3d_hostcheck.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-rdc=true", "-Xcompiler", "-fPIC",
                  "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def _newer(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise SystemExit(f"build failed: {os.path.basename(cmd[-1])}")
    return r.stdout + r.stderr


def build(jobs=None, force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) \
        + glob.glob(os.path.join(HERE, "..", "include", "*.h"))
    cus = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    objs, work = [], []
    for cu in cus:
        obj = os.path.join(BUILD, os.path.basename(cu)[:-3] + ".o")
        objs.append(obj)
        if force or not _newer(obj, [cu] + headers):
            work.append([NVCC] + NVFLAGS + ["-c", cu, "-o", obj])
    host_obj = os.path.join(BUILD, "tables_host.o")
    host_src = os.path.join(CSRC, "tables_host.cpp")
    if force or not _newer(host_obj, [host_src] + headers):
        work.append(["g++", "-O2", "-std=c++17", "-fPIC", "-I" + os.path.join(CUDA, "include"),
                     "-c", host_src, "-o", host_obj])
    logs = []
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count()) as ex:
        for out in ex.map(_run, work):
            logs.append(out)
    if verbose:
        for s in logs:
            sys.stdout.write(s)
    if force or work or not os.path.exists(LIB):
        _run([NVCC] + ARCH + ["-shared", "-rdc=true", "-cudart", "static", "-Xcompiler", "-fPIC",
                              "-o", LIB] + objs + [host_obj, "-lpthread"])
    hc_src = os.path.join(CSRC, "hostcheck.cpp")
    if force or not _newer(HOSTCHECK, [hc_src, host_src] + headers):
        _run(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-I" + os.path.join(CUDA, "include"),
              "-o", HOSTCHECK, hc_src, host_src])
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.jobs, a.force, a.verbose))
