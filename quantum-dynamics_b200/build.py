"""Build libqd.so (all CUDA kernels + the C ABI) in-tree for sm_100a.

    python quantum-dynamics_b200/build.py [--force]

Output: quantum-dynamics_b200/lib/libqd.so.  Each .cu is compiled with nvcc
for sm_100a only; the object files are linked into one shared library with
the CUDA runtime linked statically.  Also lib/libqd_libcmp.so from
compare/qd_libcmp.cu: the same passes on cuFFT and cuBLAS, which only the
benchmark's library comparison loads (the propagator never links them); and
bin/qd_run from cli/qd_run.cpp, the run-file driver over the C ABI.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libqd.so")
RUN_SRC = os.path.join(HERE, "cli", "qd_run.cpp")
RUN_BIN = os.path.join(HERE, "bin", "qd_run")
CMP_SRC = os.path.join(HERE, "compare", "qd_libcmp.cu")
CMP_LIB = os.path.join(HERE, "lib", "libqd_libcmp.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr", f"-I{os.path.join(REPO, 'include')}", f"-I{CSRC}"]


def _newer(src_list, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list)


def build(force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        [os.path.join(REPO, "include", "qd.h")]
    objs = []
    procs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or _newer([src] + headers, obj):
            cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                                stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if out and (verbose or p.returncode):
            sys.stdout.write(out.decode())
        if p.returncode:
            failed.append(src)
    if failed:
        raise RuntimeError("nvcc failed for: " + ", ".join(failed))
    if force or procs or _newer(objs, LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcuda"]
        subprocess.run(cmd, check=True)
    if force or _newer([RUN_SRC, LIB, os.path.join(REPO, "include", "qd.h")], RUN_BIN):
        os.makedirs(os.path.dirname(RUN_BIN), exist_ok=True)
        cmd = ["g++", "-O2", "-std=c++17", "-Wall", f"-I{os.path.join(REPO, 'include')}",
               RUN_SRC, "-o", RUN_BIN, f"-L{os.path.dirname(LIB)}", "-lqd",
               "-Wl,-rpath,$ORIGIN/../lib"]
        subprocess.run(cmd, check=True)
    if force or _newer([CMP_SRC], CMP_LIB):
        cmd = [NVCC] + ARCH + FLAGS + ["-shared", CMP_SRC, "-o", CMP_LIB, "-lcufft", "-lcublas"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
