"""Build libaxj.so in-tree for sm_100a (nvcc cross-compiles; no GPU needed).

    python -m axisymmetricjet_b200.build [--force]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libaxj.so")
SOURCES = ["axj_api.cu", "axj_kernels.cu", "axj_mlp.cu", "axj_noalloc.cu", "axj_prep.cu"]
HEADERS = ["axj_common.cuh", "axj_point.cuh", "axj_pow.cuh", "axj_kernels.cuh", "axj_mlp.cuh", "axj_prep.cuh"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-Xcompiler",
              "-fPIC", "-shared", "-cudart", "static"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "axj.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    """Compile every source to an object in parallel (they share no device symbols),
    then link the shared library with the static CUDA runtime."""
    if not force and not stale():
        return OUT
    from concurrent.futures import ThreadPoolExecutor
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    comp = [f for f in NVCC_FLAGS if f not in ("-shared", "-cudart", "static")]
    jobs = []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        jobs.append((obj, [nvcc()] + comp + ["-c", "-o", obj, os.path.join(CSRC, src)]))
    if verbose:
        for _, cmd in jobs:
            print(" ".join(cmd))
    with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
        procs = list(ex.map(lambda c: subprocess.run(c, cwd=CSRC, capture_output=True, text=True),
                            [cmd for _, cmd in jobs]))
    for (obj, cmd), pr in zip(jobs, procs):
        if pr.returncode != 0:
            sys.stderr.write(pr.stdout + pr.stderr)
            raise subprocess.CalledProcessError(pr.returncode, cmd)
    link = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-cudart", "static", "-o", OUT]
    link += [obj for obj, _ in jobs]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True, cwd=CSRC)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(OUT)
