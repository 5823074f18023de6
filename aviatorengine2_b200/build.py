"""Build the library: nvcc for sm_100a, the host scene code with g++.

Produces aviatorengine2_b200/libae_b200.so in the source tree (the built .so
travels with the tree; nothing is installed).  Usage:

    python -m aviatorengine2_b200.build [--force]
"""
import hashlib
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libae_b200.so")
BUILD = os.path.join(HERE, "_build")
ROOT = os.path.dirname(HERE)

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
                  "-Xptxas", "-O3", "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]
CXXFLAGS = ["-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", "-I" + os.path.join(ROOT, "include")]


def _sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    hdr = sorted(f for f in os.listdir(CSRC) if f.endswith((".h", ".cuh")))
    return cu, cpp, hdr


def _digest(files):
    h = hashlib.sha256()
    for f in files:
        with open(f, "rb") as fh:
            h.update(f.encode() + fh.read())
    h.update(" ".join(NVFLAGS + CXXFLAGS).encode())
    return h.hexdigest()


def build(force=False, verbose=False):
    cu, cpp, hdr = _sources()
    files = [os.path.join(CSRC, f) for f in cu + cpp + hdr] + [os.path.join(ROOT, "include", "ae_b200.h")]
    digest = _digest(files)
    stamp = OUT + ".sha256"
    if not force and os.path.exists(OUT) and os.path.exists(stamp) and open(stamp).read() == digest:
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    jobs = [([NVCC] + NVFLAGS + ["-c", os.path.join(CSRC, f), "-o", os.path.join(BUILD, f + ".o")]) for f in cu]
    jobs += [(["g++"] + CXXFLAGS + ["-c", os.path.join(CSRC, f), "-o", os.path.join(BUILD, f + ".o")]) for f in cpp]
    objs = [cmd[-1] for cmd in jobs]

    def run(cmd):
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)

    # One compiler process per source file, as many at a time as there are
    # cores; the first failure is raised.
    with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as pool:
        for fut in [pool.submit(run, cmd) for cmd in jobs]:
            fut.result()
    tmp = OUT + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-cudart=static", "-lpthread"]
    subprocess.check_call(cmd)
    os.replace(tmp, OUT)
    with open(stamp, "w") as fh:
        fh.write(digest)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
