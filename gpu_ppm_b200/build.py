"""Builds libppm_b200.so for sm_100a with nvcc (in-tree, gpu_ppm_b200/_build/)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libppm_b200.so")
RUN = os.path.join(OUT_DIR, "ppm_run")

SOURCES = ["kernels.cu", "fold_tc.cu", "engine.cu", "noalloc.cu", "fit.cu", "capi.cpp", "serve.cpp", "lensgen.cpp",
           "response.cpp", "util.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "ppm.h"), __file__]
    return not os.path.exists(RUN) or any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not _needs_build():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    objs = []
    procs = []
    for src in SOURCES:
        obj = os.path.join(OUT_DIR, src + ".o")
        cmd = [NVCC, "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O2", *ARCH, "-Xptxas", "-v" if verbose else "-O3",
               "-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cpp"):
            cmd.insert(1, "-x")
            cmd.insert(2, "cu")
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or (verbose and out):
            sys.stderr.write(f"--- {src}\n{out}\n")
        failed |= p.returncode != 0
    if failed:
        raise RuntimeError("nvcc failed")
    tmp = LIB + f".{os.getpid()}.tmp"
    subprocess.run([NVCC, "-shared", *ARCH, "-o", tmp, *objs, "-lpthread"], check=True)
    os.replace(tmp, LIB)
    # the drop-in driver links the library from its own directory
    subprocess.run(["g++", "-std=c++17", "-O2", os.path.join(CSRC, "ppm_run.cpp"), "-o", RUN + ".tmp",
                    f"-L{OUT_DIR}", "-lppm_b200", "-Wl,-rpath,$ORIGIN"], check=True)
    os.replace(RUN + ".tmp", RUN)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
