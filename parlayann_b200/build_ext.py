"""Compile libparlayann_b200.so in-tree for sm_100a (B200) with nvcc."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
SOURCES = ["capi.cu", "build.cu", "bruteforce.cu", "batch.cu", "tile.cu", "range.cu", "noalloc.cu", "quant.cu", "synth.cpp", "serve.cpp"]
OUT = os.path.join(HERE, "libparlayann_b200.so")
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-O3", "-shared",
]


def needs_rebuild() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "parlayann_b200.h"))
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every source to an object in parallel (one nvcc per file), then link."""
    if not force and not needs_rebuild():
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]
    objdir = tempfile.mkdtemp(prefix="pann_build_")
    try:
        objs, procs = [], []
        for src in SOURCES:
            obj = os.path.join(objdir, src + ".o")
            cmd = [nvcc, *compile_flags, "-c", os.path.join(CSRC, src), "-o", obj]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            procs.append((src, subprocess.Popen(cmd, cwd=CSRC, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
            objs.append(obj)
        failed = []
        for src, pr in procs:
            out, _ = pr.communicate()
            if pr.returncode != 0:
                failed.append(src)
                sys.stderr.write(out.decode(errors="replace"))
        if failed:
            raise subprocess.CalledProcessError(1, "nvcc " + " ".join(failed))
        link = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objs, "-o", OUT + ".tmp"]
        if verbose:
            print(" ".join(link), file=sys.stderr)
        subprocess.run(link, check=True, cwd=CSRC)
    finally:
        shutil.rmtree(objdir, ignore_errors=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
