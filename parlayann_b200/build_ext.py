"""Compile libparlayann_b200.so in-tree for sm_100a (B200) with nvcc."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
SOURCES = ["capi.cu", "build.cu", "bruteforce.cu", "batch.cu", "tile.cu", "range.cu", "noalloc.cu", "quant.cu", "score.cu", "order.cu", "synth.cpp", "serve.cpp"]
OUT = os.path.join(HERE, "libparlayann_b200.so")
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-O3", "-shared",
]


OBJDIR = os.path.join(HERE, "_build")


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(HERE, "..", "include", "parlayann_b200.h"))
    return [h for h in hs if os.path.exists(h)]


def _stale(src: str, obj: str, newest_header: float) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(os.path.join(CSRC, src)) > t or newest_header > t


def needs_rebuild() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "parlayann_b200.h"))
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the sources whose object is missing or older than the source or
    any header (one nvcc per file, in parallel) into _build/, then link."""
    if not force and not needs_rebuild():
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]
    os.makedirs(OBJDIR, exist_ok=True)
    newest = max((os.path.getmtime(h) for h in _headers()), default=0.0)
    objs, procs = [], []
    for src in SOURCES:
        obj = os.path.join(OBJDIR, src + ".o")
        objs.append(obj)
        if not force and not _stale(src, obj, newest):
            continue
        cmd = [nvcc, *compile_flags, "-c", os.path.join(CSRC, src), "-o", obj + ".tmp"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((src, obj, subprocess.Popen(cmd, cwd=CSRC, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for src, obj, pr in procs:
        out, _ = pr.communicate()
        if pr.returncode != 0:
            failed.append(src)
            sys.stderr.write(out.decode(errors="replace"))
        else:
            os.replace(obj + ".tmp", obj)
    if failed:
        raise subprocess.CalledProcessError(1, "nvcc " + " ".join(failed))
    link = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objs, "-o", OUT + ".tmp"]
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.run(link, check=True, cwd=CSRC)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
