"""Builds liblsp.so (all CUDA kernels, the engine and the C ABI) in-tree for sm_100a.

    python -m liquidsimulation_b200.build [--force] [--verbose]

nvcc cross-compiles without a GPU. Every translation unit is compiled with
-fmad=false -prec-div=true -prec-sqrt=true -ftz=false (device) and
-ffp-contract=off (host), so each floating-point operation rounds exactly once,
as in the reference CPU solver; the bit-exact parity tests rely on that.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(ROOT, "_build")
OUT = os.path.join(PKG, "liblsp.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise FileNotFoundError("nvcc not found")


def _host_cc() -> list:
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def flags() -> list:
    return (ARCH + _host_cc() + [
        "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
        "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
        "-Xcompiler", "-fPIC,-O3,-ffp-contract=off,-fno-fast-math",
        "-I" + os.path.join(ROOT, "include"),
    ])


def sources() -> list:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _digest(paths, extra) -> str:
    h = hashlib.sha256()
    for p in paths:
        with open(p, "rb") as f:
            h.update(p.encode())
            h.update(f.read())
    h.update(" ".join(extra).encode())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False) -> str:
    nvcc = _nvcc()
    srcs = sources()
    headers = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh")))
    headers.append(os.path.join(ROOT, "include", "lsp.h"))
    f = flags()
    stamp = os.path.join(BUILD, "liblsp.stamp")
    digest = _digest(srcs + headers, f)
    if not force and os.path.exists(OUT) and os.path.exists(stamp) and open(stamp).read() == digest:
        return OUT
    os.makedirs(BUILD, exist_ok=True)

    def compile_one(src):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        cmd = [nvcc, *f, "-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd.insert(1 + len(ARCH) + len(_host_cc()), "-x")
            cmd.insert(2 + len(ARCH) + len(_host_cc()), "cu")
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr:
            print(r.stderr)
        return obj

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, srcs))
    tmp = OUT + ".tmp"
    cmd = [nvcc, *ARCH, *_host_cc(), "-shared", "-o", tmp, *objs, "-lcudart_static", "-lrt", "-lpthread", "-ldl"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, OUT)
    with open(stamp, "w") as fh:
        fh.write(digest)
    return OUT


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    sys.exit(main())
