"""Builds libwbte.so (the sm_100a kernels and the C ABI of include/wbte.h).

    python -m weighted_bte_b200.build        # incremental
    python -m weighted_bte_b200.build --force

Each .cu under csrc/ is compiled in parallel with
`nvcc -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo` and linked
against the static CUDA runtime, so the library does not depend on which
libcudart another component of the process loads.
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libwbte.so")
SOURCES = ["k_arith.cu", "k_gt.cu", "k_hash.cu", "k_msm.cu", "k_opening.cu", "k_pairing.cu", "runtime.cu", "server.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", CSRC, "-I", INCLUDE]
# Code-layout variant of the shipped library (see fields.cuh): one out-of-line
# copy of the Fp and of the Fp2 product.  Measured on B200 (weighted_btx,
# B = 512): 2.5x the throughput of fully inlined arithmetic, whose hot loops
# overflow the instruction cache (ncu: "no instruction" stalls dominate).
DEFAULT_DEFINES: list = ["WBTE_FP_NOINLINE", "WBTE_FP2_NOINLINE"]
# Per-file exceptions: the pairing kernels (Fp6/Fp12 towers over inlined Fp2
# products calling the one out-of-line Fp product) measured 5-16 % faster with
# Fp2 inlined, while the curve kernels (MSM, transforms) are faster with it
# out of line.  Each .cu is its own translation unit with internal-linkage
# field functions, so the layouts do not mix.
SOURCE_UNDEFINES: dict = {"k_pairing.cu": ["WBTE_FP2_NOINLINE"]}
# Per-file additions: the GT transform kernels (k_gt.cu), bound by
# instruction fetch, keep the Fp2 product out of line and take the Fp sums
# out of line too (the batched truncated transform of 64 batches: 140 ->
# 124 ms; the same layout slows the Miller and final-exponentiation kernels).
# The fetch-bound tower kernels also take the Fp product as a rolled loop of
# rows (WBTE_FP_ROLLED rows per iteration: a third to a half of the code of
# the straight-line product for about 10 % more instructions).  Measured on
# B200 at 128 batches of B = 512 per group: the GT transform 246 -> 185 ms
# (4 rows), the opening multi-Miller loops 72.7 -> 65.4 ms (6 rows), the hard
# parts 47.3 -> 44.9 ms and the easy parts 13.8 -> 12.7 ms (4 rows); the curve
# kernels (MSMs, G1 transforms, fixed-base tables) measured 2-7 % slower and
# keep the straight-line product.
SOURCE_DEFINES: dict = {"k_gt.cu": ["WBTE_FPADD_NOINLINE", "WBTE_FP_ROLLED=4"],
                        "k_pairing.cu": ["WBTE_FP_ROLLED=4"],
                        "k_opening.cu": ["WBTE_FP_ROLLED=6"]}


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libwbte")
    return path


def _headers_digest() -> str:
    h = hashlib.sha256()
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cuh", ".h")):
            with open(os.path.join(CSRC, name), "rb") as f:
                h.update(name.encode() + f.read())
    with open(os.path.join(INCLUDE, "wbte.h"), "rb") as f:
        h.update(f.read())
    h.update(" ".join(ARCH + FLAGS).encode())
    return h.hexdigest()


def _flags_for(src: str) -> list:
    drop = {f"-D{d}" for d in SOURCE_UNDEFINES.get(src, [])}
    return [f for f in FLAGS if f not in drop] + [f"-D{d}" for d in SOURCE_DEFINES.get(src, [])]


def _compile(src: str, digest: str, force: bool) -> str:
    path = os.path.join(CSRC, src)
    flags = _flags_for(src)
    with open(path, "rb") as f:
        key = hashlib.sha256(f.read() + digest.encode() + " ".join(flags).encode()).hexdigest()[:16]
    obj = os.path.join(BUILD, f"{src[:-3]}.{key}.o")
    if os.path.exists(obj) and not force:
        return obj
    cmd = [nvcc()] + ARCH + flags + ["-c", path, "-o", obj + ".tmp"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stderr[-6000:]}")
    os.replace(obj + ".tmp", obj)
    return obj


def build(force: bool = False, verbose: bool = True, defines=None, lib_path: str = None) -> str:
    """Compile and link.  `defines` (e.g. ["WBTE_FP_NOINLINE"]) select code-layout
    variants; `lib_path` names the output (default: weighted_bte_b200/libwbte.so)."""
    global FLAGS, BUILD
    if not os.path.exists(os.path.join(CSRC, "field_asm.cuh")) or force:
        subprocess.run([sys.executable, os.path.join(CSRC, "gen_field.py")], check=True)
    defines = DEFAULT_DEFINES if defines is None else list(defines)
    lib = lib_path or LIB
    saved = (FLAGS, BUILD)
    FLAGS = FLAGS + [f"-D{d}" for d in defines]
    BUILD = os.path.join(PKG, "_build", "-".join(defines) or "base")
    try:
        os.makedirs(BUILD, exist_ok=True)
        digest = _headers_digest()
        with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
            objs = list(ex.map(lambda s: _compile(s, digest, force), SOURCES))
        stamp = hashlib.sha256(("".join(objs) + lib).encode()).hexdigest()
        stamp_file = os.path.join(BUILD, "link.stamp")
        if os.path.exists(lib) and os.path.exists(stamp_file) and not force:
            with open(stamp_file) as f:
                if f.read() == stamp:
                    return lib
        cmd = [nvcc()] + ARCH + ["-shared", "-o", lib + ".tmp"] + objs + ["-cudart", "static"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stderr[-6000:]}")
        os.replace(lib + ".tmp", lib)
        with open(stamp_file, "w") as f:
            f.write(stamp)
        # drop objects of older source versions
        keep = set(objs)
        for name in os.listdir(BUILD):
            p = os.path.join(BUILD, name)
            if name.endswith(".o") and p not in keep:
                os.remove(p)
    finally:
        FLAGS, BUILD = saved
    if verbose:
        print(f"built {lib}")
    return lib


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--define", action="append", default=None)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    build(force=a.force, defines=a.define, lib_path=a.out)
