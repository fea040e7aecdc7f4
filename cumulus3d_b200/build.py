"""Builds the native libraries in-tree.

* ``cumulus3d_b200/libpatchstereo.so`` — the engine: CUDA kernels for sm_100a (parity, fast and bounds-checked
  builds of the same source) + the host runtime and C ABI (include/patchstereo.h).  CUDA runtime linked statically;
  no PyTorch.
* ``cumulus3d_b200/libps_synth.so`` — the synthetic scene renderer (host code).
* ``oracle/_build/libps_oracle.so`` — the CPU oracle (test infrastructure), via oracle/Makefile.

Run ``python -m cumulus3d_b200.build`` (or ``__graft_entry__.build()``).  Nothing is compiled at import time.
"""
from __future__ import annotations

import os
import pathlib
import subprocess
import sys

ROOT = pathlib.Path(__file__).resolve().parent.parent
PKG = ROOT / "cumulus3d_b200"
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
ENGINE = PKG / "libpatchstereo.so"
SYNTH = PKG / "libps_synth.so"
ORACLE = ROOT / "oracle" / "_build" / "libps_oracle.so"

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I", str(CSRC), "-I", str(ROOT / "include")]
# Parity build: no contraction, IEEE division / square root, no flush-to-zero.
PARITY = ["--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false", "-DPS_FAST=0"]
FAST = ["--use_fast_math", "-DPS_FAST=1"]


def _newer(out: pathlib.Path, deps) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(pathlib.Path(d).stat().st_mtime > t for d in deps)


def _headers():
    return list(CSRC.glob("*.h")) + [ROOT / "include" / "patchstereo.h"]


def build_engine(force: bool = False, verbose: bool = False) -> pathlib.Path:
    OBJ.mkdir(exist_ok=True)
    hdr = _headers()
    jobs = []
    objs = []
    specs = [
        ("k_parity.o", CSRC / "ps_kernels.cu", PARITY),
        ("k_fast.o", CSRC / "ps_kernels.cu", FAST),
        ("k_checked.o", CSRC / "ps_kernels.cu", PARITY + ["-DPS_CHECKED=1"]),
        ("runtime.o", CSRC / "ps_runtime.cu", ["-Xcompiler", "-fopenmp"]),
        ("noalloc.o", CSRC / "ps_noalloc.cu", PARITY),
        ("cnn.o", CSRC / "ps_cnn.cu", []),
        ("post.o", CSRC / "ps_post.cu", PARITY),
        ("neighbors.o", CSRC / "ps_neighbors.cu", PARITY),
        ("io.o", CSRC / "ps_io.cpp", []),
    ]
    for name, src, flags in specs:
        out = OBJ / name
        objs.append(out)
        if force or _newer(out, [src] + hdr):
            cmd = [NVCC] + ARCH + COMMON + flags + ["-c", str(src), "-o", str(out)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    for cmd, p in jobs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed ({' '.join(cmd)}):\n{out}")
        if verbose and out:
            sys.stdout.write(out)
    if force or jobs or _newer(ENGINE, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", str(ENGINE)] + [str(o) for o in objs] + [
            "-Xcompiler", "-fopenmp", "-lgomp", "-cudart", "static"]
        subprocess.run(cmd, check=True)
    return ENGINE


def build_synth(force: bool = False) -> pathlib.Path:
    src = CSRC / "ps_synth.cpp"
    if force or _newer(SYNTH, [src]):
        subprocess.run(["g++", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared",
                        "-std=c++17", str(src), "-o", str(SYNTH)], check=True)
    return SYNTH


def build_oracle(force: bool = False) -> pathlib.Path:
    args = ["make", "-s", "-C", str(ROOT / "oracle")]
    if force:
        args.append("-B")
    subprocess.run(args, check=True)
    return ORACLE


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_synth(force)
    build_oracle(force)
    build_engine(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print("built:", ENGINE, SYNTH, ORACLE)
