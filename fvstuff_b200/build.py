"""Build libfvb.so (and the command-line drivers) for sm_100a, in-tree.

Every CUDA/C++ source under fvstuff_b200/csrc is compiled with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` and linked into
``fvstuff_b200/libfvb.so``; the drivers in ``csrc/cli`` become
``fvstuff_b200/bin/*``.  Rebuilds only what is older than its sources.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
ROOT = PKG.parent
BUILD = PKG / "_build"
LIB = PKG / "libfvb.so"
BIN = PKG / "bin"

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "-I", str(ROOT / "include"), "-I", str(CSRC), "--expt-relaxed-constexpr"]


# per-file flags: the rec3 and D2-viscosity kernels reproduce the
# reference's arithmetic operation for operation, so no multiply-add
# contraction there
FILE_FLAGS = {"fvb_rec3.cu": ["-fmad=false"], "fvb_d2av.cu": ["-fmad=false"],
              # the FP32-compensated kernel: single-precision denormals flushed
              # to zero, so its reciprocals and square roots are the bare
              # hardware approximations without the denormal-range fix-ups
              # (its states, fluxes and increments are normal numbers)
              "fvb_stage32c.cu": ["-ftz=true"]}


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed (%d): %s\n%s" % (r.returncode, " ".join(map(str, cmd)), r.stdout))
    return r.stdout


def _sources():
    return sorted(p for p in CSRC.iterdir() if p.suffix in (".cu", ".cpp"))


def _headers():
    hs = [p for p in CSRC.iterdir() if p.suffix in (".h", ".cuh")]
    hs.append(ROOT / "include" / "fvb.h")
    return hs


def _newest(paths):
    return max((p.stat().st_mtime for p in paths if p.exists()), default=0.0)


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    hdr_t = max(_newest(_headers()), Path(__file__).stat().st_mtime)
    todo = []
    objs = []
    for src in _sources():
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr_t):
            todo.append((src, obj))

    def compile_one(item):
        src, obj = item
        lang = [] if src.suffix == ".cu" else ["-x", "cu"]
        _run([NVCC, *FLAGS, *ARCH, *lang, *FILE_FLAGS.get(src.name, []), "-c", str(src), "-o", str(obj)])
        return src.name

    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 4)) as ex:
            for name in ex.map(compile_one, todo):
                if verbose:
                    print("compiled", name)
    if todo or not LIB.exists() or LIB.stat().st_mtime < _newest(objs):
        # public C-ABI symbols are marked visible in the sources; everything
        # else stays hidden
        # linked under a temporary name and renamed, so a reader never sees
        # a partly written library
        tmp = LIB.with_name(LIB.name + ".tmp")
        _run([NVCC, *ARCH, "-shared", "-o", str(tmp), *map(str, objs)])
        os.replace(tmp, LIB)
        if verbose:
            print("linked", LIB)
    _build_cli(verbose)
    return LIB


def _build_cli(verbose: bool) -> None:
    cli = CSRC / "cli"
    if not cli.is_dir():
        return
    BIN.mkdir(exist_ok=True)
    for src in sorted(cli.glob("*.cpp")):
        exe = BIN / src.stem
        deps = [src, LIB, *cli.glob("*.h")]
        if exe.exists() and exe.stat().st_mtime >= _newest(deps):
            continue
        tmp = exe.with_name(exe.name + ".tmp")
        _run(["g++", "-O2", "-std=c++17", "-I", str(ROOT / "include"), "-I", str(cli), str(src),
              "-o", str(tmp), "-L", str(PKG), "-lfvb", "-Wl,-rpath,$ORIGIN/.."])
        os.replace(tmp, exe)
        if verbose:
            print("built", exe)


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
