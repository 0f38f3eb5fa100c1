"""Build recipe for the oracle -- TEST INFRASTRUCTURE ONLY.

Two things are built here, both outside the product:

* ``oracle/liboracle.so`` -- the plain-C restatement (fvb_oracle.c), compiled
  with ``-ffp-contract=off`` so each operation rounds once, as written.
* ``oracle/_ref/`` -- the reference solvers' own kernels, compiled from the
  files where they lie in the read-only reference checkout
  (``FVB_REFERENCE_DIR``; without it, a ``reference`` folder beside the
  checkout):

  - host builds (g++ + OpenMP) of the device functions and grid-stride
    kernels, taken by line range from the reference source and compiled
    through ``ref_shim.h`` (the launches and ``main`` cannot be compiled by
    g++, so those line ranges are left out);
  - GPU builds (nvcc, sm_100a) that ``#include`` the whole reference file
    with its ``main`` renamed;
  - for ``fv_up7_ducros_2d.cu``, both as shipped (FP32) and as a mechanical
    float->double retype (FP64), which is what the FP64 product path is
    held to.

  Everything generated goes to ``oracle/_ref/`` (git-ignored).  When the
  reference checkout is absent the prebuilt files there are used as they are.

* ``oracle/_ref/libref_host_up7_f64_native.so`` (``build_timing``) -- the
  same FP64 kernels built for speed on the machine that times them: the CPU
  baseline, not a checker.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
REF_DIR = Path(os.environ.get("FVB_REFERENCE_DIR", str(HERE.parent.parent / "reference")))

UP7 = "fv_up7_ducros_2d.cu"
KEEP = "keep_fv_euler_2d.cu"
# line ranges g++ can compile: constants, device helpers, grid kernels, IC.
# Left out: includes, the CK() error macro, the shared-memory reduction with
# its <<<>>> launches, image output and main.
UP7_HOST_LINES = [(26, 38), (48, 590), (614, 639)]
KEEP_HOST_LINES = [(46, 68), (78, 393), (441, 536)]
CARB = "carb_fv_2d.cu"
# GAMMA_V and the `real` switch, then sound_speed, hllc_n, hll_n and roe_n
CARB_HOST_LINES = [(36, 36), (40, 44), (60, 211)]
REC3 = "fv_rec3_2d.cu"
# constants and floors, then everything from IDX_P to the error kernel;
# left out: includes, the CK() macro, the reductions, host code and main
REC3_HOST_LINES = [(36, 60), (65, 447)]
BAK = "fv_up7_ducros_2d.cu.bak"
# GAMMA_V, IDX, then everything from the fetch helper to the RK3 kernels,
# and the IC kernel; left out: includes, CK(), the reductions, image output
# and main
BAK_HOST_LINES = [(27, 27), (43, 446), (469, 491)]

NVCC = os.environ.get("NVCC", "nvcc")
GPU_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed (%d): %s\n%s" % (r.returncode, " ".join(cmd), r.stdout))


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def retype_f64(text: str) -> str:
    """float -> double, single-precision math calls -> double ones, and the
    ``f`` suffix dropped from every floating literal."""
    text = re.sub(r"\bfloat\b", "double", text)
    for fn in ("sqrt", "fabs", "fmin", "fmax", "tanh", "exp", "log", "pow", "sin", "cos"):
        text = re.sub(r"\b%sf\(" % fn, fn + "(", text)
    text = re.sub(r"(?<![\w.])((?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?)f\b", r"\1", text)
    left = re.findall(r"(?<![\w.])(?:\d+\.\d*|\.\d+)(?:[eE][-+]?\d+)?f\b", text)
    if left:
        raise RuntimeError("retype left float literals: %r" % left[:5])
    return text


def _extract(src: Path, ranges: list[tuple[int, int]]) -> str:
    lines = src.read_text().splitlines()
    parts = []
    for a, b in ranges:
        parts.append("#line %d \"%s\"" % (a, src))
        parts.extend(lines[a - 1:b])
    return "\n".join(parts) + "\n"


def _write_if_changed(p: Path, text: str) -> None:
    if p.exists() and p.read_text() == text:
        return
    p.write_text(text)


def build_oracle(verbose: bool = False) -> Path:
    out = HERE / "liboracle.so"
    deps = [HERE / "fvb_oracle.c", HERE / "fvb_oracle_up7.h", HERE / "fvb_oracle_keep.h",
            HERE / "fvb_oracle_rec3.h", HERE / "fvb_oracle_d2av.h", HERE / "build.py"]
    if _stale(out, deps):
        _run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off",
              "-o", str(out), str(HERE / "fvb_oracle.c"), "-lm"])
        if verbose:
            print("built", out)
    return out


def build_ref(verbose: bool = False, gpu: bool = True) -> list[Path]:
    """Compile the reference kernels into oracle/_ref/ (host and GPU)."""
    up7, keep = REF_DIR / UP7, REF_DIR / KEEP
    if not (up7.exists() and keep.exists()):
        return []
    OUT.mkdir(exist_ok=True)
    up7_text = up7.read_text()
    _write_if_changed(OUT / "up7_host_f32.inc", _extract(up7, UP7_HOST_LINES))
    _write_if_changed(OUT / "up7_host_f64.inc", retype_f64(_extract(up7, UP7_HOST_LINES)))
    _write_if_changed(OUT / "keep_host.inc", _extract(keep, KEEP_HOST_LINES))
    carb = REF_DIR / CARB
    if carb.exists():
        _write_if_changed(OUT / "carb_host.inc", _extract(carb, CARB_HOST_LINES))
    rec3 = REF_DIR / REC3
    if rec3.exists():
        _write_if_changed(OUT / "rec3_host.inc", _extract(rec3, REC3_HOST_LINES))
    bak = REF_DIR / BAK
    if bak.exists():
        _write_if_changed(OUT / "bak_host.inc", _extract(bak, BAK_HOST_LINES))
    _write_if_changed(OUT / "fv_up7_f64.cu", retype_f64(up7_text))

    host_flags = ["g++", "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared",
                  "-ffp-contract=off", "-march=x86-64-v3", "-w", "-I", str(HERE)]
    host = [
        ("libref_host_up7_f32.so", ["-DREF_UP7", "-DREF_REAL=float", "-DREF_SFX=f32",
                                    '-DREF_INC="_ref/up7_host_f32.inc"'], OUT / "up7_host_f32.inc"),
        ("libref_host_up7_f64.so", ["-DREF_UP7", "-DREF_REAL=double", "-DREF_SFX=f64",
                                    '-DREF_INC="_ref/up7_host_f64.inc"'], OUT / "up7_host_f64.inc"),
        ("libref_host_keep.so", ["-DREF_KEEP", '-DREF_INC="_ref/keep_host.inc"'], OUT / "keep_host.inc"),
    ]
    if carb.exists():
        host.append(("libref_host_carb.so", ["-DREF_CARB", "-DUSE_DOUBLE", '-DREF_INC="_ref/carb_host.inc"'],
                     OUT / "carb_host.inc"))
    if rec3.exists():
        host.append(("libref_host_rec3.so", ["-DREF_REC3", "-Dreal=double", "-Dreall=double",
                                             '-DREF_INC="_ref/rec3_host.inc"'], OUT / "rec3_host.inc"))
    if bak.exists():
        host.append(("libref_host_bak.so", ["-DREF_BAK", '-DREF_INC="_ref/bak_host.inc"'], OUT / "bak_host.inc"))
    built = []
    for name, defs, inc in host:
        out = OUT / name
        if _stale(out, [inc, HERE / "ref_host.cpp", HERE / "ref_shim.h", HERE / "build.py"]):
            _run(host_flags + defs + ["-o", str(out), str(HERE / "ref_host.cpp")])
            if verbose:
                print("built", out)
        built.append(out)

    if gpu:
        gpu_flags = [NVCC, "-O3", "-std=c++17", *GPU_ARCH, "--expt-relaxed-constexpr",
                     "-Xcompiler", "-fPIC", "-shared", "-w", "-I", str(REF_DIR), "-I", str(HERE)]
        dev = [
            ("libref_gpu_up7_f32.so", ["-DREF_UP7", "-DREF_REAL=float", "-DREF_SFX=f32",
                                       '-DREF_CU="%s"' % up7], up7),
            ("libref_gpu_up7_f64.so", ["-DREF_UP7", "-DREF_REAL=double", "-DREF_SFX=f64",
                                       '-DREF_CU="_ref/fv_up7_f64.cu"'], OUT / "fv_up7_f64.cu"),
            ("libref_gpu_keep.so", ["-DREF_KEEP", '-DREF_CU="%s"' % keep], keep),
        ]
        if bak.exists():
            dev.append(("libref_gpu_bak.so", ["-DREF_BAK", '-DREF_CU="%s"' % bak], bak))
        if rec3.exists():
            dev.append(("libref_gpu_rec3.so", ["-DREF_REC3", "-Dreal=double", "-Dreall=double",
                                               '-DREF_CU="%s"' % rec3], rec3))
        for name, defs, src in dev:
            out = OUT / name
            if _stale(out, [src, HERE / "ref_gpu.cu", HERE / "build.py"]):
                _run(gpu_flags + defs + ["-o", str(out), str(HERE / "ref_gpu.cu")])
                if verbose:
                    print("built", out)
            built.append(out)
    return built


def _cpu_signature() -> str:
    """CPU model and feature flags of this machine, and the compiler version:
    a -march=native build is only valid where all three match."""
    model, flags = "", ""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if not model and line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
            if not flags and line.startswith("flags"):
                flags = " ".join(sorted(line.split(":", 1)[1].split()))
            if model and flags:
                break
    except OSError:
        pass
    cc = subprocess.run(["g++", "--version"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                        text=True).stdout.splitlines()
    return "%s\n%s\n%s\n" % (model, flags, cc[0] if cc else "")


TIMING_LIB = "libref_host_up7_f64_native.so"


def build_timing(verbose: bool = False) -> Path | None:
    """The CPU-baseline build of the reference kernels (FP64 retype of
    fv_up7_ducros_2d.cu): ``g++ -O3 -march=native -fopenmp`` with the
    compiler's default floating-point contraction, as a user would build it
    for speed.  The pin build above keeps ``-ffp-contract=off``, which this
    one must not inherit.  Built on the machine that times it (the extracted
    source in ``_ref/`` travels; the reference checkout need not), and
    rebuilt when the CPU or compiler differs from the one it was built on.
    Returns None when the extracted source is absent."""
    inc = OUT / "up7_host_f64.inc"
    if not inc.exists():
        return None
    out, sig_file = OUT / TIMING_LIB, OUT / (TIMING_LIB + ".cpu")
    sig = _cpu_signature()
    fresh = not _stale(out, [inc, HERE / "ref_host.cpp", HERE / "ref_shim.h", HERE / "build.py"])
    if fresh and sig_file.exists() and sig_file.read_text() == sig:
        return out
    _run(["g++", "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-march=native", "-w", "-I", str(HERE),
          "-DREF_UP7", "-DREF_REAL=double", "-DREF_SFX=f64", '-DREF_INC="_ref/up7_host_f64.inc"',
          "-o", str(out), str(HERE / "ref_host.cpp")])
    sig_file.write_text(sig)
    if verbose:
        print("built", out)
    return out


def build(verbose: bool = False, gpu: bool = True) -> None:
    build_oracle(verbose)
    build_ref(verbose, gpu)


if __name__ == "__main__":
    build(verbose=True, gpu="--no-gpu" not in sys.argv)
