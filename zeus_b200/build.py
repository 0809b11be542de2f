"""Builds zeus_b200/libzeus_b200.so (sm_100a) in-tree with nvcc.

Each translation unit compiles in parallel; an object is rebuilt only when
it is older than any source or header under csrc/ or include/.  The
exact-mode unit is compiled with -fmad=false (no multiply-add contraction).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
INCLUDE = ROOT / "include"
BUILD = HERE / "_build"
LIB = HERE / "libzeus_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = [
    "-std=c++20",
    "--expt-relaxed-constexpr",
    "-O3",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC",
    "-I",
    str(INCLUDE),
    "-I",
    str(CSRC),
] + ARCH

# (source, extra flags)
UNITS = [
    ("zb_exact.cu", ["-fmad=false"]),
    ("zb_fast.cu", []),
    ("zb_fast_thread.cu", []),
    ("zb_fast_tile.cu", []),
    ("zb_fast_cta.cu", []),
    ("zb_batch.cu", []),
    ("zb_batch_512.cu", []),
    ("zb_batch_384.cu", []),
    ("zb_noalloc.cu", ["-fmad=false"]),
    ("zb_fit.cu", []),
    ("zb_grad.cu", []),
    ("zb_plan.cu", []),
    ("zb_traj.cu", []),
    ("zb_sobol.cu", []),
    ("zb_runtime.cu", []),
]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build")
    return exe


def _deps_mtime() -> float:
    files = list(CSRC.glob("*")) + list(INCLUDE.glob("*.h")) + [Path(__file__)]
    return max(f.stat().st_mtime for f in files if f.is_file())


def _compile(src: str, extra: list[str], newest: float, verbose: bool) -> Path:
    obj = BUILD / (Path(src).stem + ".o")
    if obj.exists() and obj.stat().st_mtime >= newest:
        return obj
    cmd = [nvcc(), *COMMON, *extra, "-c", str(CSRC / src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    newest = _deps_mtime()
    with cf.ThreadPoolExecutor(max_workers=jobs or len(UNITS)) as ex:
        objs = list(ex.map(lambda u: _compile(u[0], u[1], newest, verbose), UNITS))
    if LIB.exists() and LIB.stat().st_mtime >= max(o.stat().st_mtime for o in objs):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), "-shared", *ARCH, "-o", str(tmp), *map(str, objs)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


BIN = HERE / "_bin"
DROPIN_SRC = ROOT / "tests" / "cpp" / "dropin_test.cu"
DROPIN_BIN = BIN / "dropin_test"


def build_dropin_test(verbose: bool = False) -> Path:
    """Compiles the C++ drop-in test program against libzeus_b200.so."""
    lib = build(verbose)
    BIN.mkdir(exist_ok=True)
    deps = [DROPIN_SRC, INCLUDE / "zeus.cuh", lib] + list(CSRC.glob("*.cuh"))
    if DROPIN_BIN.exists() and DROPIN_BIN.stat().st_mtime >= max(
            d.stat().st_mtime for d in deps):
        return DROPIN_BIN
    cmd = [nvcc(), *COMMON, str(DROPIN_SRC), "-o", str(DROPIN_BIN), "-L", str(HERE),
           "-lzeus_b200", "-Xlinker", "-rpath,$ORIGIN/.."]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"drop-in test build failed:\n{r.stdout}\n{r.stderr}")
    return DROPIN_BIN


REF_EXAMPLES_BIN = BIN / "ref_examples"
# programs built from the reference's examples, unchanged, against include/:
# name -> (sources relative to the reference's examples/ directory, or to
# this repository for the repo's own driver)
REF_PROGRAMS = {
    "optimize_rosenbrock": ["optimize_rosenbrock.cu", "optimization_utils.cc"],
    "optimize_rastrigin": ["optimize_rastrigin.cu", "optimization_utils.cc"],
    "optimize_ackley": ["optimize_ackley.cu", "optimization_utils.cc"],
    "fit_dijet_spectrum": ["fit_dijet_spectrum.cu"],
    "ref_objectives_test": [ROOT / "tests" / "cpp" / "ref_objectives_test.cu"],
}


def _ref_tree(reference_dir: Path) -> Path:
    """A build tree in which the reference's example sources sit beside this
    library's include/ in place of the reference's own:
    <tree>/examples/<file> are links to the reference's example files, and
    <tree>/include links to include/, so a relative include such as
    "../include/traits.hpp" (optimization_utils.hpp:4) reaches this
    library's header.  Only links are made; no source is copied."""
    tree = BUILD / "ref_examples"
    ex = tree / "examples"
    (ex / "simulation" / "fitting").mkdir(parents=True, exist_ok=True)
    src = Path(reference_dir) / "examples"
    files = [f for f in src.iterdir() if f.is_file()]
    files.append(src / "simulation" / "fitting" / "LogLikelihood.h")
    for f in files:
        link = ex / f.relative_to(src)
        if link.is_symlink() and link.resolve() == f.resolve():
            continue
        if link.is_symlink() or link.exists():
            link.unlink()
        link.symlink_to(f)
    inc = tree / "include"
    if not inc.is_symlink():
        inc.symlink_to(INCLUDE)
    return tree


def build_reference_examples(reference_dir, verbose: bool = False) -> list[Path]:
    """Compiles the reference's example programs (optimize_rosenbrock.cu,
    optimize_rastrigin.cu, optimize_ackley.cu with optimization_utils.cc,
    fit_dijet_spectrum.cu) and tests/cpp/ref_objectives_test.cu (which
    includes the reference's gaussian.hpp and LogLikelihood.h) against this
    library's include/ and libzeus_b200.so, into zeus_b200/_bin/ref_examples/.
    The reference's sources are compiled where they lie, unmodified."""
    lib = build(verbose)
    tree = _ref_tree(Path(reference_dir))
    REF_EXAMPLES_BIN.mkdir(parents=True, exist_ok=True)
    headers = [INCLUDE / h for h in ("zeus.cuh", "duals.cuh", "matrix.hpp", "traits.hpp")]
    deps_common = headers + [lib] + list(CSRC.glob("*.cuh"))

    def one(item):
        name, srcs = item
        paths = [s if isinstance(s, Path) else tree / "examples" / s for s in srcs]
        out = REF_EXAMPLES_BIN / name
        newest = max(p.stat().st_mtime for p in deps_common + [q.resolve() for q in paths])
        if out.exists() and out.stat().st_mtime >= newest:
            return out
        cmd = [nvcc(), *COMMON, "-I", str(tree / "examples"), *map(str, paths), "-o",
               str(out), "-L", str(HERE), "-lzeus_b200", "-Xlinker",
               "-rpath,$ORIGIN/../.."]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"{name}: build against include/ failed:\n{r.stdout}\n"
                               f"{r.stderr}")
        return out

    with cf.ThreadPoolExecutor(max_workers=len(REF_PROGRAMS)) as ex:
        return list(ex.map(one, REF_PROGRAMS.items()))


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
