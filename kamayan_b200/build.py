"""Build libkmy_hydro.so (CUDA, sm_100a) in-tree with nvcc.

Each translation unit under csrc/ compiles in parallel to an object in
_build/, then everything links into kamayan_b200/lib/libkmy_hydro.so.
"""
from __future__ import annotations

import os
import shlex
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libkmy_hydro.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr",
]


# Per-unit flags.  The FP32 fused stage uses approximate division/square root
# and flushes denormals: its results are checked against FP64 at an L1 of 1e-5,
# and the reciprocal/sqrt unit is its busiest pipe.
EXTRA_FLAGS = {
    "kmy_fused_f32.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    # same arithmetic as the single-mesh FP32 stage, so a solve gives the same
    # bits alone and inside a batch
    "kmy_batch_f32.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    # the z-streamed stage's FP32 instantiations (hydro and constrained
    # transport), and the device reconstruction functions as the FP32 stage
    # kernels compile them
    "kmy_slab_f32.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    "kmy_slab_mhd.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    # the streamed CT face update and cell pass: their FP32 instantiations
    # round as the FP32 stage kernels do (FP64 division is unaffected)
    "kmy_ct.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    "kmy_kat.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    # adaptive mesh: no FMA contraction, so prolongation, restriction and the
    # refinement estimator round exactly as written (tags are threshold tests)
    "kmy_amr.cu": ["-fmad=false"],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"


def user_flags() -> list[str]:
    """Extra nvcc flags for every unit from KMY_NVCC_FLAGS, for example
    "-DSLAB_F64_NR=0 -DKMY_F64_NR=0" (IEEE division and square root in the
    fused FP64 stages).  A change of these flags rebuilds every unit."""
    return shlex.split(os.environ.get("KMY_NVCC_FLAGS", ""))


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + [PKG.parent / "include" / "kmy_hydro.h"]
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def compile_one(src: Path, verbose_ptxas: bool = False, force: bool = False) -> Path:
    obj = BUILD / (src.stem + ".o")
    if not force and not _stale(obj, src) and not verbose_ptxas:
        return obj
    cmd = [nvcc(), "-ccbin", host_cxx(), *NVCC_FLAGS, *EXTRA_FLAGS.get(src.name, []), *user_flags(), "-c",
           str(src), "-o", str(obj)]
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    if verbose_ptxas:
        (BUILD / (src.stem + ".ptxas.txt")).write_text(r.stderr)
    return obj


def build(jobs: int | None = None, verbose_ptxas: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    srcs = sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    # the user flags the objects were built with; a change rebuilds them all
    stamp = BUILD / "user_flags.txt"
    flags = " ".join(user_flags())
    force = (stamp.read_text() if stamp.exists() else "") != flags
    with ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: compile_one(s, verbose_ptxas, force), srcs))
    stamp.write_text(flags)
    newest = max(o.stat().st_mtime for o in objs)
    if not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [nvcc(), "-ccbin", host_cxx(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a",
               "-cudart", "static", *map(str, objs), "-o", str(LIB)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="--ptxas" in sys.argv))
