"""Builds libgfk.so in-tree for sm_100a with nvcc (no GPU needed to compile)."""
import os
import pathlib
import shutil
import subprocess

PKG = pathlib.Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "_lib"
LIB = LIB_DIR / "libgfk.so"
SOURCES = ["gfk_kernels.cu", "gfk_quad_tc.cu", "gfk_host.cu", "gfk_noalloc.cu", "gfk_mlp.cu", "gfk_trace.cu",
           "gfk_surrogate.cu", "gfk_consume.cu", "gfk_disp.cu", "gfk_fdtd.cu"]
HEADERS = ["gfk_math.cuh", "gfk_solver.cuh", "gfk_kernels.cuh", "gfk_tc.cuh", "gfk_mlp.cuh", "gfk_ctx.h",
           "gfk_fft.cuh"]


def cutlass_include():
    """CuTe/CUTLASS headers (used for the UMMA descriptor bitfield definitions)."""
    import site
    cands = [os.environ.get("GFK_CUTLASS_INCLUDE")]
    for sp in site.getsitepackages() + [site.getusersitepackages()]:
        cands.append(os.path.join(sp, "flashinfer", "data", "cutlass", "include"))
    for c in cands:
        if c and pathlib.Path(c, "cute", "arch", "mma_sm100_desc.hpp").exists():
            return c
    raise RuntimeError("CuTe headers (cute/arch/mma_sm100_desc.hpp) not found; set GFK_CUTLASS_INCLUDE")


NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; libgfk needs the CUDA toolkit to build")


def stale():
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [PKG.parent / "include" / "gfk.h"]
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(force=False, verbose=False):
    """Compiles csrc/*.cu into _lib/libgfk.so; returns its path."""
    if not force and not stale():
        return LIB
    LIB_DIR.mkdir(exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *NVCC_FLAGS, "-I", cutlass_include(), "-o", str(tmp), *[str(CSRC / s) for s in SOURCES]]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
