"""Builds the engine's shared library (sm_100a CUDA kernels + C ABI) in-tree.

    python -m matrix_format_performance_b200.build [--force] [--jobs N]

Outputs matrix_format_performance_b200/lib/libmfp_spmv.so.  Objects go to
matrix_format_performance_b200/_build/.  nvcc cross-compiles for sm_100a, so
this runs on a machine without a GPU.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libmfp_spmv.so"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["capi.cu", "convert.cu"]
CPP_SOURCES = ["util.cpp", "formats.cpp", "synth.cpp"]
HEADERS = ["spmv_device.cuh", "spmv_kernels.cuh", "spmv_stream.cuh", "spmv_lowp.cuh", "mlp.cuh", "host_common.h"]

NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-O3",
                     "--expt-relaxed-constexpr", f"-I{ROOT / 'include'}"]
CXX_FLAGS = ["-O3", "-fPIC", "-std=c++17", "-ffp-contract=off", "-Wall", "-Wextra",
             "-Wno-unused-parameter", f"-I{CUDA_HOME / 'include'}", f"-I{ROOT / 'include'}"]


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)


def build(force: bool = False, jobs: int | None = None, verbose: bool = False, defines: list[str] | None = None,
          out: Path | None = None, objdir: Path | None = None) -> Path:
    """Compiles and links the library; `defines` (e.g. ["MFP_CSR_MINBLOCKS=6"]) build a variant into `out`."""
    build_dir = objdir or BUILD
    lib = out or LIB
    build_dir.mkdir(parents=True, exist_ok=True)
    lib.parent.mkdir(parents=True, exist_ok=True)
    dflags = [f"-D{d}" for d in (defines or [])]
    headers = [CSRC / h for h in HEADERS] + [ROOT / "include" / "mfp_spmv.h"]
    tasks = []
    objs = []
    for src in CU_SOURCES:
        s = CSRC / src
        o = build_dir / (src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            tasks.append([NVCC] + NVCC_FLAGS + dflags + ["-c", str(s), "-o", str(o)])
    for src in CPP_SOURCES:
        s = CSRC / src
        o = build_dir / (src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            tasks.append(["g++"] + CXX_FLAGS + dflags + ["-c", str(s), "-o", str(o)])
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for f in [ex.submit(_run, t) for t in tasks]:
            f.result()
    if force or tasks or _stale(lib, objs):
        tmp = lib.with_suffix(".so.tmp")
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", str(tmp)] + [str(o) for o in objs]
             + ["-Xlinker", "--no-undefined", "-lpthread", "-ldl", "-lrt"])
        os.replace(tmp, lib)
    if verbose:
        print(f"built {lib}")
    return lib


HOST = PKG / "host"
DRIVER = LIBDIR / "mfp_driver"
HOST_HEADERS = ["matrix_market_reader.h", "matrix_converter.h", "scoo_matrix_class.h", "measurement_class.h",
                "resizable_gpu_memory.h", "gpu_matrix_multiplier.h", "cpu_matrix_multiplier.h",
                "cusparse_yardstick.h"]


def host_compile(src: Path, out: Path, extra: list[str] | None = None) -> Path:
    """Compiles a C++ program against the host layer (host/*.h) and libmfp_spmv.so."""
    out.parent.mkdir(parents=True, exist_ok=True)
    deps = [src, LIB] + [HOST / h for h in HOST_HEADERS] + [ROOT / "include" / "mfp_spmv.h"]
    if extra and "-lmfp_yardstick" in extra:
        deps.append(YARDSTICK)
    if _stale(out, deps):
        _run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Wno-unused-parameter", f"-I{ROOT / 'include'}",
              f"-I{HOST}", f"-I{CUDA_HOME / 'include'}", str(src), "-o", str(out), f"-L{LIBDIR}", "-lmfp_spmv"]
             + (extra or []) + [f"-L{CUDA_HOME / 'lib64'}", "-lcudart_static", "-ldl", "-lrt", "-lpthread",
                                f"-Wl,-rpath,{LIBDIR}"])
    return out


YARDSTICK = LIBDIR / "libmfp_yardstick.so"


def build_yardstick() -> Path:
    """cuSPARSE yardstick (csrc/yardstick.cpp) -> lib/libmfp_yardstick.so (library code beside the engine)."""
    src = CSRC / "yardstick.cpp"
    if _stale(YARDSTICK, [src, ROOT / "include" / "mfp_yardstick.h"]):
        tmp = YARDSTICK.with_suffix(".so.tmp")
        _run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall", f"-I{ROOT / 'include'}",
              f"-I{CUDA_HOME / 'include'}", str(src), "-o", str(tmp), f"-L{CUDA_HOME / 'lib64'}", "-lcusparse",
              "-lcudart_static", "-ldl", "-lrt", "-lpthread", f"-Wl,-rpath,{CUDA_HOME / 'lib64'}"])
        os.replace(tmp, YARDSTICK)
    return YARDSTICK


def build_driver() -> Path:
    """The main.cpp-style benchmark driver (host/main.cpp) -> lib/mfp_driver."""
    build_yardstick()
    return host_compile(HOST / "main.cpp", DRIVER, ["-lmfp_yardstick"])


def clean() -> None:
    shutil.rmtree(BUILD, ignore_errors=True)
    if LIB.exists():
        LIB.unlink()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--clean", action="store_true")
    a = ap.parse_args()
    if a.clean:
        clean()
        return
    build(force=a.force, jobs=a.jobs, verbose=True)
    print(f"built {build_driver()}")


if __name__ == "__main__":
    main()
