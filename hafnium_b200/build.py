"""Build ``libhfjk.so`` (the C ABI of include/hfjk.h) for sm_100a with nvcc.

    python -m hafnium_b200.build [--force]

Each ``csrc/*.cu`` compiles to an object in parallel; the objects link into
``hafnium_b200/_build/libhfjk.so``, which the Python layer loads by path. A
source newer than the library triggers a rebuild.
"""

from __future__ import annotations

import concurrent.futures
import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT_DIR = HERE / "_build"
LIBRARY = OUT_DIR / "libhfjk.so"
INCLUDE = HERE.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-Xcompiler", "-Wshadow=local", f"-I{INCLUDE}"]


def nvcc() -> str:
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not pathlib.Path(found).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libhfjk.so")
    return found


def _host_compiler_args() -> list[str]:
    # The system g++ carries the OpenMP/runtime spec files the wrapper in $CXX may lack.
    gxx = "/usr/bin/g++"
    return ["-ccbin", gxx] if pathlib.Path(gxx).exists() else []


def sources() -> list[pathlib.Path]:
    return sorted(CSRC.glob("*.cu"))


def needs_build() -> bool:
    if not LIBRARY.exists():
        return True
    stamp = LIBRARY.stat().st_mtime
    deps = sources() + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))
    return any(p.stat().st_mtime > stamp for p in deps)


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    if not force and not needs_build():
        return LIBRARY
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    compiler = nvcc()
    host = _host_compiler_args()

    def compile_one(src: pathlib.Path) -> pathlib.Path:
        obj = OUT_DIR / (src.stem + ".o")
        cmd = [compiler, *host, *ARCH, *FLAGS, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stderr}")
        return obj

    workers = max(1, min(len(sources()), os.cpu_count() or 1))
    with concurrent.futures.ThreadPoolExecutor(workers) as pool:
        objects = list(pool.map(compile_one, sources()))
    tmp = LIBRARY.with_suffix(".so.tmp")
    cmd = [compiler, *host, *ARCH, "-shared", "-o", str(tmp), *map(str, objects), "-lcudart"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stderr}")
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
