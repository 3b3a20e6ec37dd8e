"""Build libpico_gpu.so in-tree with nvcc for sm_100a.

Each .cu under csrc/ compiles to an object in _build/ (in parallel), then the
objects link into pico_b200/libpico_gpu.so.  A stamp holding a hash of the
sources and flags skips the build when nothing changed.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libpico_gpu.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"] + ARCH + os.environ.get("PICO_NVCC_EXTRA", "").split()


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build pico_b200")
    return cand


def _host_cxx() -> list[str]:
    # The system g++ is the one nvcc is validated against here.
    if Path("/usr/bin/g++").exists():
        return ["-ccbin", "/usr/bin/g++"]
    return []


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _digest() -> str:
    h = hashlib.sha256()
    files = sorted(list(CSRC.glob("*")) + list(INCLUDE.glob("*.h")))
    for f in files:
        if f.is_file():
            h.update(f.name.encode())
            h.update(f.read_bytes())
    h.update(" ".join(NVCC_FLAGS).encode())
    return h.hexdigest()


def up_to_date() -> bool:
    stamp = BUILD / "stamp"
    return LIB.exists() and stamp.exists() and stamp.read_text() == _digest()


def build(verbose: bool = False, force: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    srcs = sources()

    def compile_one(src: Path) -> Path:
        obj = BUILD / (src.stem + ".o")
        cmd = [nvcc, *_host_cxx(), *NVCC_FLAGS, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stderr}")
        if verbose and r.stderr.strip():
            print(r.stderr, file=sys.stderr)
        return obj

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, srcs))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, *_host_cxx(), "-shared", *ARCH, "-o", str(tmp), *map(str, objs), "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    (BUILD / "stamp").write_text(_digest())
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
