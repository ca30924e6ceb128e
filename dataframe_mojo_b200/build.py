"""Build of the native parts, in tree.

``python -m dataframe_mojo_b200.build`` compiles ``csrc/*.cu`` for sm_100a into
``dataframe_mojo_b200/libdfcuda.so`` (the provider library) and the test-only
CPU oracle ``oracle/oracle.cpp`` into ``oracle/_build/liboracle.so``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libdfcuda.so"
ORACLE_SRC = ROOT / "oracle" / "oracle.cpp"
ORACLE_LIB = ROOT / "oracle" / "_build" / "liboracle.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC,-fvisibility=hidden,-O3",
    f"-I{ROOT / 'include'}",
]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libdfcuda.so")
    return path


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"command failed ({proc.returncode}): {' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def build_library(force: bool = False) -> Path:
    sources = sorted(CSRC.glob("*.cu"))
    headers = sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "dfcuda.h"]
    if not force and not _stale(LIB, sources + headers):
        return LIB
    BUILD.mkdir(exist_ok=True)
    compiler = nvcc()
    objects = [BUILD / (s.stem + ".o") for s in sources]
    with ThreadPoolExecutor(max_workers=len(sources)) as pool:
        list(pool.map(lambda so: _run([compiler, *NVCC_FLAGS, "-c", str(so[0]), "-o", str(so[1])]),
                      zip(sources, objects)))
    tmp = LIB.with_suffix(".so.tmp")
    _run([compiler, *ARCH, "-shared", "-o", str(tmp), *map(str, objects)])
    os.replace(tmp, LIB)
    return LIB


def build_oracle(force: bool = False) -> Path:
    deps = [ORACLE_SRC, ROOT / "oracle" / "oracle.h", ROOT / "include" / "dfcuda.h"]
    if not force and not _stale(ORACLE_LIB, deps):
        return ORACLE_LIB
    ORACLE_LIB.parent.mkdir(parents=True, exist_ok=True)
    cxx = shutil.which("g++") or "g++"
    tmp = ORACLE_LIB.with_suffix(".so.tmp")
    _run([cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-pthread", "-o", str(tmp), str(ORACLE_SRC)])
    os.replace(tmp, ORACLE_LIB)
    return ORACLE_LIB


def main(argv: list[str]) -> int:
    force = "--force" in argv
    print(build_library(force))
    print(build_oracle(force))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
