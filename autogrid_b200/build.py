"""Build the native library and command-line tool in-tree.

    python -m autogrid_b200.build        # or autogrid_b200.build.build()

Outputs (git-ignored, they travel with the source tree):
    autogrid_b200/_build/libautogrid_b200.so   C ABI of include/autogrid_b200.h
    autogrid_b200/_build/autogrid4_b200        drop-in for `autogrid4 -p x.gpf -l x.glg`

CUDA code is compiled for sm_100a only (-gencode arch=compute_100a,code=sm_100a).
"""
from __future__ import annotations

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
LIB = BUILD / "libautogrid_b200.so"
CLI = BUILD / "autogrid4_b200"

CXX_SOURCES = [CSRC / "host" / "params.cpp", CSRC / "host" / "job.cpp"]
CU_SOURCES = [CSRC / "capi.cu", CSRC / "kernels" / "emap.cu", CSRC / "kernels" / "near.cu",
              CSRC / "kernels" / "diag.cu", CSRC / "kernels" / "noalloc.cu", CSRC / "diff_api.cu",
              CSRC / "kernels" / "diff_emap.cu", CSRC / "kernels" / "diff_near.cu", CSRC / "kernels" / "distmap.cu",
              CSRC / "kernels" / "maptext.cu", CSRC / "kernels" / "diff_atoms.cu",
              CSRC / "kernels" / "tables.cu"]
CLI_SOURCES = [CSRC / "host" / "cli.cpp"]
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build autogrid_b200")
    return cand


def _deps() -> list[Path]:
    out = []
    for d in (CSRC, ROOT / "include"):
        for p in d.rglob("*"):
            if p.suffix in {".h", ".hpp", ".cuh", ".cu", ".cpp"}:
                out.append(p)
    return out


def _stale(target: Path) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(p.stat().st_mtime > t for p in _deps() + [Path(__file__)])


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compile every source for sm_100a; returns the library path."""
    if not force and not _stale(LIB) and not _stale(CLI):
        return LIB
    BUILD.mkdir(parents=True, exist_ok=True)
    nvcc = _nvcc()
    inc = ["-I", str(ROOT / "include"), "-I", str(CSRC)]
    jobs = []
    for src in CXX_SOURCES:
        obj = BUILD / (src.stem + ".o")
        jobs.append(["g++", "-std=c++17", "-O2", "-fPIC", "-Wall", "-Wno-unused-result", *inc,
                     "-c", str(src), "-o", str(obj)])
    for src in CU_SOURCES:
        obj = BUILD / (src.stem + ".cu.o")
        jobs.append([nvcc, "-ccbin", "g++", *GENCODE, "-lineinfo", "-O3", "-std=c++17",
                     "-Xcompiler", "-fPIC", "-Xptxas", "-warn-spills", *inc, "-c", str(src), "-o", str(obj)])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        for f in [ex.submit(_run, j) for j in jobs]:
            f.result()
    objs = [str(BUILD / (s.stem + ".o")) for s in CXX_SOURCES] + [str(BUILD / (s.stem + ".cu.o")) for s in CU_SOURCES]
    _run([nvcc, "-ccbin", "g++", *GENCODE, "-shared", "-o", str(LIB), *objs, "-lcudart_static", "-ldl", "-lrt",
          "-lpthread"])
    _run(["g++", "-std=c++17", "-O2", *inc, *[str(s) for s in CLI_SOURCES], "-o", str(CLI),
          "-L", str(BUILD), "-lautogrid_b200", "-Wl,-rpath,$ORIGIN"])
    if verbose:
        print(f"built {LIB} and {CLI}")
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
