"""Build recipe for libfxc.so (sm_100a).  Compiles every .cu under csrc/ with
nvcc and links one shared library next to this module (in-tree, so the built
library travels with the source tree)."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG.parent / "csrc"
INCLUDE = PKG.parent.parent / "include"
LIB_DIR = PKG / "lib"
LIB = LIB_DIR / "libfxc.so"
OBJ_DIR = PKG.parent / "_build"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "-Xcompiler", "-fvisibility=hidden",
    "--diag-suppress", "128",
]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(CSRC.glob("*.cu"))


def _stale(obj: Path, deps) -> bool:
    return not obj.exists() or any(obj.stat().st_mtime < d.stat().st_mtime for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ_DIR.mkdir(exist_ok=True)
    LIB_DIR.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    objs = []
    jobs = []
    for src in sources():
        obj = OBJ_DIR / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [nvcc(), *NVCC_FLAGS, "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(src),
                   "-o", str(obj)]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    if force or jobs or not LIB.exists() or _stale(LIB, objs):
        tmp = LIB.with_suffix(f".so.tmp{os.getpid()}")
        cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(tmp),
               *map(str, objs), "-Xlinker", "--no-undefined"]
        run(cmd)
        os.replace(tmp, LIB)
    return LIB


CLI_DIR = PKG.parent / "cli"
BIN_DIR = PKG.parent / "bin"
CLI_TOOLS = ("yi-corr", "yi-acf", "yi-xcf", "yi-phasedarray")


def build_cli(force: bool = False, verbose: bool = False) -> Path:
    """The yi-* tools: one C++ binary (mode from argv[0]) linked against
    libfxc.so by rpath, plus the three other names as symlinks."""
    build(force=force, verbose=verbose)
    BIN_DIR.mkdir(exist_ok=True)
    out = BIN_DIR / CLI_TOOLS[0]
    srcs = sorted(CLI_DIR.glob("*.cpp"))
    deps = srcs + sorted(CLI_DIR.glob("*.h")) + [INCLUDE / "fxc.h", LIB]
    if force or _stale(out, deps):
        tmp = out.with_name(out.name + f".tmp{os.getpid()}")
        cxx = os.environ.get("CXX") or shutil.which("g++") or "g++"
        cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", str(INCLUDE), "-I", str(CLI_DIR),
               *map(str, srcs), "-o", str(tmp), "-L", str(LIB_DIR), "-lfxc",
               "-Wl,-rpath,$ORIGIN/../fxc/lib", "-lpthread"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"g++ failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, out)
    for name in CLI_TOOLS[1:]:
        link = BIN_DIR / name
        if not link.is_symlink():
            if link.exists():
                link.unlink()
            link.symlink_to(CLI_TOOLS[0])
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
    print(build_cli(force="--force" in sys.argv, verbose=True))
