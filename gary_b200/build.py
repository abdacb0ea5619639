"""Build recipe for libgary_b200.so (sm_100a) -- plain nvcc, in-tree.

    python -m gary_b200.build            # incremental build
    python -m gary_b200.build --force    # rebuild everything

Every .cu file under csrc/ is compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) and linked into
gary_b200/libgary_b200.so next to this file, so the library travels with the
source tree.  cudart is linked statically (nvcc's default), so loading the
library needs no CUDA toolkit at run time.
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
OBJ = PKG / "_build"
LIB = PKG / "libgary_b200.so"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", *ARCH,
    "-Xcompiler", "-fPIC,-fopenmp,-O3",
    "--expt-relaxed-constexpr", "--extended-lambda",
    "-diag-suppress", "177,550",
    f"-I{INCLUDE}", f"-I{CSRC}",
]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build gary_b200")
    return cand


def _deps(src: Path) -> list[Path]:
    return [src, *CSRC.glob("*.cuh"), INCLUDE / "gary_b200.h", Path(__file__)]


def _stale(src: Path, obj: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.exists() and p.stat().st_mtime > t for p in _deps(src))


def _compile(src: Path, obj: Path, extra: list[str]) -> None:
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    extra = extra or []
    OBJ.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    jobs = []
    for s in srcs:
        o = OBJ / (s.stem + ".o")
        if force or _stale(s, o):
            jobs.append((s, o))
    if jobs:
        workers = min(len(jobs), max(1, os.cpu_count() or 1))
        with cf.ThreadPoolExecutor(workers) as ex:
            futs = {ex.submit(_compile, s, o, extra): s for s, o in jobs}
            for f in cf.as_completed(futs):
                f.result()
                if verbose:
                    print(f"  compiled {futs[f].name}")
    objs = [OBJ / (s.stem + ".o") for s in srcs]
    if force or jobs or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), "-shared", *ARCH, "-o", str(tmp), *map(str, objs), "-lgomp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
        if verbose:
            print(f"  linked {LIB}")
    return LIB


def reference_tree() -> Path | None:
    """The reference's source tree for the oracle build: $GARY_REF_TREE, else a
    `reference` directory beside this repository, when either holds its
    sources (src/Graph.cpp)."""
    for cand in (os.environ.get("GARY_REF_TREE"), ROOT.parent / "reference"):
        if cand and (Path(cand) / "src" / "Graph.cpp").exists():
            return Path(cand)
    return None


def build_oracle(verbose: bool = False) -> None:
    """Compile the CPU oracle, and the reference's own code when its tree is present."""
    ref = reference_tree()
    cmd = ["make", "-s", "-C", str(ROOT / "oracle"), f"PYTHON={sys.executable}", f"REF={ref or ''}", "all"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stdout.strip():
        print(r.stdout)


def build_shim_tests(verbose: bool = False) -> None:
    """Compile the C++ shim test programs (tests/cpp) against the built library."""
    d = ROOT / "tests" / "cpp"
    if not (d / "Makefile").exists():
        return
    cmd = ["make", "-s", "-C", str(d), f"NVCC={nvcc()}", "all"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"shim test build failed:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stdout.strip():
        print(r.stdout)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--oracle", action="store_true", help="also build oracle/")
    ap.add_argument("--shim-tests", action="store_true", help="also build tests/cpp")
    a = ap.parse_args()
    print(build(force=a.force, verbose=True))
    if a.oracle:
        build_oracle(verbose=True)
    if a.shim_tests:
        build_shim_tests(verbose=True)
