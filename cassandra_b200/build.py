"""In-tree build of the native library (libcassandra_b200.so) for sm_100a.

Every translation unit under csrc/ is compiled with nvcc for
``arch=compute_100a,code=sm_100a`` (no other architecture is emitted) and
linked into one shared library next to this file.  Objects are rebuilt only
when a source or header is newer than the object.

    python -m cassandra_b200.build          # build
    python -m cassandra_b200.build --force  # rebuild everything
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
BUILD = HERE / "_build"
LIB = HERE / "libcassandra_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++20", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-fopenmp,-fvisibility=hidden,-O3",
    f"-I{INCLUDE}",
]


def nvcc() -> str:
    for cand in (os.environ.get("CUDA_HOME", ""), "/usr/local/cuda"):
        p = Path(cand) / "bin" / "nvcc"
        if cand and p.exists():
            return str(p)
    found = shutil.which("nvcc")
    if not found:
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build cassandra_b200")
    return found


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: Path, force: bool, hdr_mtime: float, extra: list[str]) -> Path:
    obj = BUILD / (src.name + ".o")
    if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, hdr_mtime):
        return obj
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    """Compiles csrc/ into libcassandra_b200.so and returns its path."""
    BUILD.mkdir(exist_ok=True)
    extra = list(extra or [])
    hdr = _headers_mtime()
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, hdr, extra), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        # cudart is linked statically (nvcc's default), so the library needs
        # only the CUDA driver at run time.
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fopenmp", "-o", str(LIB), *map(str, objs), "-lgomp"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
        if verbose:
            print(f"linked {LIB}")
    return LIB


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true", help="pass -Xptxas -v (registers, spills, smem)")
    args = ap.parse_args(argv)
    extra = ["-Xptxas", "-v"] if args.ptxas_verbose else []
    path = build(force=args.force or args.ptxas_verbose, verbose=True, extra=extra)
    print(path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
