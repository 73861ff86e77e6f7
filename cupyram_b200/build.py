"""Build the native engine in-tree: ``python -m cupyram_b200.build``.

Compiles every ``csrc/*.cu`` for sm_100a (B200), one process per file, and
links ``libcupyram_b200.so`` next to this file.  nvcc cross-compiles, so no GPU is needed to build.
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "libcupyram_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def nvcc():
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; set NVCC or put CUDA's bin on PATH")
    return cand


def sources():
    return sorted(CSRC.glob("*.cu"))


def up_to_date():
    if not OUT.exists():
        return False
    t = OUT.stat().st_mtime
    deps = list(CSRC.glob("*")) + [HERE.parent / "include" / "cupyram_b200.h"]
    return all(d.stat().st_mtime <= t for d in deps if d.exists())


def _compile(src, obj, verbose):
    cmd = [nvcc(), *ARCH, *CFLAGS, "-I", str(HERE.parent / "include"), "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return obj


def build(force=False, verbose=False, jobs=None):
    """Compile every csrc/*.cu to an object in _build/ (in parallel: the four
    precision forms of the batched march are separate translation units), then
    link the shared library.  Objects newer than their source and than every
    header are reused."""
    if not force and up_to_date():
        return OUT
    objdir = HERE.parent / "_build"
    objdir.mkdir(exist_ok=True)
    srcs = sources()
    objs = [objdir / (s.stem + ".o") for s in srcs]
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((HERE.parent / "include").glob("*.h"))
    newest_header = max((h.stat().st_mtime for h in headers), default=0.0)
    stale = [(s, o) for s, o in zip(srcs, objs)
             if force or not o.exists() or o.stat().st_mtime < max(s.stat().st_mtime, newest_header)]
    n = jobs or min(max(len(stale), 1), os.cpu_count() or 1)
    with ThreadPoolExecutor(max_workers=max(1, n)) as ex:
        for f in [ex.submit(_compile, s, o, verbose) for s, o in stale]:
            f.result()
    cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(OUT) + ".tmp", *map(str, objs)]
    subprocess.run(cmd, check=True)
    os.replace(str(OUT) + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(p)
