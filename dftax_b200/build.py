"""Build the in-tree CUDA library ``libdfjk.so`` for sm_100a.

``python -m dftax_b200.build`` (or ``build()``) compiles every ``csrc/*.cu``
with nvcc into object files under ``dftax_b200/_build/`` and links them into
``dftax_b200/libdfjk.so`` against cuBLAS and cuSOLVER. Sources are compiled in
parallel and only when newer than their object.
"""

from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdfjk.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


_INC = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps(src: str) -> list[str]:
    """Local headers that src includes, directly or through other headers."""
    seen: set[str] = set()
    todo = [src]
    while todo:
        f = todo.pop()
        with open(f) as fh:
            text = fh.read()
        for name in _INC.findall(text):
            h = os.path.normpath(os.path.join(os.path.dirname(f), name))
            if os.path.exists(h) and h not in seen:
                seen.add(h)
                todo.append(h)
    return sorted(seen)


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OUT, os.path.basename(src) + ".o")
    newest = max([os.path.getmtime(src)] + [os.path.getmtime(d) for d in _deps(src)])
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj
    cmd = [nvcc(), *ARCH, *FLAGS, "-c", src, "-o", obj]
    if verbose:
        cmd.insert(-4, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(OUT, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcublas", "-lcusolver"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
