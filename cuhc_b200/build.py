"""Builds cuhc_b200/libcuhc.so from csrc/ for sm_100a (in-tree, no JIT).

Each translation unit compiles in parallel; the shared library is linked
with nvcc. Rebuilds only what changed: a unit is stale when it, or a header
it includes (directly or through other csrc/ headers), is newer than its
object.

    python cuhc_b200/build.py [--force] [--verbose]
"""

import concurrent.futures
import os
import pathlib
import re
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
SRC = HERE / "csrc"
OBJ = HERE / "_build"
LIBRARY = HERE / "libcuhc.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-DNDEBUG", "-Xcompiler", "-fPIC"]
CUDA_FLAGS = COMMON + ARCH + ["-lineinfo", "--expt-relaxed-constexpr"]


def _sources():
    return sorted(SRC.glob("*.cu")) + sorted(SRC.glob("*.cpp"))


_INCLUDE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.MULTILINE)


def _newest_dependency(source, cache):
    """Latest modification time of `source` and every csrc/ header it reaches
    through quoted includes."""
    seen, stack, newest = set(), [source], 0.0
    while stack:
        path = stack.pop()
        if path in seen or not path.exists():
            continue
        seen.add(path)
        newest = max(newest, path.stat().st_mtime)
        if path not in cache:
            cache[path] = [SRC / name for name in _INCLUDE.findall(path.read_text())]
        stack.extend(cache[path])
    return newest


def _compile(source, verbose):
    obj = OBJ / (source.name + ".o")
    if source.suffix == ".cu":
        cmd = [NVCC, *CUDA_FLAGS, "-c", str(source), "-o", str(obj)]
        if verbose:
            cmd[1:1] = ["-Xptxas", "-v"]
    else:
        cmd = [NVCC, *COMMON, "-x", "cu", "-c", str(source), "-o", str(obj)]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{result.stdout}{result.stderr}")
    return obj, result.stderr


def build(force=False, verbose=False, jobs=None):
    """Compiles stale units and links libcuhc.so; returns its path."""
    OBJ.mkdir(exist_ok=True)
    sources = _sources()
    cache = {}
    stale = []
    for source in sources:
        obj = OBJ / (source.name + ".o")
        if (force or not obj.exists()
                or obj.stat().st_mtime < _newest_dependency(source, cache)):
            stale.append(source)
    # Objects of units that no longer exist must not be linked.
    for obj in OBJ.glob("*.o"):
        if not (SRC / obj.name[:-2]).exists():
            obj.unlink()
    logs = []
    if stale:
        with concurrent.futures.ThreadPoolExecutor(jobs or os.cpu_count() or 4) as pool:
            for obj, log in pool.map(lambda s: _compile(s, verbose), stale):
                logs.append((obj, log))
    objects = [OBJ / (s.name + ".o") for s in sources]
    if stale or not LIBRARY.exists():
        tmp = LIBRARY.with_suffix(".so.tmp")
        cmd = [NVCC, *ARCH, "-shared", *map(str, objects), "-o", str(tmp), "-lcudart"]
        subprocess.run(cmd, check=True)
        tmp.replace(LIBRARY)
    if verbose:
        for obj, log in logs:
            print(f"== {obj.name}\n{log}")
    return LIBRARY


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
