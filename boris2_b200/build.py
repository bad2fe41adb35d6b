"""Build the CUDA library boris2_b200/_lib/libboris_b200.so for sm_100a (in-tree).

Every translation unit under csrc/ is compiled separately (in parallel) with
``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and linked into one
shared object exposing the C ABI of include/boris_b200.h.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "libboris_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-ccbin", "g++",
         "--expt-relaxed-constexpr", "-I", os.path.join(HERE, "..", "include")]


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _compile(src, extra):
    obj = os.path.join(OBJDIR, src + ".o")
    cmd = [NVCC] + ARCH + FLAGS + extra + ["-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    return obj, r.stderr


def _stale(src, hdr_mtime, force):
    """A translation unit is recompiled when forced, when its object is missing, or when the object is
    older than the source or than the newest shared header / build recipe."""
    obj = os.path.join(OBJDIR, src + ".o")
    if force or not os.path.exists(obj):
        return True
    return os.path.getmtime(obj) < max(os.path.getmtime(os.path.join(CSRC, src)), hdr_mtime)


def build(force=False, verbose=False, extra=None):
    """Compile the stale translation units and link; returns the path of the shared library."""
    extra = list(extra or [])
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    hdr = os.path.join(HERE, "..", "include", "boris_b200.h")
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if not f.endswith((".cu", ".cpp"))]
    hdr_mtime = max([os.path.getmtime(h) for h in headers] + [os.path.getmtime(hdr), os.path.getmtime(__file__)])
    todo = [s for s in _sources() if extra or _stale(s, hdr_mtime, force)]
    objs = [os.path.join(OBJDIR, s + ".o") for s in _sources()]
    if not todo and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, extra), todo))
    objs = [os.path.join(OBJDIR, s + ".o") for s in _sources()]
    if verbose:
        for _, err in results:
            if err.strip():
                print(err, file=sys.stderr)
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    return LIB


if __name__ == "__main__":
    force = "--force" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(force=force, verbose=bool(extra), extra=extra))
