"""Build libicarat_gpu.so in-tree for sm_100a (B200).

Each CUDA translation unit is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` into ``_build/`` and
linked into ``icarat2_b200/libicarat_gpu.so``.  Run ``python -m
icarat2_b200.build`` (or ``build()``); nothing is compiled at import time.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libicarat_gpu.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                  "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _compile(nvcc, src, verbose):
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    deps = [path] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith(".cuh")]
    deps.append(os.path.join(HERE, "..", "include", "icarat_gpu.h"))
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj, ""
    flags = list(NVFLAGS)
    if verbose:
        flags += ["-Xptxas", "-v"]
    cmd = [nvcc] + flags + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed on %s:\n%s\n%s" % (src, r.stdout, r.stderr))
    return obj, r.stderr


def build(verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(nvcc, s, verbose), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for (o, log), s in zip(results, srcs):
            if log:
                sys.stderr.write("== %s\n%s" % (s, log))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < newest:
        cmd = [nvcc] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    build_examples()
    return OUT


EXAMPLES = os.path.join(HERE, "examples")


def build_examples():
    """C++ sample drivers written against include/icarat_b200.hpp."""
    include = os.path.join(HERE, "..", "include")
    for src in sorted(os.listdir(EXAMPLES)):
        if not src.endswith(".cpp"):
            continue
        exe = os.path.join(EXAMPLES, src[:-4])
        deps = [os.path.join(EXAMPLES, src), OUT, os.path.join(include, "icarat_b200.hpp"),
                os.path.join(include, "icarat_gpu.h")]
        if os.path.exists(exe) and all(os.path.getmtime(exe) >= os.path.getmtime(d)
                                       for d in deps):
            continue
        cmd = ["g++", "-O2", "-std=c++17", "-I", include, "-o", exe,
               os.path.join(EXAMPLES, src), "-L", HERE, "-licarat_gpu",
               "-Wl,-rpath,$ORIGIN/.."]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("example build failed:\n%s\n%s" % (r.stdout, r.stderr))


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
