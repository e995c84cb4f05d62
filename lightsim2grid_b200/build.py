"""Build recipe of the native engine (nvcc, sm_100a), in-tree.

``python -m lightsim2grid_b200.build`` compiles ``csrc/*.cpp`` and ``csrc/*.cu`` into
``_lib/liblightsim2grid_b200.so``: every source to its own object (in parallel, under
``_lib/obj``), then one link.  nvcc cross-compiles without a GPU.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
OBJDIR = os.path.join(LIBDIR, "obj")
LIB = os.path.join(LIBDIR, "liblightsim2grid_b200.so")
SOURCES = ["pf_plan.cpp", "pf_capi.cpp", "pf_engine.cu", "pf_noalloc.cu", "pf_flows.cu", "pf_assembly.cu",
           "pf_server.cpp", "pf_tile.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17"] + ARCH + ["-lineinfo", "-Xcompiler", "-fPIC"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".hpp", ".cuh"))]
    hs.append(os.path.join(HERE, "..", "include", "lightsim2grid_b200.h"))
    return [h for h in hs if os.path.exists(h)]


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "lightsim2grid_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _obj(src):
    return os.path.join(OBJDIR, os.path.splitext(src)[0] + ".o")


def build(force=False, verbose=False):
    """Compile the engine if a source is newer than the library; return the library path.
    An object is rebuilt when its source or any header is newer than it (or with force)."""
    if not force and not needs_build():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    newest_header = max((os.path.getmtime(h) for h in _headers()), default=0.0)
    nvcc = _nvcc()

    def compile_one(src):
        path, obj = os.path.join(CSRC, src), _obj(src)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(path)
                and os.path.getmtime(obj) >= newest_header):
            return None
        cmd = [nvcc] + FLAGS + (["-Xptxas=-v"] if verbose else []) + ["-c", path, "-o", obj + ".tmp"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
        os.replace(obj + ".tmp", obj)
        return src

    with ThreadPoolExecutor(max_workers=max(1, min(len(SOURCES), os.cpu_count() or 1))) as ex:
        list(ex.map(compile_one, SOURCES))
    tmp = LIB + ".tmp"
    subprocess.check_call([nvcc] + ARCH + ["-shared", "-o", tmp] + [_obj(s) for s in SOURCES])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
