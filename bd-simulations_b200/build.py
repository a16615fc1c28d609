"""Build recipe of libbd_b200.so (in-tree, sm_100a) and the bdkap driver.

    python bd-simulations_b200/build.py [--force]

Compiles every source under csrc/ with nvcc for sm_100a (CUDA sources) or
the host C++ compiler through nvcc (host sources), links one shared library
with the CUDA runtime linked statically, and builds the host driver
host/bdkap_main.cpp against it. Objects go to _build/ next to this file.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbd_b200.so")
EXE = os.path.join(HERE, "bdkap")
INC = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INC, "-I" + CSRC]
CUFLAGS = ARCH + COMMON + ["-lineinfo", "--expt-relaxed-constexpr"]


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(INC, "bd_api.h"))
    return hs


def _compile(src, force):
    obj = os.path.join(BUILD, src + ".o")
    path = os.path.join(CSRC, src)
    newest = max([os.path.getmtime(path)] + [os.path.getmtime(h) for h in _headers()])
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj
    if src.endswith(".cu"):
        cmd = [NVCC] + CUFLAGS + ["-c", path, "-o", obj]
    else:
        # host sources see the device structs through the engine header
        cmd = [NVCC] + CUFLAGS + ["-x", "cu", "-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s" % (" ".join(cmd), r.stderr[-6000:]))
    return obj


def build(force=False, jobs=8):
    os.makedirs(BUILD, exist_ok=True)
    with ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), _sources()))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs + ["-lpthread", "-ldl", "-lrt"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: %s\n%s" % (" ".join(cmd), r.stderr[-6000:]))
    main_src = os.path.join(HERE, "host", "bdkap_main.cpp")
    if os.path.exists(main_src):
        hdr = os.path.join(HERE, "host", "RunZustand.hpp")
        deps = [main_src, LIB] + ([hdr] if os.path.exists(hdr) else [])
        if force or not os.path.exists(EXE) or os.path.getmtime(EXE) < max(os.path.getmtime(d) for d in deps):
            cmd = ["g++", "-O2", "-std=c++17", "-I" + INC, "-I" + os.path.join(HERE, "host"), main_src,
                   "-L" + HERE, "-lbd_b200", "-Wl,-rpath,$ORIGIN", "-o", EXE]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError("driver build failed:\n" + r.stderr[-4000:])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
