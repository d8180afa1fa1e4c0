"""Build recipe of libjms_b200.so (sm_100a) -- run ``python -m jmultislicelib_b200.build``.

Compiles the CUDA passes and the C++ host library in csrc/ with nvcc for
sm_100a only and links them into jmultislicelib_b200/libjms_b200.so (in tree,
next to this file), exporting the C ABI of include/jms_b200.h.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libjms_b200.so")
APP = os.path.join(HERE, "jmsbench")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O3", f"-I{ROOT}/include"]
SOURCES = ["jms_kernels.cu", "jms_host.cpp", "jms_generators.cpp", "jms_capi.cpp", "jms_class.cpp", "jms_noalloc.cu", "jms_pgr.cu",
           "jms_pgr_host.cpp", "jms_sli.cpp", "jms_nn.cu", "jms_tc.cu"] + [f"jms_inst_{k}.cu" for k in range(10)] + [f"jms_pgr_ops_{k}.cu" for k in range(3)]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    inc = os.path.join(ROOT, "include")
    return hs + [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]


def _compile(src: str, verbose: bool) -> str:
    s = os.path.join(CSRC, src)
    o = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    if _newer(o, [s] + _headers()):
        cmd = [NVCC, *ARCH, *COMMON, "-c", s, "-o", o]
        if verbose and src.endswith(".cu"):
            cmd.insert(1, "-Xptxas=-v")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr[-4000:]}")
        if verbose:
            sys.stderr.write(r.stderr)
    return o


def build(verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    with cf.ThreadPoolExecutor(min(len(SOURCES), os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if _newer(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
    # the reference-bench-compatible STEM driver (apps/jmsbench.cpp) over the C ABI
    app_src = os.path.join(HERE, "apps", "jmsbench.cpp")
    if _newer(APP, [app_src, LIB, os.path.join(ROOT, "include", "jms_b200.h")]):
        cmd = ["g++", "-std=c++17", "-O2", "-o", APP, app_src, f"-I{ROOT}/include", f"-L{HERE}", "-ljms_b200",
               "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"jmsbench build failed:\n{r.stderr[-4000:]}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
