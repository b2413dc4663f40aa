"""Builds the native libraries (sm_100a) in place with nvcc.

libpicgpu.so  -- the IFE-PIC step: CUDA kernels, the C-ABI of
                 include/picgpu.h and the host-side mesh builder.
libpicunet.so -- the learned preconditioner's network: tcgen05 implicit-GEMM
                 convolutions (CUTLASS SM100 collectives instantiated here)
                 and the network's own kernels (include/picunet.h).

FP64 kernels are compiled with --fmad=false; where a fused multiply-add is
wanted the source calls fma() explicitly, so the arithmetic is fixed by the
source text.  Each source compiles to its own object, rebuilt only when it or
one of its library's headers changed, so the CUTLASS unit (a minute or more)
is not rebuilt for unrelated edits.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_obj")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

LIBS = {
    "libpicgpu.so": {"sources": ["picgpu.cu", "sort_mcc.cu", "precond.cu", "mesh_build.cpp", "ife_dev.cu", "noalloc.cu",
                                 "diag.cu"],
                     "headers": ["csrc/pic_ctx.h", "csrc/pic_common.h", "csrc/pic_mcc_kin.h", "csrc/ife_elem.h",
                                 "../include/picgpu.h"],
                     "flags": ["--fmad=false"], "cutlass": False},
    "libpicunet.so": {"sources": ["unet_conv.cu", "unet_ops.cu"], "headers": ["../include/picunet.h"],
                      "flags": [], "cutlass": True},
}


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def cutlass_include() -> list[str]:
    """CUTLASS/CuTe header trees vendored with the Python packages of the image."""
    import site
    roots = []
    for sp in site.getsitepackages() + [site.getusersitepackages()]:
        roots.append(os.path.join(sp, "flashinfer", "data", "cutlass"))
        roots.append(os.path.join(sp, "tilelang", "3rdparty", "cutlass"))
    for r in roots:
        if os.path.exists(os.path.join(r, "include", "cutlass", "cutlass.h")):
            return ["-I" + os.path.join(r, "include"), "-I" + os.path.join(r, "tools", "util", "include")]
    raise RuntimeError("CUTLASS headers not found")


def _compile(src: str, spec: dict, verbose: bool) -> str:
    os.makedirs(OBJ, exist_ok=True)
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    deps = [src, os.path.abspath(__file__)] + [os.path.normpath(os.path.join(HERE, h)) for h in spec["headers"]]
    if os.path.exists(obj) and all(os.path.getmtime(d) <= os.path.getmtime(obj) for d in deps):
        return obj
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", *spec["flags"],
           "-Xcompiler", "-fPIC,-O2,-ffp-contract=off", "-c", src, "-o", obj + ".tmp"]
    if spec["cutlass"]:
        cmd += ["--expt-relaxed-constexpr", *cutlass_include()]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed on " + src)
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(obj + ".tmp", obj)
    return obj


def build(force: bool = False, verbose: bool = False, libs=None) -> dict:
    """Compile (only what changed) and link; return {library: path}."""
    out = {}
    for lib, spec in LIBS.items():
        if libs is not None and lib not in libs:
            continue
        srcs = [os.path.join(CSRC, s) for s in spec["sources"]]
        if force:
            for s in srcs:
                o = os.path.join(OBJ, os.path.basename(s) + ".o")
                if os.path.exists(o):
                    os.remove(o)
        with ThreadPoolExecutor(max_workers=min(4, len(srcs))) as ex:
            objs = list(ex.map(lambda s: _compile(s, spec, verbose), srcs))
        path = os.path.join(HERE, lib)
        if force or not os.path.exists(path) or any(os.path.getmtime(o) > os.path.getmtime(path) for o in objs):
            cmd = [nvcc(), *ARCH, "-shared", "-o", path + ".tmp", *objs]
            res = subprocess.run(cmd, capture_output=True, text=True)
            if res.returncode != 0:
                sys.stderr.write(res.stdout + res.stderr)
                raise RuntimeError("link failed for " + lib)
            os.replace(path + ".tmp", path)
        out[lib] = path
    return out


if __name__ == "__main__":
    for k, v in build(force="--force" in sys.argv, verbose="-v" in sys.argv).items():
        print(k, v)
