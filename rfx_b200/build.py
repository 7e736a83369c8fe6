"""Build recipe for the in-tree CUDA library ``rfx_b200/librfxb200.so``.

Compiles every ``rfx_b200/csrc/*.cu`` for sm_100a only and links them into one
shared library exporting the C ABI of ``include/rfxb200.h``.  The CUDA runtime
is linked statically so the library does not depend on which libcudart the
host process loaded first.

Usage: ``python -m rfx_b200.build [--verbose]`` (``--verbose`` adds
``-Xptxas -v``: registers, spills and shared memory per kernel).
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "librfxb200.so")
FFI_SRC = os.path.join(CSRC, "ffi", "rfxb_ffi.cc")
FFI_LIB = os.path.join(HERE, "librfxb200_ffi.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build rfx_b200")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def build(verbose: bool = False, force: bool = False) -> str:
    srcs = sources()
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "rfxb200.h"))
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(d) <= t for d in deps):
            return LIB
    cmd = [nvcc_path(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-cudart", "static", "-I", os.path.join(ROOT, "include"), "-o", LIB + ".tmp", *srcs]
    if verbose:
        cmd[1:1] = ["-Xptxas", "-v"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + res.stdout + res.stderr)
    if verbose:
        sys.stdout.write(res.stdout + res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def ffi_include_dir():
    """jaxlib's XLA FFI header directory, or None without jax."""
    try:
        import jax
        inc = jax.ffi.include_dir()
    except Exception:
        return None
    return inc if inc and os.path.isdir(inc) else None


def build_ffi(force: bool = False):
    """Compile the XLA FFI handlers (``csrc/ffi/rfxb_ffi.cc``) into
    ``librfxb200_ffi.so`` linked against ``librfxb200.so``.  Returns the
    library path, or None when jaxlib's FFI headers are not installed (the
    handlers need them; nothing else in the package does)."""
    inc = ffi_include_dir()
    if inc is None:
        return None
    lib = build(force=force)
    if not force and os.path.exists(FFI_LIB) and os.path.getmtime(FFI_LIB) >= max(
            os.path.getmtime(FFI_SRC), os.path.getmtime(lib)):
        return FFI_LIB
    cmd = [nvcc_path(), "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-I", inc,
           "-I", os.path.join(ROOT, "include"), "-o", FFI_LIB + ".tmp", FFI_SRC, "-L", HERE, "-lrfxb200",
           "-Xlinker", "-rpath,$ORIGIN"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + res.stdout + res.stderr)
    os.replace(FFI_LIB + ".tmp", FFI_LIB)
    return FFI_LIB


if __name__ == "__main__":
    v = "--verbose" in sys.argv
    print(build(verbose=v, force=True))
