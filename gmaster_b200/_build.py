"""Build recipe for the in-tree CUDA library ``gmaster_b200/libgm_b200.so`` (sm_100a).

``python -m gmaster_b200._build`` compiles every ``csrc/*.cu`` with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` into a shared object next to this file.
The library exposes only the C ABI declared in ``include/gm_b200.h``.
"""

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libgm_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def _deps():
    return (sources() + sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh")))
            + [os.path.join(ROOT, "include", "gm_b200.h")])


def up_to_date():
    if not os.path.exists(LIB):
        return False
    built = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= built for p in _deps())


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def build(force=False, verbose=False, jobs=None):
    """Compile each source to an object in parallel, then link the shared library."""
    if not force and up_to_date():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                    "-I" + os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]
    if verbose:
        flags += ["-Xptxas", "-v"]
    procs = []
    objs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        cmd = [nvcc()] + flags + ["-c", src, "-o", obj]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for cmd, proc in procs:
        out, _ = proc.communicate()
        text = out.decode(errors="replace")
        if proc.returncode != 0:
            failed.append((cmd, text))
        elif verbose and text:
            sys.stdout.write(text)
    if failed:
        msg = "\n".join(" ".join(c) + "\n" + t for c, t in failed)
        raise RuntimeError("nvcc failed:\n" + msg)
    tmp = LIB + f".tmp{os.getpid()}"
    subprocess.check_call([nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"])
    os.replace(tmp, LIB)
    return LIB


FFI_LIB = os.path.join(HERE, "libgm_b200_ffi.so")


def ffi_include_dir():
    """jaxlib's XLA FFI header directory, or None where JAX is not installed."""
    try:
        import jax.ffi

        path = jax.ffi.include_dir()
    except Exception:  # JAX absent or too old: no FFI headers
        return None
    return path if os.path.exists(os.path.join(path, "xla", "ffi", "api", "ffi.h")) else None


def build_ffi():
    """Compile csrc/ffi/gm_ffi.cc (the jax.ffi handlers) where jaxlib's headers exist;
    returns the library path, or None when they do not."""
    inc = ffi_include_dir()
    if inc is None:
        return None
    lib = build()
    src = os.path.join(HERE, "csrc", "ffi", "gm_ffi.cc")
    cuda_inc = os.path.join(os.path.dirname(os.path.dirname(nvcc())) if os.path.sep in nvcc() else "/usr/local/cuda",
                            "include")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I" + inc, "-I" + cuda_inc,
                           "-I" + os.path.join(ROOT, "include"), src, "-o", FFI_LIB, lib,
                           "-Wl,-rpath," + HERE])
    return FFI_LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
    if build_ffi():
        print(FFI_LIB)
