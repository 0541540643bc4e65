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


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
