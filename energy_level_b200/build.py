"""Build recipe of the native library ``libel_b200.so`` (sm_100a only).

Every ``.cu`` file under ``csrc/`` is compiled by nvcc for
``arch=compute_100a,code=sm_100a`` and linked into one shared library with a
plain C ABI (``include/energy_level_b200.h``).  The library is built in-tree
next to this file so that it travels with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libel_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def nvcc() -> str:
    path = os.path.join(CUDA_HOME, "bin", "nvcc")
    if os.path.exists(path):
        return path
    found = shutil.which("nvcc")
    if not found:
        raise RuntimeError("nvcc not found; set CUDA_HOME")
    return found


def _flags(verbose_ptx: bool = False) -> list[str]:
    flags = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
             "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), *ARCH]
    if verbose_ptx:
        flags += ["-Xptxas", "-v"]
    return flags


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(ROOT, "include", "energy_level_b200.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose_ptx: bool = False, quiet: bool = True) -> str:
    """Compile the library if any source is newer than it; return its path."""
    if not force and not verbose_ptx and not _needs_build():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    cc = nvcc()
    flags = _flags(verbose_ptx)

    def compile_one(src: str) -> tuple[str, str]:
        obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
        cmd = [cc, *flags, "-c", src, "-o", obj]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), res.stderr))
        return obj, res.stderr

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        results = list(pool.map(compile_one, sources()))
    if verbose_ptx or not quiet:
        for _, log in results:
            if log.strip():
                sys.stderr.write(log)
    objs = [o for o, _ in results]
    tmp = LIB + ".tmp"
    cmd = [cc, *ARCH, "-shared", "-o", tmp, *objs, "-cudart", "shared",
           "-Xlinker", "-rpath=" + os.path.join(CUDA_HOME, "lib64")]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), res.stderr))
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptx="-v" in sys.argv, quiet=False))
