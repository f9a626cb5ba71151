"""Builds origami_b200/liborigami_b200.so (host C++ + sm_100a CUDA) in-tree.

    python -m origami_b200.build [--force] [--debug] [-D NAME=VALUE ...] [--out DIR]

Every translation unit is compiled by nvcc (host .cpp files go to the host
compiler through nvcc) with ``-gencode arch=compute_100a,code=sm_100a``; the
CUDA runtime is linked statically so the library needs only the driver.
Objects are cached under origami_b200/_build/ and rebuilt when a source or
header is newer than the object.  ``-D`` passes tuning macros (for example
OG_PAIR_MIN_BLOCKS) and ``--out`` writes that variant's objects and library
to another directory, leaving the default build untouched.
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "liborigami_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# FP32 pair kernels flush denormals (no subnormal fix-up paths around the
# MUFU rsqrt / ex2); every FP64 path is unaffected by -ftz.
PER_FILE_FLAGS = {"pair_kernels.cu": ["-ftz=true"]}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_compiler() -> list[str]:
    # nvcc picks `gcc` from PATH; prefer the system compiler when present.
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp")) + glob.glob(os.path.join(CSRC, "engine", "*.cu")))


def headers() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True)
                  + glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True)
                  + glob.glob(os.path.join(ROOT, "include", "*.h")))


def _stale(obj: str, src: str, hdr_mtime: float) -> bool:
    if not os.path.exists(obj):
        return True
    m = os.path.getmtime(obj)
    return m < os.path.getmtime(src) or m < hdr_mtime


def build(force: bool = False, debug: bool = False, verbose: bool = False, defines: list[str] | None = None,
          out_dir: str | None = None) -> str:
    build_dir = os.path.join(out_dir, "_build") if out_dir else BUILD
    lib = os.path.join(out_dir, "liborigami_b200.so") if out_dir else LIB
    os.makedirs(build_dir, exist_ok=True)
    nv = nvcc()
    hdr_mtime = max((os.path.getmtime(h) for h in headers()), default=0.0)
    opt = ["-O0", "-g", "-G"] if debug else ["-O3", "-lineinfo"]
    common = [nv, *ARCH, *host_compiler(), "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "-I", os.path.join(ROOT, "include"), "--expt-relaxed-constexpr",
              *[f"-D{d}" for d in (defines or [])]]
    jobs = []
    objs = []
    for src in sources():
        rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
        obj = os.path.join(build_dir, rel + ".o")
        objs.append(obj)
        if force or _stale(obj, src, hdr_mtime):
            extra = PER_FILE_FLAGS.get(os.path.basename(src), [])
            jobs.append([*common, *opt, *extra, "-c", src, "-o", obj])

    def run(cmd: list[str]) -> tuple[int, str, list[str]]:
        p = subprocess.run(cmd, capture_output=True, text=True)
        return p.returncode, p.stdout + p.stderr, cmd

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for rc, out, cmd in ex.map(run, jobs):
            if verbose or rc != 0:
                sys.stderr.write(" ".join(cmd) + "\n" + out)
            if rc != 0:
                raise RuntimeError(f"compile failed: {cmd[-3]}")
    if force or jobs or not os.path.exists(lib):
        link = [nv, *ARCH, *host_compiler(), "-shared", "-o", lib, *objs, "-ldl", "-lpthread"]
        rc, out, _ = run(link)
        if verbose or rc != 0:
            sys.stderr.write(" ".join(link) + "\n" + out)
        if rc != 0:
            raise RuntimeError("link failed")
    if out_dir:  # a variant library finds the data tables next to itself
        data = os.path.join(out_dir, "data")
        if not os.path.exists(data):
            os.symlink(os.path.join(PKG, "data"), data)
    return lib


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--debug", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("-D", dest="defines", action="append", default=[], help="NAME=VALUE tuning macro")
    ap.add_argument("--out", default=None, help="directory for a variant build")
    args = ap.parse_args()
    print(build(force=args.force, debug=args.debug, verbose=args.verbose, defines=args.defines, out_dir=args.out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
