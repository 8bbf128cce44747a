"""Build recipe for the native library (sm_100a only).

Compiles every ``csrc/*.cu`` and ``csrc/*.cpp`` with nvcc for
``compute_100a``/``sm_100a`` into ``rtscan_b200/librtscan_b200.so`` (kept in
the source tree so it travels with the repository snapshot), and the
drop-in command-line driver ``rtscan_b200/rtscan_b200_cli`` linked against it.

    python -m rtscan_b200.build [--force] [-j N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import hashlib
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "librtscan_b200.so")
CLI = os.path.join(PKG, "rtscan_b200_cli")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3,-fvisibility=hidden",
          "-I", os.path.join(ROOT, "include")]
CU_FLAGS = ARCH + COMMON + ["--expt-relaxed-constexpr", "-Xptxas", "-O3"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _digest(paths):
    h = hashlib.sha256()
    for p in sorted(paths):
        with open(p, "rb") as f:
            h.update(p.encode() + f.read())
    h.update(" ".join(CU_FLAGS).encode())
    return h.hexdigest()


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def build(force: bool = False, jobs: int = 8, verbose: bool = False) -> str:
    srcs = [s for s in sources() if os.path.basename(s) != "cli.cpp"]
    headers = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    stamp = os.path.join(OUT, "stamp")
    digest = _digest(sources() + headers)
    if not force and os.path.exists(LIB) and os.path.exists(CLI) and os.path.exists(stamp):
        with open(stamp) as f:
            if f.read().strip() == digest:
                return LIB
    os.makedirs(OUT, exist_ok=True)
    cc = nvcc()

    def compile_one(src):
        obj = os.path.join(OUT, os.path.basename(src) + ".o")
        cmd = [cc] + CU_FLAGS + ["-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [cc] + ARCH + COMMON + ["-x", "cu", "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        return obj

    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(compile_one, srcs))
    tmp = LIB + ".tmp"
    subprocess.run([cc] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcuda"], check=True)
    os.replace(tmp, LIB)
    cli_src = os.path.join(CSRC, "cli.cpp")
    if os.path.exists(cli_src):
        subprocess.run([cc] + ARCH + COMMON + ["-x", "cu", cli_src, "-o", CLI, "-L", PKG, "-lrtscan_b200",
                        "-Xlinker", "-rpath,$ORIGIN"], check=True)
    with open(stamp, "w") as f:
        f.write(digest)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, jobs=a.j, verbose=a.v))


if __name__ == "__main__":
    sys.exit(main())
