"""Build libamrvac_gpu.so (sm_100a) in-tree with nvcc.

    python -m amrvac_b200.build            # build if sources changed
    python -m amrvac_b200.build --force

Each translation unit under csrc/ is compiled in parallel to
_build/<name>.o and linked into amrvac_b200/libamrvac_gpu.so.
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.environ.get("AMRVAC_BUILD_DIR", os.path.join(HERE, "_build"))
LIB = os.environ.get("AMRVAC_LIB_OUT", os.path.join(HERE, "libamrvac_gpu.so"))
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr", "-I", INCLUDE]
EXTRA = os.environ.get("AMRVAC_NVCC_EXTRA", "").split()
UNITS = ["capi.cu", "aux.cu", "k_hd.cu", "k_mhd2.cu", "k_mhd3.cu", "noalloc.cu", "ensemble.cu", "adjoint.cu", "amr.cu", "amr_plan.cu", "k_mp5_hd.cu", "k_mp5_mhd.cu",
         "k_bn8.cu", "k_bn10.cu", "k_bn12.cu", "k_bn32.cu", "k_tune.cu", "smallavg.cu"]


def _digest() -> str:
    h = hashlib.sha256()
    for d in (CSRC, INCLUDE):
        for name in sorted(os.listdir(d)):
            if name.endswith((".cu", ".cuh", ".h")):
                with open(os.path.join(d, name), "rb") as f:
                    h.update(name.encode())
                    h.update(f.read())
    h.update(" ".join(ARCH + FLAGS + EXTRA).encode())
    return h.hexdigest()


def _compile(unit: str, verbose: bool) -> str:
    src = os.path.join(CSRC, unit)
    obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
    cmd = [NVCC, *ARCH, *FLAGS, *EXTRA, "-c", src, "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {unit}:\n{r.stderr}")
    return r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    stamp = os.path.join(BUILD, "stamp")
    dig = _digest()
    if not force and os.path.exists(LIB) and os.path.exists(stamp):
        with open(stamp) as f:
            if f.read().strip() == dig:
                return LIB
    with cf.ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        logs = list(ex.map(lambda u: _compile(u, verbose), UNITS))
    if verbose:
        for u, log in zip(UNITS, logs):
            with open(os.path.join(BUILD, u + ".ptxas.txt"), "w") as f:
                f.write(log)
    objs = [os.path.join(BUILD, u.replace(".cu", ".o")) for u in UNITS]
    tmp = LIB + ".tmp"
    r = subprocess.run([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    with open(stamp, "w") as f:
        f.write(dig)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
