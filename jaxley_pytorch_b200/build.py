"""Build libjxb in-tree with nvcc for sm_100a (`python -m jaxley_pytorch_b200.build`)."""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

_HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(_HERE)
CSRC = os.path.join(_HERE, "csrc")
OUT_DIR = os.path.join(_HERE, "_build")
LIB = os.path.join(OUT_DIR, "libjxb.so")

NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
    # float32: denormals flush to zero, so the reciprocal and exp2 approximations
    # run without their denormal fix-ups (the simulated quantities are far from the
    # denormal range; float64 is unaffected).
    "-ftz=true",
]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


INST = "jxb_sim_inst.cu"  # compiled once per (element type, kind, CTA size class)


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def units():
    """`(source, object, extra flags)` of every compilation unit."""
    out = []
    for src in sources():
        base = os.path.basename(src)[:-3]
        if os.path.basename(src) != INST:
            out.append((src, os.path.join(OUT_DIR, base + ".o"), []))
            continue
        for tname, tag in (("float", "f32"), ("double", "f64")):
            for bwd, kind in ((0, "fwd"), (1, "bwd")):
                # 384: float adjoint CTAs of 12 warps, two per SM with up to 80 registers
                for nt in (256, 384, 512, 1024) if (tag, kind) == ("f32", "bwd") else (256, 512, 1024):
                    fn = f"sim_kernel_{tag}_{kind}_{nt}"
                    out.append((src, os.path.join(OUT_DIR, f"{base}_{tag}_{kind}_{nt}.o"),
                                [f"-DJXB_INST_T={tname}", f"-DJXB_INST_BWD={bwd}",
                                 f"-DJXB_INST_NT={nt}", f"-DJXB_INST_FN={fn}"]))
    return out


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h")))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in sources() + headers())


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    jobs = []
    for src, obj, flags in units():
        cmd = [_nvcc(), *NVCC_FLAGS, *extra, *flags, "-I", os.path.join(ROOT, "include"), "-I", CSRC,
               "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        jobs.append(cmd)
    with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as pool:
        for r in pool.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs):
            if verbose or r.returncode:
                sys.stdout.write(r.stdout)
                sys.stderr.write(r.stderr)
            if r.returncode:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    objs = [obj for _, obj, _ in units()]
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", tmp,
           "-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
    print(LIB)
