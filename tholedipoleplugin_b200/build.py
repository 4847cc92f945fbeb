"""Builds the in-tree shared library libtholedipole_b200.so with nvcc for
sm_100a (B200).  The library is the product: the C ABI of
include/tholedipole_b200.h over the hand-written kernels in csrc/."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libtholedipole_b200.so")
SOURCES = ["tdp_kernels.cu", "tdp_sym.cu", "tdp_ewald.cu", "tdp_capi.cu", "tdp_md.cu", "tdp_noalloc.cu",
           "tdp_adjoint.cu", "tdp_batch.cu", "tdp_precond.cu"]
# Sources whose FP32 pair arithmetic is compiled with subnormal flushing.
FTZ = {"tdp_kernels.cu", "tdp_sym.cu", "tdp_ewald.cu", "tdp_batch.cu"}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    inc = os.path.join(ROOT, "include")
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(inc, f) for f in os.listdir(inc)]
    return any(os.path.getmtime(d) > t for d in deps if os.path.isfile(d))


def _adapter_stale() -> bool:
    outs = [ADAPTER_LIB, ADAPTER_DRIVER]
    if not all(os.path.exists(o) for o in outs):
        return True
    t = min(os.path.getmtime(o) for o in outs)
    deps = [LIB] + [os.path.join(dp, f) for dp, _, fs in os.walk(ADAPTER) for f in fs]
    return any(os.path.getmtime(d) > t for d in deps if os.path.isfile(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        if _adapter_stale():
            build_adapter(verbose)
        return LIB
    objs = []
    build_dir = os.path.join(HERE, "_build")
    os.makedirs(build_dir, exist_ok=True)
    common = [nvcc(), "-std=c++17", "-O3", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "-I", os.path.join(ROOT, "include"), "-I", CSRC]
    for src in SOURCES:
        obj = os.path.join(build_dir, src.replace(".cu", ".o"))
        # The pair kernels never see subnormal FP32 operands (squared distances
        # are >= ~1e-4 nm^2 or masked to +inf), so flushing subnormals removes
        # the fix-up around every reciprocal square root.
        extra = ["-ftz=true"] if src in FTZ else []
        cmd = common + extra + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart", "-lcufft"], check=True)
    os.replace(tmp, LIB)
    build_adapter(verbose)
    return LIB


ADAPTER = os.path.join(HERE, "openmm_adapter")
ADAPTER_LIB = os.path.join(HERE, "libtholedipole_b200_openmm.so")
ADAPTER_DRIVER = os.path.join(HERE, "_build", "adapter_driver")


def build_adapter(verbose: bool = False) -> str:
    """The OpenMM-facing kernel adapter (CudaCalcTholeDipoleForceKernel, its
    factory and registration symbols) over the C ABI, built here against the
    OpenMM stand-in headers, plus its test driver."""
    inc = ["-I", os.path.join(ADAPTER, "standin"), "-I", os.path.join(ADAPTER, "plugin"), "-I", ADAPTER,
           "-I", os.path.join(ROOT, "include")]
    srcs = [os.path.join(ADAPTER, f) for f in ("CudaTholeDipoleKernels.cpp", "CudaTholeDipoleKernelFactory.cpp")]
    srcs += [os.path.join(ADAPTER, "plugin", "TholeDipoleForce.cpp"), os.path.join(ADAPTER, "standin", "openmm_standin.cpp")]
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", *inc, "-o", ADAPTER_LIB, *srcs, "-L", HERE,
           "-ltholedipole_b200", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.makedirs(os.path.dirname(ADAPTER_DRIVER), exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O2", *inc, "-o", ADAPTER_DRIVER, os.path.join(ADAPTER, "adapter_driver.cpp"),
           "-L", HERE, "-ltholedipole_b200_openmm", "-ltholedipole_b200", "-Wl,-rpath," + HERE]
    subprocess.run(cmd, check=True)
    return ADAPTER_LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
