"""Build libds_b200.so (CUDA kernels for sm_100a + host C++ + C ABI) in-tree.

    python -m parallel_ds_b200.build          # library
    python -m parallel_ds_b200.build --all    # library + the CPU oracle (tests)

nvcc cross-compiles for sm_100a without a GPU.  Floating-point contraction is
off (-fmad=false on the device, -ffp-contract=off on the host) wherever the
arithmetic decides indices or is compared bit for bit with the reference's
x86-64 build (the iteration kernels, the factorisations, the single-kernel
entry points): every multiply and add rounds on its own there.  The PDHG
warm start, the scorer network and the batched solver are checked against
their restatements within tolerances, so they keep fused multiply-adds
(FMA_TRANSLATION_UNITS).
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libds_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOST_CXX = "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# translation units compiled with fused multiply-adds (all others: -fmad=false)
FMA_TRANSLATION_UNITS = {"pdhg.cu", "mlp.cu", "batch.cu"}
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-ccbin", HOST_CXX,
                     "-Xcompiler", "-fPIC,-fopenmp,-ffp-contract=off",
                     "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills",
                     "-I", os.path.join(ROOT, "include")]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off",
             "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    return r.stdout + r.stderr


def sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    return cu, cpp


def _stale(obj, src, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + deps)


def build(verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    cu, cpp = sources()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "ds_api.h"))
    objs = []
    for f in cu:
        src, obj = os.path.join(CSRC, f), os.path.join(OBJ, f + ".o")
        if _stale(obj, src, headers):
            fmad = [] if f in FMA_TRANSLATION_UNITS else ["-fmad=false"]
            out = _run([NVCC] + NVCC_FLAGS + fmad + ["-c", src, "-o", obj])
            if verbose and out.strip():
                print(out)
        objs.append(obj)
    for f in cpp:
        src, obj = os.path.join(CSRC, f), os.path.join(OBJ, f + ".o")
        if _stale(obj, src, headers):
            _run([HOST_CXX] + CXX_FLAGS + ["-c", src, "-o", obj])
        objs.append(obj)
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        _run([NVCC] + ARCH + ["-shared", "-ccbin", HOST_CXX, "-o", LIB] + objs + ["-lgomp"])
    return LIB


def build_oracle():
    out = _run(["make", "-C", os.path.join(ROOT, "oracle")])
    ref = os.environ.get("DS_REFERENCE_ROOT", "/root/reference")
    if os.path.exists(os.path.join(ref, "src", "gpu", "cudaKernels.cu")):
        # the reference's own kernels, the same-box per-kernel baseline (oracle/_ref)
        out += _run(["make", "-C", os.path.join(ROOT, "oracle"), "ref", "REF=" + ref])
    return out


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    if "--all" in sys.argv:
        build_oracle()
    print(LIB)
