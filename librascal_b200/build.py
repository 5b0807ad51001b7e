"""Build the in-tree shared library librascal_b200/_lib/librascal_b200.so.

Compiles the CUDA kernels and the C++ host code for sm_100a with nvcc and
links them into one C-ABI library (include/rascal_b200.h). Usage:

    python -m librascal_b200.build          # or: python librascal_b200/build.py

Objects are rebuilt only when a source or header is newer than the object.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "librascal_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# (source, extra flags). The neighbour list and the host spline builder are
# compiled without FMA contraction so their FP64 results are reproducible
# bit for bit against the CPU restatement.
SOURCES = [
    ("nl.cu", ["--fmad=false"], "nl"),
    ("util.cu", [], "util"),
    ("expansion.cu", ["--fmad=false", "-DRGPU_PART_FP64"], "expansion_f64"),
    ("expansion.cu", ["-DRGPU_PART_FP32"], "expansion_f32"),
    ("powerspectrum.cu", ["--fmad=false", "-DRGPU_PART_FP64"], "powerspectrum_f64"),
    ("ps_fast.cu", [], "ps_fast"),
    ("ps_tc.cu", [], "ps_tc"),
    ("gemm.cu", [], "gemm"),
    ("gemm_tc.cu", [], "gemm_tc"),
    ("noalloc.cu", [], "noalloc"),
    ("peaks.cu", [], "peaks"),
    # the adjoint's instantiations unroll the spherical-harmonics recurrence
    # per max_angular: four translation units by range of L, compiled in
    # parallel (the first also holds the dispatch)
    ("adjoint.cu", ["-DRGPU_ADJ_L0=0", "-DRGPU_ADJ_L1=6", "-DRGPU_ADJ_DISPATCH"], "adjoint_l0"),
    ("adjoint.cu", ["-DRGPU_ADJ_L0=7", "-DRGPU_ADJ_L1=9"], "adjoint_l7"),
    ("adjoint.cu", ["-DRGPU_ADJ_L0=10", "-DRGPU_ADJ_L1=11"], "adjoint_l10"),
    ("adjoint.cu", ["-DRGPU_ADJ_L0=12", "-DRGPU_ADJ_L1=12"], "adjoint_l12"),
    ("training.cu", [], "training"),
    ("api.cu", [], "api"),
    ("radial_gto.cpp", ["-Xcompiler", "-ffp-contract=off"], "radial_gto"),
    ("json_lite.cpp", [], "json_lite"),
]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "--extended-lambda", "-I" + SRC, "-I" + os.path.join(os.path.dirname(HERE), "include")]


def _headers():
    hs = [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(os.path.dirname(HERE), "include", "rascal_b200.h"))
    return hs


def build(verbose=False, jobs=None):
    os.makedirs(OUT, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    newest_header = max(os.path.getmtime(h) for h in _headers())
    procs, objs = [], []
    for src, flags, name in SOURCES:
        s = os.path.join(SRC, src)
        o = os.path.join(OBJ, name + ".o")
        objs.append(o)
        if os.path.exists(o) and os.path.getmtime(o) >= max(os.path.getmtime(s), newest_header):
            continue
        if src.endswith(".cu"):
            cmd = [NVCC] + ARCH + COMMON + flags + ["-c", s, "-o", o]
        else:
            cmd = [NVCC] + COMMON + flags + ["-x", "c++", "-c", s, "-o", o]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out.decode()))
        elif verbose and out:
            print(out.decode())
    if failed:
        msg = "\n".join("--- %s ---\n%s" % f for f in failed)
        raise RuntimeError("nvcc failed:\n" + msg)
    if procs or not os.path.exists(LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
