"""Compiles the reference's own CUDA kernels (boojum-cuda native/*.cu, from /root/reference) plus
the C++ host driver oracle/ref_harness.cu into oracle/_ref/libbcref.so.

TEST INFRASTRUCTURE ONLY.  The reference's sources are compiled where they lie; nothing is
copied into this repository.  The Poseidon2 kernels need the constants header that the
reference generates at build time from boojum (build/poseidon2_gl.rs); this script fills the
reference's own template (poseidon2_gl_constants.cuh.template) with the round constants the
product library uses (its placeholder set, or the file named by GLC_P2_ROUND_CONSTANTS), in the
same {lo, hi} u32-pair format, under oracle/_ref/generated/.

Built like the reference's CMake project: separable compilation, --expt-relaxed-constexpr,
C++17; for sm_100a.  Outputs go to oracle/_ref/ only.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
REF_NATIVE = os.environ.get("GLC_REFERENCE_NATIVE", "/root/reference/crates/boojum-cuda/native")
OUT = os.path.join(HERE, "_ref")
GEN = os.path.join(OUT, "generated")
OBJ = os.path.join(OUT, "obj")
LIB = os.path.join(OUT, "libbcref.so")
SOURCES = ["context.cu", "ntt.cu", "ops_complex.cu", "poseidon2/gl/poseidon2_gl_st.cu",
           "poseidon2/gl/poseidon2_gl_mt.cu", "poseidon2/gl/poseidon2_gl_queries.cu"]
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "--expt-relaxed-constexpr", "-rdc=true",
         "-Xcompiler", "-fPIC", "-w"]


def round_constants() -> list[int]:
    path = os.environ.get("GLC_P2_ROUND_CONSTANTS")
    if path:
        text = open(path).read()
    else:
        text = open(os.path.join(REPO, "zksync-crypto-gpu_b200", "csrc", "p2_round_constants_placeholder.inc")).read()
        text = "\n".join(l for l in text.splitlines() if not l.lstrip().startswith("//"))
    vals = [int(t, 0) for t in re.findall(r"0[xX][0-9a-fA-F]+|\b\d+\b", text.replace("ull", ""))]
    if len(vals) != 360:
        raise ValueError("expected 360 round constants, found %d" % len(vals))
    return vals


def write_constants_header() -> None:
    tpl = open(os.path.join(REF_NATIVE, "poseidon2", "gl", "poseidon2_gl_constants.cuh.template")).read()
    vals = round_constants()
    rows = []
    for r in range(30):
        row = "".join("{%#010x,%#010x}," % (v & 0xFFFFFFFF, v >> 32) for v in vals[12 * r:12 * r + 12])
        rows.append("  {" + row + "},")
    text = tpl.replace("%RATE%", "8").replace("%CAPACITY%", "4").replace("%HALF_NUM_FULL_ROUNDS%", "4") \
        .replace("%NUM_PARTIAL_ROUNDS%", "22").replace("%ALL_ROUND_CONSTANTS%", "\n" + "\n".join(rows) + "\n")
    os.makedirs(GEN, exist_ok=True)
    with open(os.path.join(GEN, "poseidon2_gl_constants.cuh"), "w") as f:
        f.write(text)


def build() -> str:
    if not os.path.isdir(REF_NATIVE):
        raise FileNotFoundError("reference sources not found at %s" % REF_NATIVE)
    os.makedirs(OBJ, exist_ok=True)
    write_constants_header()
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    objs = []
    procs = []
    for src in SOURCES + ["@harness"]:
        path = os.path.join(HERE, "ref_harness.cu") if src == "@harness" else os.path.join(REF_NATIVE, src)
        obj = os.path.join(OBJ, os.path.basename(path) + ".o")
        objs.append(obj)
        cmd = [nvcc, *FLAGS, "-I", GEN, "-I", REF_NATIVE, "-c", path, "-o", obj]
        procs.append((path, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
    for path, p in procs:
        out, err = p.communicate()
        if p.returncode:
            raise RuntimeError("nvcc failed on %s\n%s\n%s" % (path, out, err))
    r = subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-rdc=true", "-shared", "-o", LIB, *objs],
                       capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError("link failed\n%s\n%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    print(build())
    sys.exit(0)
