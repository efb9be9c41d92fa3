#!/usr/bin/env python3
"""Build oracle/_ref/libradm2_ref.so: the reference's own mechanism code, on the CPU.

TEST INFRASTRUCTURE ONLY (the checker's checker).

The reference (mgpu.cu) does not build with CUDA 12.9: it uses texture
references (mgpu.cu:201-203, 2748, 2812-2814) that CUDA 12 removed, and its
integrator's stage loop is commented out (mgpu.cu:3595-3625).  Its per-cell
mechanism kernels are, however, plain C once the CUDA qualifiers are shimmed.
This recipe cuts these functions out of mgpu.cu where it lies, unmodified:

    ARR2, TROE, TROEE, THERMAL_T2, k46      mgpu.cu:708-750
    dev_Update_RCONST                        mgpu.cu:752-919
    dev_Fun                                  mgpu.cu:1084-1386
    dev_Jac_SP                               mgpu.cu:1672-2652
    dev_KppDecomp                            mgpu.cu:2726-2780
    dev_KppSolve                             mgpu.cu:2854-3096
    dev_convert (WRF -> KPP conversion)      mgpu.cu:513-646

and compiles them with g++ for one cell per call, behind the shim in
oracle/ref_harness.cpp (CUDA qualifiers as no-ops, blockIdx/threadIdx as
host variables, the LU_DIAG/CROW/ICOL texture fetches as reads of the CSR
tables recovered from dev_KppSolve -- the reference never fills its own).
Outputs go to oracle/_ref/ only (git-ignored; the built .so travels with the
repository snapshot to machines that have no copy of the reference).

Usage:  python oracle/build_ref.py /path/to/mgpu.cu
        (or the path in the environment variable RADM2_REFERENCE_MGPU; without either, or
        when the file is absent, nothing is built and a prebuilt oracle/_ref is kept)
"""
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")

FUNCTIONS = [
    r"__device__\s+double\s+ARR2\s*\(",
    r"__device__\s+double\s+TROE\s*\(",
    r"__device__\s+double\s+TROEE\s*\(",
    r"__device__\s+double\s+THERMAL_T2\s*\(",
    r"__device__\s+double\s+k46\s*\(",
    r"__global__\s+void\s+dev_Update_RCONST\s*\(",
    r"__global__\s+void\s+dev_Fun\s*\(",
    r"__global__\s+void\s+dev_Jac_SP\s*\(",
    r"__global__\s+void\s+dev_KppDecomp\s*\(",
    r"__global__\s+void\s+dev_KppSolve\s*\(",
    r"__global__\s+void\s+dev_convert\s*\(",
]

# Object-like and function-like #defines from the reference's header block that the
# extracted functions use (sizes, species indices, min/max/abs macros).
DEFINE_RE = re.compile(r"^#define\s+(NSPEC|NVAR|NVARACT|NFIX|NREACT|NVARST|NFIXST|NONZERO|LU_NONZERO|CNVAR|NPH|"
                       r"navgdro|mwh|mwo|mwair|mwh2o|dens2con_a|dens2con_w|"
                       r"ind_\w+|indf_\w+|Pj_\w+|ZERO|ONE|TWO|HALF|THREE_HUNDRED|DeltaMin|MAX|MIN|ABS|SQRT)\b")


def function_text(src, signature):
    m = re.search(signature, src)
    if not m:
        raise SystemExit("not found in reference: " + signature)
    i = src.index("{", m.end())
    depth = 0
    for j in range(i, len(src)):
        if src[j] == "{":
            depth += 1
        elif src[j] == "}":
            depth -= 1
            if depth == 0:
                return src[m.start():j + 1]
    raise SystemExit("unbalanced braces: " + signature)


def main():
    src_path = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RADM2_REFERENCE_MGPU", "")
    if not src_path or not os.path.exists(src_path):
        print("reference not present (%s); keeping any prebuilt oracle/_ref" % src_path)
        return 0
    with open(src_path) as f:
        src = f.read()
    os.makedirs(OUT, exist_ok=True)
    header = [l for l in src.split("\n")[:200] if DEFINE_RE.match(l)]
    parts = ["/* Cut from %s by oracle/build_ref.py; not part of the repository. */" % src_path]
    parts += header
    parts.append("#define MY_I(i) (i)")
    for sig in FUNCTIONS:
        parts.append(function_text(src, sig))
    inc = os.path.join(OUT, "ref_extract.inc")
    with open(inc, "w") as f:
        f.write("\n".join(parts) + "\n")
    so = os.path.join(OUT, "libradm2_ref.so")
    cmd = ["g++", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-w", "-I", OUT,
           os.path.join(HERE, "ref_harness.cpp"), "-o", so]
    subprocess.check_call(cmd)
    print("built", so)
    return 0


if __name__ == "__main__":
    sys.exit(main())
