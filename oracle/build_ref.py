#!/usr/bin/env python3
"""Build recipe for oracle/_ref/libclref.so: the reference's own kernel on the CPU.

TEST INFRASTRUCTURE ONLY.  Reads the reference sources where they lie (under the
reference checkout given by --reference, else the LP_REFERENCE_DIR environment
variable, else /root/reference) and writes every output into oracle/_ref/, which is
git-ignored.  Nothing is copied into the repository's history.  reference_dir() is
the one place the default location is named; the tests and the build step ask it.

Steps
  1. src/Simulation/MCLightPropagation.cl is read and the OpenCL vector literals
     ``(floatN)(a, b, ...)`` / ``(intN)(...)`` are rewritten to C++ constructor calls
     ``floatN(a, b, ...)``.  That is the only change: in C++ the original spelling
     would parse as a cast of a comma expression.  The result is written to
     oracle/_ref/MCLightPropagation_cpu.cpp.
  2. g++ compiles oracle/ref_entry.cpp, which includes oracle/clshim.hpp (OpenCL
     built-ins as C++) and the rewritten kernel inside ``namespace clref``, together
     with src/PSNR/PSNR.cpp compiled unchanged, into oracle/_ref/libclref.so.
Compiler flags match oracle/Makefile (-O2 -ffp-contract=off, no fast-math) so the
reference build and the restatement round identically.
"""
import argparse
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")

VEC_LITERAL = re.compile(r"\((u?(?:char|short|int|long|float|double)(?:2|3|4|8|16))\)\s*\(")


def reference_dir() -> str:
    """The reference checkout: $LP_REFERENCE_DIR, else /root/reference."""
    return os.environ.get("LP_REFERENCE_DIR") or "/root/reference"


def reference_present(root: str = "") -> bool:
    return os.path.isfile(os.path.join(root or reference_dir(), "src", "Simulation", "MCLightPropagation.cl"))


def rewrite(src: str) -> str:
    return VEC_LITERAL.sub(lambda m: m.group(1) + "(", src)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=reference_dir())
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    cl = os.path.join(a.reference, "src", "Simulation", "MCLightPropagation.cl")
    psnr_dir = os.path.join(a.reference, "src", "PSNR")
    if not os.path.isfile(cl):
        print(f"build_ref: reference kernel not found at {cl} (set LP_REFERENCE_DIR); the live pin "
              f"oracle/_ref is not built, the committed fixtures in tests/golden/ still pin the oracle",
              file=sys.stderr)
        return 0
    os.makedirs(OUT, exist_ok=True)
    so = os.path.join(OUT, "libclref.so")
    inputs = [cl, os.path.join(psnr_dir, "PSNR.cpp"), os.path.join(HERE, "ref_entry.cpp"),
              os.path.join(HERE, "clshim.hpp"), os.path.abspath(__file__)]
    if (not a.force and os.path.isfile(so)
            and os.path.getmtime(so) >= max(os.path.getmtime(p) for p in inputs)):
        return 0
    with open(cl, "r", encoding="utf-8", errors="replace") as f:
        src = f.read()
    cpu_src = os.path.join(OUT, "MCLightPropagation_cpu.cpp")
    with open(cpu_src, "w") as f:
        f.write(rewrite(src))
    flags = ["-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-std=c++14", "-w"]
    cmd = [os.environ.get("CXX", "g++"), *flags, "-shared", "-o", so,
           f"-DLP_CL_SOURCE=\"{cpu_src}\"",
           f"-DLP_PSNR_HEADER=\"{os.path.join(psnr_dir, 'PSNR.hpp')}\"",
           "-I", HERE,
           os.path.join(HERE, "ref_entry.cpp"),
           os.path.join(psnr_dir, "PSNR.cpp")]
    print(" ".join(cmd))
    subprocess.check_call(cmd)
    return 0


if __name__ == "__main__":
    sys.exit(main())
