"""Writes the reference's OpenCL kernel sources out as C++ translation units.
TEST INFRASTRUCTURE ONLY (run by oracle/Makefile; outputs under oracle/_ref/).

The reference keeps each OpenCL program as a C++ raw string literal in
include/Aster/kernels/*.cl.h. This copies the text of the three programs its
OpenCL Barnes-Hut solver (BH_hyper, src/solvers/full_GPU.cpp:152-168) builds
its tree with into <out>/<namespace>.cpp, after the OpenCL-C shim
(cl_c_shim.h) and inside a namespace of its own, so that the kernels compile
with g++ and run on the CPU under cl_runner.cpp's work-group emulator.

One textual change: in the bitonic start kernel the work-group array
`__local ulong local_buffer` becomes `static ulong local_buffer`, one copy
shared by the work-items of the group the emulator is running (what __local
means); everything else is the reference's text.

usage: python extract_cl.py <reference source tree> <output directory>
"""
import re
import sys
from pathlib import Path

PROGRAMS = [  # (file under include/Aster/kernels, string variable, namespace)
    ("morton_writer.cl.h", "morton_writer3d", "clk_morton"),
    ("radix.cl.h", "radix_cl", "clk_radix"),
    ("BHH_specific.cl.h", "BHH_tree_cl3d", "clk_tree"),
]


def main(ref: str, out: str) -> None:
    outdir = Path(out)
    outdir.mkdir(parents=True, exist_ok=True)
    for fname, var, ns in PROGRAMS:
        text = (Path(ref) / "include" / "Aster" / "kernels" / fname).read_text()
        m = re.search(r"std::string\s+" + var + r'\s*=\s*R"CLC\((.*?)\)CLC"', text, re.S)
        if m is None:
            raise SystemExit(f"{fname}: no raw string {var}")
        src = m.group(1)
        if ns == "clk_radix":
            if src.count("__local ulong local_buffer") != 1:
                raise SystemExit("radix.cl.h: expected one __local ulong local_buffer")
            src = src.replace("__local ulong local_buffer", "static ulong local_buffer")
        (outdir / f"{ns}.cpp").write_text(
            f'#include "cl_c_shim.h"\nnamespace {ns} {{\n#line 1 "{fname}:{var}"\n{src}\n}}  // namespace {ns}\n')


if __name__ == "__main__":
    if len(sys.argv) != 3:
        raise SystemExit(__doc__)
    main(sys.argv[1], sys.argv[2])
