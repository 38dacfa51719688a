"""Test infrastructure: embed an OP2 application's kernel headers in a C++
source that registers them with libop2b at start-up.

  python embed_kernels.py OUT.cpp [prelude=PATH ...] [NAME=PATH ...]

The reference's applications keep each loop's kernel in a header named after
it (apps/c/jac1/dp/res.h ...), which OP2's code generator turns into device
code before the application is built.  For the drop-in checks, oracle/Makefile
links the generated file into the unmodified application; its static
initialiser hands the sources to op2b_register_prelude / op2b_register_kernel,
and libop2b compiles each loop at its first call.  The output goes to
oracle/_ref/ (a build product, never committed).
"""
import sys


def c_bytes(data: bytes) -> str:
    return ",".join(str(b) for b in data) + ",0"


def main(argv):
    out, items = argv[0], [a.split("=", 1) for a in argv[1:]]
    lines = ['#include "op2b.h"', ""]
    regs = []
    for k, (name, path) in enumerate(items):
        with open(path, "rb") as f:
            lines.append(f"static const char op2b_src_{k}[] = {{{c_bytes(f.read())}}};")
        if name == "prelude":
            regs.append(f"    op2b_register_prelude(op2b_src_{k});")
        else:
            regs.append(f'    op2b_register_kernel("{name}", op2b_src_{k});')
    lines += ["", "namespace {", "struct RegisterKernels {", "  RegisterKernels() {", *regs,
              "  }", "} register_kernels;", "}  // namespace", ""]
    with open(out, "w") as f:
        f.write("\n".join(lines))


if __name__ == "__main__":
    main(sys.argv[1:])
