"""Test infrastructure: embed an OP2 application's kernel headers in a C++
source that registers them with libop2b at start-up.

  python embed_kernels.py OUT.cpp [prelude=PATH ...] [NAME=PATH ...] [loops=PATH ...]

The reference's applications keep each loop's kernel in a header named after
it (apps/c/jac1/dp/res.h ...), which OP2's code generator turns into device
code before the application is built.  For the drop-in checks, oracle/Makefile
links the generated file into the unmodified application; its static
initialiser hands the sources to op2b_register_prelude / op2b_register_kernel,
and libop2b compiles each loop at its first call.  loops=PATH is for
programs that define their kernels in the main source (apps/c/min,
tests/functional/*): the definitions of every kernel an op_par_loop in PATH
names become one prelude (a kernel may call another), and each loop name is
registered as defined there.  The output goes to oracle/_ref/ (a build
product, never committed).
"""
import re
import sys


def function_text(src: str, func: str) -> str:
    """The definition of `func` in `src`: from its return type to the brace
    that closes its body."""
    m = re.search(r"^[^\n;{}]*\b" + re.escape(func) + r"\s*\([^)]*\)\s*\{", src, flags=re.M)
    if not m:
        raise SystemExit(f"embed_kernels: no definition of {func}")
    depth, i = 0, m.end() - 1
    while True:
        depth += {"{": 1, "}": -1}.get(src[i], 0)
        i += 1
        if depth == 0:
            return src[m.start():i] + "\n"


def c_bytes(data: bytes) -> str:
    return ",".join(str(b) for b in data) + ",0"


def main(argv):
    out, items = argv[0], [a.split("=", 1) for a in argv[1:]]
    lines = ['#include "op2b.h"', ""]
    regs = []
    for k, (name, path) in enumerate(items):
        with open(path, "rb") as f:
            data = f.read()
        if name == "loops":
            src = data.decode()
            loops = list(dict.fromkeys(re.findall(r"\bop_par_loop\s*\(\s*(\w+)\s*,", src)))
            data = "".join(function_text(src, f) for f in loops).encode()
        lines.append(f"static const char op2b_src_{k}[] = {{{c_bytes(data)}}};")
        if name == "loops":
            regs.append(f"    op2b_register_prelude(op2b_src_{k});")
            regs += [f'    op2b_register_kernel("{f}", "/* defined in the prelude */");'
                     for f in loops]
        elif name == "prelude":
            regs.append(f"    op2b_register_prelude(op2b_src_{k});")
        else:
            regs.append(f'    op2b_register_kernel("{name}", op2b_src_{k});')
    lines += ["", "namespace {", "struct RegisterKernels {", "  RegisterKernels() {", *regs,
              "  }", "} register_kernels;", "}  // namespace", ""]
    with open(out, "w") as f:
        f.write("\n".join(lines))


if __name__ == "__main__":
    main(sys.argv[1:])
