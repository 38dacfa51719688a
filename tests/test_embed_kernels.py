"""oracle/embed_kernels.py: the registration file it writes for programs
whose kernels live in headers or in the main source."""
import os
import re
import subprocess
import sys
import tempfile

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SCRIPT = os.path.join(REPO, "oracle", "embed_kernels.py")

MAIN = r'''
#include "op_seq.h"
void helper(double *v) { *v += 1.0; }
void first(double *v, const double *w) {
  if (*w > 0) { helper(v); }
}
int main() {
  op_par_loop(first, "first", s, op_arg_dat(d, -1, OP_ID, 1, "double", OP_RW));
  op_par_loop(first, "first", s, op_arg_dat(d, -1, OP_ID, 1, "double", OP_RW));
  op_par_loop(second, "second", s);
}
void second(int *i) { *i = 0; }
'''


def _strings(src):
    """The C strings of the generated file, decoded from their byte lists."""
    return [bytes(int(b) for b in body.split(",")[:-1]).decode()
            for body in re.findall(r"\[\] = \{([^}]*)\};", src)]


def test_loops_mode_takes_every_named_kernel_from_the_source():
    with tempfile.TemporaryDirectory() as tmp:
        main = os.path.join(tmp, "app.cpp")
        out = os.path.join(tmp, "reg.cpp")
        open(main, "w").write(MAIN)
        subprocess.run([sys.executable, SCRIPT, out, f"loops={main}"], check=True)
        src = open(out).read()
    (prelude,) = _strings(src)
    # each kernel named by an op_par_loop once, in order of first use, whole
    assert prelude.index("void first(") < prelude.index("void second(")
    assert prelude.count("void first(") == 1 and "{ helper(v); }\n}" in prelude
    assert "void helper(" not in prelude and "int main" not in prelude
    assert "op2b_register_prelude(op2b_src_0);" in src
    assert re.findall(r'op2b_register_kernel\("(\w+)"', src) == ["first", "second"]


def test_header_mode_registers_files_under_their_names():
    with tempfile.TemporaryDirectory() as tmp:
        h = os.path.join(tmp, "res.h")
        t = os.path.join(tmp, "user_types.h")
        open(h, "w").write("inline void res(double *a) { *a = 1.0; }\n")
        open(t, "w").write("typedef double real;\n")
        out = os.path.join(tmp, "reg.cpp")
        subprocess.run([sys.executable, SCRIPT, out, f"prelude={t}", f"res={h}"], check=True)
        src = open(out).read()
    assert _strings(src) == ["typedef double real;\n", "inline void res(double *a) { *a = 1.0; }\n"]
    assert "op2b_register_prelude(op2b_src_0);" in src
    assert 'op2b_register_kernel("res", op2b_src_1);' in src
