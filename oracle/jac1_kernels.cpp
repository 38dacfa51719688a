// Test infrastructure: the drop-in check of a second OP2 application.
//
// The reference's jac1 application (apps/c/jac1/dp/jac.cpp) is compiled,
// unmodified, against this repository's headers and linked with libop2b.so
// and with this file.  Its loops (res, update) have no hand-written device
// kernel; this object registers the application's own kernel headers
// (res.h, update.h, user_types.h -- embedded by oracle/Makefile from the
// reference tree when the binary is built) at start-up, where OP2's code
// generator would have produced their device code, and libop2b compiles them
// at their first op_par_loop call.
#include "op2b.h"

extern "C" const char op2b_jac1_res_h[], op2b_jac1_update_h[], op2b_jac1_user_types_h[];

namespace {
struct RegisterJac1Kernels {
  RegisterJac1Kernels() {
    op2b_register_prelude(op2b_jac1_user_types_h);
    op2b_register_kernel("res", op2b_jac1_res_h);
    op2b_register_kernel("update", op2b_jac1_update_h);
  }
} register_jac1_kernels;
}  // namespace
