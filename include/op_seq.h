/*
 * op_seq.h -- drop-in replacement of the reference's op2/include/op_seq.h
 * for applications that call op_par_loop(kernel, name, set, args...).
 *
 * The reference header runs the user's kernel on the host over every set
 * element (op_seq.h:30-3881).  Here op_par_loop hands the argument list to
 * libop2b (op_par_loop_c), which runs the device loop registered under
 * `name` after checking the arguments against its signature; the host kernel
 * pointer is not called.  A loop without a device implementation, or with a
 * mismatching argument list, prints the library's message and exits, as the
 * reference's error paths do.
 */
#ifndef OP2B_OP_SEQ_H
#define OP2B_OP_SEQ_H

#include "op_lib_cpp.h"

template <typename... K, typename... A>
void op_par_loop(void (*kernel)(K *...), char const *name, op_set set, A... arguments) {
  (void)kernel;
  op_arg args[sizeof...(A) > 0 ? sizeof...(A) : 1] = {arguments...};
  if (op_par_loop_c(name, set, (int)sizeof...(A), args) != 0) {
    printf("op_par_loop(%s) error -- %s\n", name, op2b_last_error());
    exit(-1);
  }
}

#endif /* OP2B_OP_SEQ_H */
