/*
 * op_lib_c.h -- the name under which OP2 applications include the C API
 * (op2/include/op_lib_c.h), mapped onto libop2b's C ABI (op2b.h).
 */
#ifndef OP2B_OP_LIB_C_H
#define OP2B_OP_LIB_C_H

#include <math.h>
#include <stdio.h>

#include "op2b.h"
#include "op_hdf5.h" /* as op2/include/op_lib_c.h:131 */

#endif /* OP2B_OP_LIB_C_H */
