/*
 * op_profile.h -- the profiling calls of the reference
 * (op2/include/op_profile.h: op_profile_start/enter/next/exit/end/output) for
 * applications built against libop2b.  Region timing is not kept; every
 * loop's device time is recorded by the library with CUDA events and
 * op_profile_output prints that table (op_timing_output).
 */
#ifndef OP2B_OP_PROFILE_H
#define OP2B_OP_PROFILE_H

#include "op2b.h"

inline void op_profile_start(const char *) {}
inline void op_profile_enter(const char *) {}
inline void op_profile_enter_kernel(const char *, const char *, const char *) {}
inline void op_profile_next(const char *) {}
inline void op_profile_exit() {}
inline void op_profile_end() {}
inline void op_profile_output() { op_timing_output(); }

#endif /* OP2B_OP_PROFILE_H */
