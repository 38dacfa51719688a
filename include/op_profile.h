/*
 * op_profile.h -- the reference's region profiler (op2/include/op_profile.h,
 * op2/src/externlib/op_profile.cpp:557-580: op_profile_start / enter /
 * enter_kernel / next / exit / end / output) for applications built against
 * libop2b.
 *
 * Regions form a tree under the name given to op_profile_start.  Each
 * region's time is device time on the library's stream, between CUDA events
 * recorded at its enter and exit (no device synchronisation at the
 * boundaries).  OP_PROFILE_LEVEL (read at op_profile_start) selects the
 * detail as in the reference: 0 off, 1 application regions (default), 2 and
 * 3 also one kernel node per op_par_loop under the region it ran in.
 * op_profile_output prints the tree; with OP_PROFILE_JSON_OUTPUT=<file> it
 * also writes it as JSON (the reference's node fields; times in ns).
 */
#ifndef OP2B_OP_PROFILE_H
#define OP2B_OP_PROFILE_H

#include "op2b.h"

#ifdef __cplusplus
extern "C" {
#endif

/* op_profile.cpp:557 -- open the root region (reads OP_PROFILE_LEVEL) */
void op_profile_start(const char *name);
/* op_profile.cpp:559 -- open a child region of the innermost open one */
void op_profile_enter(const char *name);
/* op_profile.cpp:560 -- open a kernel node "name/target/variant" (level >= 2) */
void op_profile_enter_kernel(const char *name, const char *target, const char *variant);
/* op_profile.cpp:564 -- close the innermost region and open a sibling */
void op_profile_next(const char *name);
/* op_profile.cpp:566 -- close the innermost region */
void op_profile_exit(void);
/* op_profile.cpp:567 -- close every open region, the root included */
void op_profile_end(void);
/* op_profile.cpp:569 -- print the tree (and write OP_PROFILE_JSON_OUTPUT) */
void op_profile_output(void);
/* op_profile.cpp:570 -- write the tree as JSON to `filename` */
void op_profile_output_json(const char *filename);

#ifdef __cplusplus
}
#endif

#endif /* OP2B_OP_PROFILE_H */
