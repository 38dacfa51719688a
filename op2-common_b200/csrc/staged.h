// Indirect-increment loops (res_calc, bres_calc) in their three strategies
// and the plans they use.  Internal to libop2b.
#pragma once

#include "loops.h"
#include "op2b.h"

namespace op2b {

struct Plan;

template <typename T> struct ResCalcArgs {
  int nedge;
  const int *pedge, *pecell;
  const T *x, *q, *adt;
  T *res;
  AirConst<T> k;
};

template <typename T> struct BresCalcArgs {
  int nbedge;
  const int *pbedge, *pbecell, *bound;
  const T *x, *q, *adt;
  T *res;
  AirConst<T> k;
};

// Plan for the loop (built on the device on first use, then cached):
// OP_STAGE_ALL with the reference translator's `inds` for the loop.
Plan *get_res_plan(const char *name, op_set set, int nargs, op_arg *args);
Plan *get_bres_plan(const char *name, op_set set, int nargs, op_arg *args);

// mode: OP2B_INC_ATOMIC, OP2B_INC_COLOR or OP2B_INC_HYBRID
template <typename T>
cudaError_t run_res_calc(const LaunchCtx &c, const ResCalcArgs<T> &a, Plan *plan, int mode);
template <typename T>
cudaError_t run_bres_calc(const LaunchCtx &c, const BresCalcArgs<T> &a, Plan *plan, int mode);

}  // namespace op2b
