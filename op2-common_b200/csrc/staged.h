// Indirect-increment loops (res_calc) in their three strategies and the
// execution plans they use.  Internal to libop2b.
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

// Plan for the loop (built on the device on first use, then cached).
const Plan *get_res_plan(const char *name, op_set set, int nargs, op_arg *args);

template <typename T>
cudaError_t run_res_calc(const LaunchCtx &c, const ResCalcArgs<T> &a, const Plan *plan, int mode);

}  // namespace op2b
