// Inverse maps and the owner-computes ("gather") indirect loops.  Internal.
#pragma once

#include "loops.h"
#include "op2b.h"

namespace op2b {

// Inverse of a map from -> to: for target t, entries off[t] .. off[t+1]-1 of
// ent hold element*dim + slot of every (element, slot) mapping to t, sorted
// ascending.  rows lists the targets with at least one entry (all targets
// when all_rows).
struct InvMap {
  const long long *off;
  const int *ent;
  const int *rows;
  int nrows, nto, dim;
  bool all_rows;
};

const InvMap *get_inverse_map(op_map map);
void release_inverse_maps();

template <typename T>
cudaError_t launch_res_calc_gather(const LaunchCtx &c, const InvMap &inv, const int *pedge,
                                   const int *pecell, const T *x, const T *q, const T *adt,
                                   T *res, const AirConst<T> &k);
template <typename T>
cudaError_t launch_bres_calc_gather(const LaunchCtx &c, const InvMap &inv, const int *pbedge,
                                    const int *bound, const T *x, const T *q, const T *adt,
                                    T *res, const AirConst<T> &k);

}  // namespace op2b
