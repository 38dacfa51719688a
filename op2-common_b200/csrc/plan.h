// Internal representation of a GPU-built execution plan (plan.cu).
#pragma once

#include <string>
#include <vector>

#include "op2b_plan.h"

namespace op2b {

struct Plan {
  // identity (what op_plan_core matches a cached plan on, :314-347)
  std::string name;
  op_set set = nullptr;
  int nargs = 0, ninds = 0, part_size = 0, staging = 0, bsize = 0;
  int colouring = 0;      // OP2B_COLOUR_GREEDY or OP2B_COLOUR_JP
  int colour_rounds = 0;  // Jones-Plassmann rounds run (0 for the greedy order)
  std::vector<op_dat> dats;
  std::vector<op_map> maps;
  std::vector<int> idxs, accs, optflags, inds;

  // device arrays
  int *thrcol_d = nullptr, *nthrcol_d = nullptr, *blk_col_d = nullptr, *blkmap_d = nullptr;
  int *ind_map_d = nullptr, *ind_offs_d = nullptr, *ind_sizes_d = nullptr;
  short *loc_map_d = nullptr;
  int *col_reord_d = nullptr;  // OP_STAGE_PERMUTE / OP_COLOR2: elements by thread colour
  std::vector<void *> owned;
  double build_ms = 0.0;
  int max_ind_size[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // per staged slot, max over blocks
  long long col_offsets_len = 0;
  std::vector<char> params_blob;  // the PlanParams the kernels ran with
  // per staged indirection: 1 where a listed target is also listed by
  // another block (built on first request, for the staged-hybrid loops)
  std::vector<unsigned char *> shared_d;

  // host copies behind the public struct
  op_plan pub{};
  std::string name_store;
  std::vector<int> h_offset, h_nelems, h_thrcol, h_nthrcol, h_blkmap, h_ncolblk, h_nsharedCol;
  std::vector<int> h_ind_map, h_ind_offs, h_ind_sizes, h_nindirect, h_inds_staged;
  std::vector<int *> h_ind_maps;
  std::vector<short> h_loc_map;
  std::vector<short *> h_loc_maps;
  std::vector<int> h_col_reord, h_col_offsets_flat;
  std::vector<int *> h_col_offsets;

  ~Plan();
};

// colouring: the reference's serial greedy order (bit-exact integers) or
// Jones-Plassmann rounds (parallel, validated conflict-free)
enum { OP2B_COLOUR_GREEDY = 0, OP2B_COLOUR_JP = 1 };
Plan *build_plan(const char *name, op_set set, int part_size, int nargs, op_arg *args,
                 int ninds, int *inds, int staging, int colouring = OP2B_COLOUR_GREEDY);
const Plan *find_plan(const op_plan *o);
int validate_plan(const Plan &pl, long detail[8]);
// shared flags of staged indirection `slot`, aligned with its ind_map entries
const unsigned char *plan_shared_flags(Plan &pl, int slot);
// device pointer to the start of staged indirection `slot`'s ind_map
const int *plan_ind_map_slot(const Plan &pl, int slot);
// max over blocks of ind_sizes of staged indirection `slot`
int plan_max_ind_size(const Plan &pl, int slot);

}  // namespace op2b
