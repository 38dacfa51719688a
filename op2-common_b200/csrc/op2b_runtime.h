// Internal state of libop2b's host runtime.  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "loops.h"
#include "op2b.h"

namespace op2b {

struct LoopStat {
  double total_ms = 0.0;  // summed CUDA-event device time
  double last_ms = 0.0;
  double bytes_per_call = 0.0;  // algorithmic bytes of one call
  double plan_ms = 0.0;   // plan construction time (device)
  long calls = 0;
  long timed = 0;
};

struct PendingTime {
  std::string name;     // the loop whose statistics take the time ("" for none)
  cudaEvent_t e0, e1;
  int node = -1;        // the profiler's region or kernel node that takes it too
};

struct Plan;  // plan.h

// A loop call whose launch is deferred to the next library call, so that it
// can be fused with the loop that follows it (save_soln into adt_calc,
// res_calc with bres_calc).  Any other call launches it first, alone.
struct PendingLoop {
  int kind = 0;  // 0 none, 1 save_soln, 2 res_calc
  op_set set = nullptr;
  op_dat src = nullptr, dst = nullptr;  // save_soln: q (read), qold (written)
  op_map pedge = nullptr, pecell = nullptr;
  op_dat x = nullptr, q = nullptr, adt = nullptr, res = nullptr;  // res_calc
  int rb = 0;           // bytes per real (8 double, 4 float)
  double bytes = 0.0;   // algorithmic bytes of the deferred call
  AirConst<double> kd{};
  AirConst<float> kf{};
};

// Speculative adt_calc: update also computes, for the adt_calc that usually
// follows it (over the last adt_calc's arguments), the time step of its new q
// and writes it into `shadow`, a second array of adt's size.  While `inplace`
// holds, shadow is the program's next adt: the matching adt_calc then only
// swaps the two arrays (the adt dat takes shadow's, shadow the old one), and
// any other call drops the early values (restore_spec), so nothing observes
// them; the adt dat's array was not written.
// save_soln by renaming: save_soln (q -> qold) launches nothing; qold is
// taken to hold q's values until q changes.  Loops that only read q run
// meanwhile.  The update that reads qold and writes q then reads q's array
// and writes qold's, and the two dats swap arrays: q holds the new solution
// and qold the saved one, with no copy.  Any other call first makes the copy
// (materialize_save).
struct LazySave {
  op_dat src = nullptr, dst = nullptr;  // q, qold
};

struct SpecAdt {
  op_map pcell = nullptr;                               // the last adt_calc's arguments
  op_dat x = nullptr, q = nullptr, adt = nullptr;
  int rb = 0;
  bool inplace = false;    // shadow holds the next adt_calc's result
  void *shadow = nullptr;  // device buffer of adt's allocation size
  size_t shadow_bytes = 0;
  AirConst<double> kd{};   // constants the early adt was computed with
  AirConst<float> kf{};
};

// Speculative res_calc + bres_calc.  After an update that computed the
// next adt_calc ahead (SpecAdt), Airfoil calls adt_calc, res_calc and
// bres_calc with the arguments of the last fused res_calc + bres_calc pair.
// The update call launches that pair right behind the update kernel, before
// it waits for the update's gbl results, so the GPU never idles on the
// host's round trip.  The update left res zero, so the launch is undone by
// zeroing res.  `stage` follows the program: 1 launched, 2 res_calc called
// with the learned arguments (bres_calc pending); 0 when bres_calc matched
// too or nothing was launched.  Any other call settles it first
// (settle_res): res back to zero, and at stage 2 res_calc deferred again.
struct ResLearn {
  bool valid = false;
  op_set eset = nullptr, bset = nullptr;
  op_map pedge = nullptr, pecell = nullptr, pbedge = nullptr, pbecell = nullptr;
  op_dat x = nullptr, q = nullptr, adt = nullptr, res = nullptr, bound = nullptr;
  int rb = 0;
  double res_bytes = 0.0, fused_bytes = 0.0;
  double res_read_bytes = 0.0;  // the pair's read of res, saved when res is known zero
  AirConst<double> kd{};  // constants of the learned (and the launched) pair
  AirConst<float> kf{};
};

struct Runtime {
  ~Runtime() {
    if (stage_alloc.joinable()) stage_alloc.join();
  }
  bool initialised = false;
  int device = 0, nsm = 148, cc_major = 0, cc_minor = 0;
  cudaStream_t stream = nullptr, own_stream = nullptr;
  long launches = 0;

  // options (argv tokens of op_set_args, env, op2b_set_option)
  int opt_diags = 0;
  bool opt_abort = false;
  bool opt_timing = true;
  int opt_timing_stride = 16;  // time one call in this many of each loop (1: every call)
  int opt_block_size = 0;
  int opt_part_size = 0;
  int opt_cache_line = 128;
  int opt_maps_base = 0;
  int opt_inc_mode = OP2B_INC_GATHER;
  int opt_gather_kernel = 6;  // OP2B_GATHER_CORNER (gather.h)
  int opt_gather_minb = 0;    // __launch_bounds__ minimum blocks of the gather kernels
  int opt_bres_kernel = 1;    // bres_calc gather: 0 = inverse-map walk, 1 = boundary records
  int opt_fuse = 1;           // defer save_soln / res_calc to fuse them with the next loop
  int opt_speculate = 1;      // update also computes the next adt_calc's result (SpecAdt)
  int opt_adt_minb = 0;       // adt_calc: __launch_bounds__ minimum blocks (0 = none)
  int opt_host_mirror = 1;    // op_dat::data holds a host copy of the declared values
  int opt_rename_save = 1;    // save_soln by renaming (LazySave)
  int opt_speculate_res = 1;  // update launches the res_calc + bres_calc after it (ResLearn)
  int opt_lazy_res = 1;       // update leaves res unwritten, recorded as zero (res_zero)
  int opt_host_threads = 8;   // threads of a large host copy (host copies of maps and dats)
  int opt_pipe_block = 256;   // threads per CTA of the pipelined gather (64, 96, 128, 256)
  int opt_pipe_hints = 0;     // register pipeline: evict-first hints on once-read streams
  int opt_plan_mode = 0;      // colouring: 0 = serial greedy for op_plan_get and the plan-
                              // driven loops (bit-exact), Jones-Plassmann for the run-time
                              // compiled loops' colourings; 1 = Jones-Plassmann for every
                              // plan; 2 = serial greedy for every plan
  int opt_atomic_seg = 1;     // inc_mode 0: 1 = segmented (warp-combined) atomics, 0 = per edge
  int opt_jit_warp = 1;       // generated loops: coalesced direct rows, vector gathers, warp-combined increments
  int opt_jit_exact = 0;      // generated loops that only increment one dat: owner computes, bit-exact
  int opt_update_rev = 1;     // the update kernel walks the cells downwards (L2 reuse after the pair)
  int opt_atomic_blocks = 4096; // inc_mode 0: 256-thread CTAs per SM in res_calc's grid (at most)
  int ring_used = 0;          // the last res_calc launch ran over the flux-ring records
  int opt_gemm_tma = 0;       // op2b_gemm_bf16 engine 0: TMA-fed kernel for k-major operands
  int opt_host_staging = 1;   // large device -> pageable host copies: 0 the driver's copies,
                              // 1 through two pinned staging buffers (pinned while op_renumber
                              // waits for the device)
  int opt_pdl = 1;            // the iteration's kernels by programmatic dependent launch
  int opt_gemm_rows = 1;      // persistent GEMM: stores whole rows through shared memory
  int opt_gemm_ws = 2;        // TMA-fed products: 0 = a CTA per tile, 1 / 2 = the persistent
                              // warp-specialised kernel with 8 / 16 epilogue warps
  bool opt_check_plans = false;
  bool quiet_errors = false;  // set_error records without printing or aborting

  std::vector<std::unique_ptr<op_set_core>> sets;
  std::vector<std::unique_ptr<op_map_core>> maps;
  std::vector<std::unique_ptr<op_dat_core>> dats;
  std::map<std::string, std::vector<double>> consts;
  std::map<std::string, std::string> const_types;  // "double", "float" or "int"
  long const_version = 0;                          // bumped by every op_decl_const
  std::map<const int *, op_map> map_ptrs;  // user array -> map (op_renumber_ptr)

  // fused-update reduction
  RedScratch red{};
  void *red_base = nullptr;
  void *pinned = nullptr;      // 4 KiB mapped pinned host page for reduction read-back
  void *pinned_dev = nullptr;  // its device address
  char *stage = nullptr;       // 2 x kStageChunk pinned buffers for large device -> host copies
  std::thread stage_alloc;     // pins them in the background from op_init on
  cudaEvent_t stage_ev[2] = {nullptr, nullptr};
  long long red_seq = 0;       // sequence number of the last update launch
  unsigned long long *check_d = nullptr;  // device word for op_decl_map's range check

  // timing
  std::map<std::string, LoopStat> stats;
  std::vector<cudaEvent_t> ev_free;
  std::vector<PendingTime> pending;
  std::string cur_loop;
  cudaEvent_t cur_ev0 = nullptr, cur_ev1 = nullptr;

  PendingLoop pend;
  LazySave lazy;
  ResLearn rlearn;
  int sres_stage = 0;  // speculative res_calc + bres_calc: 0 none, 1 launched, 2 res_calc seen
  // A dat the program holds all zeros while its array does not: the update
  // zeroes res, and the res_calc + bres_calc after it rewrite every element
  // starting from zero, so the update leaves the array as it is.  The fused
  // pair then starts from 0 instead of reading res; anything else that
  // touches the dat first zeroes the array (materialize_res).
  op_dat res_zero = nullptr;
  SpecAdt spec;
  std::set<op_dat> exposed;  // dats whose device pointer was handed out (no speculation)
  std::set<op_dat> zero_mirror;  // dats declared without data: their host copy is zeros
  std::set<op_dat> overlays;     // op_decl_dat_overlay: storage owned by another dat
  std::map<const char *, op_dat> orig_ptrs;  // caller's array -> the dat declared from it

  LaunchCtx ctx();
  // initialised, with any deferred loop launched (false on error)
  bool ready();
  // a deferred loop or a renamed save_soln is outstanding
  bool outstanding() const {
    return pend.kind != 0 || lazy.src != nullptr || sres_stage != 0 || res_zero != nullptr;
  }
  bool materialize_res();   // op2b_dispatch.cpp: zero the array of res_zero
  bool flush_pending();     // op2b_dispatch.cpp: everything settled and launched
  bool settle_res();        // op2b_dispatch.cpp: undo a speculative res_calc + bres_calc
  bool flush_loop();        // op2b_dispatch.cpp: the deferred loop only
  bool materialize_save();  // op2b_dispatch.cpp: the renamed save_soln's copy
  bool restore_spec();   // op2b_dispatch.cpp: put the old adt back if adt is ahead
  void begin_loop(const char *name);
  void count_call(const char *name) { stats[name].calls++; }  // a call with no launch
  void end_loop(double bytes);
  void resolve_timing();
  const double *const_ptr(const char *name, int dim);
};

Runtime &rt();
// region profiler (profile.cpp): a resolved time for node `id`; the kernel
// node a loop starting now is timed into (-1 = none); op_exit's clean-up
void profile_submit(int id, float ms);
int profile_loop_node(const std::string &loop);
bool profile_times_loops();
void profile_on_exit();

void set_error(const char *fmt, ...);
bool cuda_ok(cudaError_t e, const char *what);
// Device -> pageable host copy on the library stream, through pinned buffers
// with the host-side copies spread over threads (synchronous).
bool download_host(void *dst, const void *src_d, size_t bytes, const char *what);
constexpr size_t kStageChunk = (size_t)4 << 20;
// pin the staging buffers on a thread of their own (op_renumber, while the
// device works)
void stage_in_background();
// several device -> host copies in one staged pipeline (synchronous)
struct HostDownload {
  void *dst;
  const void *src_d;
  size_t bytes;
};
bool download_host_many(const std::vector<HostDownload> &jobs, const char *what);
int type_bytes(const char *type);
bool is_real(const char *type, int bytes);

// renumber.cu
void resolve_renumbering_for_fetch(op_dat dat);
void fetch_original_order(op_dat dat, char *dst, int low, int high);
void release_renumbering();
// plan.cu
void release_plans();
// jit.cpp: loops without a hand-written kernel, compiled from the user's
// kernel source at run time
bool jit_has_kernel(const char *name);
int jit_par_loop(const char *name, op_set set, int nargs, op_arg *args);
void release_jit();
// airfoil_gather.cu
void release_inverse_maps();

}  // namespace op2b
