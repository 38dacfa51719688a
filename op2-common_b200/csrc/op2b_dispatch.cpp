// op_par_loop dispatch: a loop is identified by its name and must match the
// argument signature of the device loop registered under that name.  The
// signatures are those of the Airfoil calls in
// apps/c/airfoil/airfoil_plain/dp/airfoil.cpp:225-277 (and the rms-only
// update of apps/c/airfoil/airfoil_tempdats/dp/airfoil.cpp); a dat of type
// "double" selects the FP64 kernels, "float" the FP32-storage kernels of the
// mixed-precision form.  Anything else is an error -- there is no host
// execution path.
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "op2b_runtime.h"
#include "gather.h"
#include "staged.h"

using namespace op2b;

namespace {

const char *acc_name(int a) {
  static const char *n[] = {"OP_READ", "OP_WRITE", "OP_RW", "OP_INC", "OP_MIN", "OP_MAX",
                            "OP_WORK"};
  return (a >= 0 && a <= 6) ? n[a] : "?";
}

// a loop function's return value when the arguments do not match its
// signature (nothing launched, nothing changed)
constexpr int kSigMismatch = -2;

struct Sig {
  const char *loop;
  op_set set;
  op_arg *a;
  int nargs;
  bool ok = true;

  bool fail(int i, const char *what) {
    if (ok) set_error("op_par_loop(%s): argument %d: %s", loop, i, what);
    ok = false;
    return false;
  }
  // a dat argument with the given dimension, access, map (NULL = direct) and index
  bool dat(int i, int dim, int acc, op_map map, int idx) {
    if (!ok) return false;
    if (i >= nargs) return fail(i, "missing");
    const op_arg &x = a[i];
    char buf[256];
    if (x.argtype != OP_ARG_DAT || !x.dat) return fail(i, "expected an op_arg_dat");
    if (!x.opt) return fail(i, "optional argument switched off; this loop needs it");
    if (x.dat->dim != dim || x.dim != dim) {
      snprintf(buf, sizeof(buf), "expected dim %d, got dat dim %d / arg dim %d", dim,
               x.dat->dim, x.dim);
      return fail(i, buf);
    }
    if (x.acc != acc) {
      snprintf(buf, sizeof(buf), "expected %s, got %s", acc_name(acc), acc_name(x.acc));
      return fail(i, buf);
    }
    if (x.type && x.dat->type && type_bytes(x.type) != type_bytes(x.dat->type)) {
      snprintf(buf, sizeof(buf), "type '%s' does not match dat type '%s'", x.type, x.dat->type);
      return fail(i, buf);
    }
    if (map == nullptr) {
      if (x.map != nullptr || x.idx != -1) return fail(i, "expected a direct (OP_ID) argument");
      if (x.dat->set != set) return fail(i, "dat is not defined on the loop's set");
    } else {
      if (x.map != map) return fail(i, "expected the same map as the loop's other arguments");
      if (x.idx != idx) {
        snprintf(buf, sizeof(buf), "expected map index %d, got %d", idx, x.idx);
        return fail(i, buf);
      }
      if (map->from != set) return fail(i, "map does not start from the loop's set");
      if (map->to != x.dat->set) return fail(i, "map does not point to the dat's set");
    }
    return true;
  }
  bool gbl(int i, int dim, int acc, int bytes) {
    if (!ok) return false;
    if (i >= nargs) return fail(i, "missing");
    const op_arg &x = a[i];
    if (x.argtype != OP_ARG_GBL) return fail(i, "expected an op_arg_gbl");
    if (x.dim != dim || x.size != dim * bytes || x.acc != acc || !x.data)
      return fail(i, "global argument of the wrong dimension, type or access");
    return true;
  }
  int real_bytes(std::initializer_list<int> idx) {
    int b = 0;
    for (int i : idx) {
      if (!ok) return 0;
      const op_arg &x = a[i];
      int tb = type_bytes(x.dat->type);
      if (!is_real(x.dat->type, tb)) {
        fail(i, "dat must be of type double or float");
        return 0;
      }
      if (b && tb != b) {
        fail(i, "all real dats of this loop must have the same precision");
        return 0;
      }
      b = tb;
    }
    return b;
  }
};

template <typename T> AirConst<T> air_consts(bool &ok) {
  AirConst<T> k{};
  Runtime &r = rt();
  const double *gam = r.const_ptr("gam", 1), *gm1 = r.const_ptr("gm1", 1),
               *cfl = r.const_ptr("cfl", 1), *eps = r.const_ptr("eps", 1),
               *qinf = r.const_ptr("qinf", 4);
  ok = gam && gm1 && cfl && eps && qinf;
  if (!ok) return k;
  k.gam = (T)*gam;
  k.gm1 = (T)*gm1;
  k.cfl = (T)*cfl;
  k.eps = (T)*eps;
  for (int i = 0; i < 4; i++) k.qinf[i] = (T)qinf[i];
  return k;
}

// the constants of a speculative adt equal the current ones
bool consts_match(const SpecAdt &sp, int rb) {
  bool ok;
  if (rb == 8) {
    AirConst<double> k = air_consts<double>(ok);
    return ok && memcmp(&k, &sp.kd, sizeof(k)) == 0;
  }
  AirConst<float> k = air_consts<float>(ok);
  return ok && memcmp(&k, &sp.kf, sizeof(k)) == 0;
}

// Spin until the device publishes `seq` at *flag.  Every few thousand spins
// the stream is queried so a failed kernel is reported instead of waited
// for; the wait gives up after 120 s.
bool wait_for_sequence(volatile long long *flag, long long seq, const char *what) {
  Runtime &r = rt();
  auto t0 = std::chrono::steady_clock::now();
  for (long spins = 0; *flag != seq; spins++) {
    if ((spins & 4095) == 4095) {
      cudaError_t q = cudaStreamQuery(r.stream);
      if (q != cudaSuccess && q != cudaErrorNotReady) return cuda_ok(q, what);
      if (q == cudaSuccess && *flag != seq) {
        set_error("%s: the stream finished without publishing the result", what);
        return false;
      }
      if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(120)) {
        set_error("%s: no result after 120 s", what);
        return false;
      }
    }
  }
  std::atomic_thread_fence(std::memory_order_acquire);
  return true;
}

int finish(cudaError_t e, const char *loop) {
  if (e != cudaSuccess) {
    set_error("op_par_loop(%s): kernel launch failed: %s", loop, cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

// A loop may run while a renamed save_soln is outstanding when it neither
// touches qold nor writes q: qold's array is stale, q's is current.
bool save_compatible(const Runtime &r, const op_arg *a, int nargs) {
  for (int i = 0; i < nargs; i++) {
    if (a[i].argtype != OP_ARG_DAT || !a[i].dat) continue;
    if (a[i].dat == r.lazy.dst || (a[i].dat == r.lazy.src && a[i].acc != OP_READ)) return false;
  }
  return true;
}

// A loop may run while a speculative res_calc + bres_calc is outstanding
// when it neither touches res nor writes what the pair reads.
bool res_compatible(const Runtime &r, const op_arg *a, int nargs) {
  const ResLearn &L = r.rlearn;
  for (int i = 0; i < nargs; i++) {
    if (a[i].argtype != OP_ARG_DAT || !a[i].dat) continue;
    const op_dat d = a[i].dat;
    if (d == L.res) return false;
    if (a[i].acc != OP_READ && (d == L.x || d == L.q || d == L.adt || d == L.bound)) return false;
  }
  return true;
}

bool touches(const op_arg *a, int nargs, op_dat d) {
  for (int i = 0; i < nargs; i++)
    if (a[i].argtype == OP_ARG_DAT && a[i].dat == d) return true;
  return false;
}

// Settle what is outstanding before a loop with these arguments: a
// speculative res_calc + bres_calc, a renamed save_soln and a res known to be
// zero stay when the loop can run beside them; the deferred loop is launched.
// keep_zero: the caller handles res_zero itself (a res_calc it defers).
bool flush_for(Runtime &r, const op_arg *a, int nargs, bool keep_zero = false) {
  bool ok = true;
  if (r.sres_stage && !res_compatible(r, a, nargs)) ok = r.settle_res();
  if (r.pend.kind) ok = r.flush_loop() && ok;
  if (r.lazy.src && !save_compatible(r, a, nargs)) ok = r.materialize_save() && ok;
  if (r.res_zero && !keep_zero && touches(a, nargs, r.res_zero)) ok = r.materialize_res() && ok;
  return ok;
}

bool consts_are(const AirConst<double> &kd, const AirConst<float> &kf, int rb) {
  bool ok;
  if (rb == 8) {
    AirConst<double> k = air_consts<double>(ok);
    return ok && memcmp(&k, &kd, sizeof(k)) == 0;
  }
  AirConst<float> k = air_consts<float>(ok);
  return ok && memcmp(&k, &kf, sizeof(k)) == 0;
}

// res_calc and the bres_calc after it in one launch: over the flux-ring
// records (each in-range flux computed once) when gather_kernel 7 asks for it
// and the numbering allows it, else the corner kernel
template <typename T>
static cudaError_t launch_fused_pair(Runtime &r, const SlotRecords &cr, const BresRecords &br,
                                     const int *bound, const T *x, const T *q, const T *adt,
                                     T *res, const AirConst<T> &k, bool zero) {
  r.ring_used = r.opt_gather_kernel == OP2B_GATHER_RING && build_ring_records(&cr, r.nsm, 256);
  if (r.ring_used) return launch_res_ring<T>(r.ctx(), cr, bound, x, q, adt, res, k, zero);
  return launch_res_bres_corner<T>(r.ctx(), cr, br, bound, x, q, adt, res, k, r.opt_pipe_block,
                                   zero);
}

// the update's call launches the res_calc + bres_calc pair learned last
// (ResLearn) right behind it, on the arrays it leaves: q, adt (the next
// adt_calc's, computed ahead) and res (zero)
void launch_speculative_res(Runtime &r, const op_arg *a, int rb) {
  const ResLearn &L = r.rlearn;
  const SpecAdt &sp = r.spec;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(r.stream, &cap);
  if (!r.opt_speculate_res || !L.valid || !sp.inplace || cap != cudaStreamCaptureStatusNone ||
      L.rb != rb || L.q != a[1].dat || L.res != a[2].dat || L.adt != a[3].dat ||
      sp.q != L.q || sp.adt != L.adt || sp.x != L.x || !r.overlays.empty() ||
      r.exposed.count(L.x) || r.exposed.count(L.q) || r.exposed.count(L.adt) ||
      r.exposed.count(L.res) || r.exposed.count(L.bound) || !consts_are(L.kd, L.kf, rb) ||
      memcmp(rb == 8 ? (const void *)&sp.kd : (const void *)&sp.kf,
             rb == 8 ? (const void *)&L.kd : (const void *)&L.kf,
             rb == 8 ? sizeof(L.kd) : sizeof(L.kf)) != 0)
    return;
  const SlotRecords *cr = get_corner_records(L.pecell, L.pedge);
  const BresRecords *br = cr && cr->corners ? get_bres_records(L.pbecell, L.pbedge) : nullptr;
  if (!br || !link_boundary_records(cr, br, L.pbecell)) {
    cudaGetLastError();
    return;
  }
  const int *bound = (const int *)L.bound->data_d;
  const bool zero = r.res_zero == L.res;  // the update left res zero without writing it
  cudaError_t e;
  r.begin_loop("res_calc+bres_calc");
  // adt: the next adt_calc's result, still in the second array
  if (rb == 8)
    e = launch_fused_pair<double>(r, *cr, *br, bound, (const double *)L.x->data_d,
                                  (const double *)L.q->data_d, (const double *)sp.shadow,
                                  (double *)L.res->data_d, L.kd, zero);
  else
    e = launch_fused_pair<float>(r, *cr, *br, bound, (const float *)L.x->data_d,
                                 (const float *)L.q->data_d, (const float *)sp.shadow,
                                 (float *)L.res->data_d, L.kf, zero);
  r.end_loop(L.fused_bytes - (zero ? L.res_read_bytes : 0.0));
  if (e == cudaSuccess) r.sres_stage = 1;
  else cudaGetLastError();  // not launched: the program's calls run as usual
}

// ---------------------------------------------------------------- save_soln
int loop_save_soln(const char *name, op_set set, int nargs, op_arg *a) {
  Sig s{name, set, a, nargs};
  if (nargs != 2) return s.fail(nargs, "save_soln takes 2 arguments"), kSigMismatch;
  int dim = a[0].dat ? a[0].dat->dim : 0;
  s.dat(0, dim, OP_READ, nullptr, -1);
  s.dat(1, dim, OP_WRITE, nullptr, -1);
  if (!s.ok) return kSigMismatch;
  if (a[0].dat->size != a[1].dat->size) return s.fail(1, "element size differs from argument 0"), kSigMismatch;
  Runtime &r = rt();
  if (r.lazy.src == a[0].dat && r.lazy.dst == a[1].dat) {  // qold is already q
    if (r.pend.kind && !r.flush_loop()) return -1;
    r.count_call("save_soln(renamed)");
    return 0;
  }
  if (!flush_for(r, a, nargs)) return -1;
  if (r.lazy.src && !r.materialize_save()) return -1;  // one renamed save_soln at a time
  if (r.spec.inplace && (a[1].dat == r.spec.x || a[1].dat == r.spec.q ||
                         a[1].dat == r.spec.adt || a[0].dat == r.spec.adt) &&
      !r.restore_spec())
    return -1;
  size_t bytes = (size_t)set->size * (size_t)a[0].dat->size;
  int tb = a[0].dat->type ? type_bytes(a[0].dat->type) : 0;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(r.stream, &cap);
  if (r.opt_rename_save && a[0].dat != a[1].dat && a[0].dat->set == a[1].dat->set &&
      !r.exposed.count(a[0].dat) && !r.exposed.count(a[1].dat) && r.overlays.empty() &&
      cap == cudaStreamCaptureStatusNone) {
    // renamed: no launch now; the update that next writes q swaps the arrays
    r.lazy.src = a[0].dat;
    r.lazy.dst = a[1].dat;
    r.count_call("save_soln(renamed)");
    return 0;
  }
  if (r.opt_fuse && dim == 4 && is_real(a[0].dat->type, tb) && a[0].dat != a[1].dat) {
    // deferred: launched with the next loop call (fused into an adt_calc on
    // the same q) or alone before any other call
    r.pend = PendingLoop{};
    r.pend.kind = 1;
    r.pend.set = set;
    r.pend.src = a[0].dat;
    r.pend.dst = a[1].dat;
    r.pend.rb = tb;
    r.pend.bytes = 2.0 * (double)bytes;
    return 0;
  }
  r.begin_loop(name);
  cudaError_t e = launch_copy(r.ctx(), a[0].dat->data_d, a[1].dat->data_d, bytes);
  r.end_loop(2.0 * (double)bytes);
  return finish(e, name);
}

// ---------------------------------------------------------------- adt_calc
int loop_adt_calc(const char *name, op_set set, int nargs, op_arg *a) {
  Sig s{name, set, a, nargs};
  if (nargs != 6) return s.fail(nargs, "adt_calc takes 6 arguments"), kSigMismatch;
  op_map pcell = a[0].map;
  if (!pcell || pcell->dim != 4) return s.fail(0, "expected a dim-4 map (cells -> nodes)"), kSigMismatch;
  for (int i = 0; i < 4; i++) s.dat(i, 2, OP_READ, pcell, i);
  if (s.ok && (a[1].dat != a[0].dat || a[2].dat != a[0].dat || a[3].dat != a[0].dat))
    return s.fail(1, "arguments 0-3 must be the same dat"), kSigMismatch;
  s.dat(4, 4, OP_READ, nullptr, -1);
  s.dat(5, 1, OP_WRITE, nullptr, -1);
  int rb = s.real_bytes({0, 4, 5});
  if (!s.ok) return kSigMismatch;
  Runtime &r = rt();
  int C = set->size, N = a[0].dat->set->size;
  double bytes = 16.0 * C + (double)rb * (2.0 * N + 5.0 * C);
  PendingLoop &pd = r.pend;
  SpecAdt &sp = r.spec;
  const bool hit = sp.inplace && sp.pcell == pcell && sp.x == a[0].dat && sp.q == a[4].dat &&
                   sp.adt == a[5].dat && sp.rb == rb && consts_match(sp, rb);
  if (hit) {
    // the update before this call already wrote this adt_calc's result into
    // the second array: it becomes adt's
    sp.inplace = false;
    std::swap(sp.adt->data_d, *reinterpret_cast<char **>(&sp.shadow));
    sp.shadow_bytes = ((size_t)C * rb + 255) & ~(size_t)255;
    r.count_call("adt_calc(in update)");
    return 0;
  }
  if (r.sres_stage && !r.settle_res()) return -1;  // it read the adt computed ahead
  if (sp.inplace && !r.restore_spec()) return -1;
  sp.pcell = pcell;  // what the next update may compute ahead
  sp.x = a[0].dat;
  sp.q = a[4].dat;
  sp.adt = a[5].dat;
  sp.rb = rb;
  if (pd.kind == 1 && pd.src == a[4].dat && pd.set == set && pd.rb == rb &&
      pd.dst != a[0].dat && pd.dst != a[5].dat) {
    // save_soln (q -> qold) and this adt_calc in one pass over q: the fused
    // call moves adt_calc's bytes plus qold's write
    op_dat qold = pd.dst;
    const double fused = bytes + 4.0 * rb * (double)C;
    pd = PendingLoop{};
    bool ok;
    cudaError_t e;
    r.begin_loop("save_soln+adt_calc");
    if (rb == 8) {
      AirConst<double> k = air_consts<double>(ok);
      if (!ok) return -1;
      e = launch_adt_save<double>(r.ctx(), C, pcell->map_d, (const double *)a[0].dat->data_d,
                                  (const double *)a[4].dat->data_d, (double *)a[5].dat->data_d,
                                  (double *)qold->data_d, k);
    } else {
      AirConst<float> k = air_consts<float>(ok);
      if (!ok) return -1;
      e = launch_adt_save<float>(r.ctx(), C, pcell->map_d, (const float *)a[0].dat->data_d,
                                 (const float *)a[4].dat->data_d, (float *)a[5].dat->data_d,
                                 (float *)qold->data_d, k);
    }
    r.end_loop(fused);
    return finish(e, name);
  }
  if (!flush_for(r, a, nargs)) return -1;
  r.begin_loop(name);
  cudaError_t e;
  bool ok;
  if (rb == 8) {
    AirConst<double> k = air_consts<double>(ok);
    if (!ok) return -1;
    e = launch_adt_calc<double>(r.ctx(), C, pcell->map_d, (const double *)a[0].dat->data_d,
                                (const double *)a[4].dat->data_d, (double *)a[5].dat->data_d, k,
                                r.opt_adt_minb);
  } else {
    AirConst<float> k = air_consts<float>(ok);
    if (!ok) return -1;
    e = launch_adt_calc<float>(r.ctx(), C, pcell->map_d, (const float *)a[0].dat->data_d,
                               (const float *)a[4].dat->data_d, (float *)a[5].dat->data_d, k,
                               r.opt_adt_minb);
  }
  r.end_loop(bytes);
  return finish(e, name);
}

// ---------------------------------------------------------------- res_calc
// the slot-record gather kernels (option gather_kernel), all bit-identical
template <typename T>
static cudaError_t res_gather_slots(Runtime &r, const SlotRecords &s, const ResCalcArgs<T> &p,
                                    const AirConst<T> &k) {
  switch (r.opt_gather_kernel) {
    case OP2B_GATHER_RING:
      r.ring_used = s.corners && build_ring_records(&s, r.nsm, 256);
      if (r.ring_used)
        return launch_res_ring<T>(r.ctx(), s, nullptr, p.x, p.q, p.adt, p.res, k, false);
      if (s.corners)  // neighbours too far apart in the numbering for the ring
        return launch_res_calc_gather_corner<T>(r.ctx(), s, p.x, p.q, p.adt, p.res, k,
                                                r.opt_pipe_block, r.opt_gather_minb);
      return launch_res_calc_gather_regpipe<T>(r.ctx(), s, p.x, p.q, p.adt, p.res, k,
                                               r.opt_pipe_block);
    case OP2B_GATHER_LANES:
      return launch_res_calc_gather4<T>(r.ctx(), s, p.x, p.q, p.adt, p.res, k);
    case OP2B_GATHER_PIPE:
      return launch_res_calc_gather_pipe<T>(r.ctx(), s, p.x, p.q, p.adt, p.res, k,
                                            r.opt_pipe_block);
    case OP2B_GATHER_REGPIPE:
      return launch_res_calc_gather_regpipe<T>(r.ctx(), s, p.x, p.q, p.adt, p.res, k,
                                               r.opt_pipe_block);
    case OP2B_GATHER_CORNER:
      if (s.corners)
        return launch_res_calc_gather_corner<T>(r.ctx(), s, p.x, p.q, p.adt, p.res, k,
                                                r.opt_pipe_block, r.opt_gather_minb);
      // edges touching more than four nodes per cell: the slot-record pipeline
      return launch_res_calc_gather_regpipe<T>(r.ctx(), s, p.x, p.q, p.adt, p.res, k,
                                               r.opt_pipe_block);
    default:
      return launch_res_calc_gather_cell4<T>(r.ctx(), s, p.x, p.q, p.adt, p.res, k);
  }
}

int loop_res_calc(const char *name, op_set set, int nargs, op_arg *a) {
  Sig s{name, set, a, nargs};
  if (nargs != 8) return s.fail(nargs, "res_calc takes 8 arguments"), kSigMismatch;
  op_map pedge = a[0].map, pecell = a[2].map;
  if (!pedge || pedge->dim != 2) return s.fail(0, "expected a dim-2 map (edges -> nodes)"), kSigMismatch;
  if (!pecell || pecell->dim != 2) return s.fail(2, "expected a dim-2 map (edges -> cells)"), kSigMismatch;
  s.dat(0, 2, OP_READ, pedge, 0);
  s.dat(1, 2, OP_READ, pedge, 1);
  s.dat(2, 4, OP_READ, pecell, 0);
  s.dat(3, 4, OP_READ, pecell, 1);
  s.dat(4, 1, OP_READ, pecell, 0);
  s.dat(5, 1, OP_READ, pecell, 1);
  s.dat(6, 4, OP_INC, pecell, 0);
  s.dat(7, 4, OP_INC, pecell, 1);
  if (s.ok && (a[1].dat != a[0].dat || a[3].dat != a[2].dat || a[5].dat != a[4].dat ||
               a[7].dat != a[6].dat))
    return s.fail(1, "paired arguments must name the same dat"), kSigMismatch;
  int rb = s.real_bytes({0, 2, 4, 6});
  if (!s.ok) return kSigMismatch;
  Runtime &r = rt();
  const ResLearn &L = r.rlearn;
  if (r.sres_stage == 1 && !r.spec.inplace && set == L.eset && pedge == L.pedge &&
      pecell == L.pecell && a[0].dat == L.x && a[2].dat == L.q && a[4].dat == L.adt &&
      a[6].dat == L.res && rb == L.rb && consts_are(L.kd, L.kf, rb)) {
    r.sres_stage = 2;  // launched by the update before, with bres_calc's increments
    r.count_call("res_calc(speculated)");
    return 0;
  }
  if (r.sres_stage && !r.settle_res()) return -1;
  if (!flush_for(r, a, nargs, true)) return -1;
  if (r.spec.inplace && !r.restore_spec()) return -1;
  int E = set->size, N = a[0].dat->set->size, C = a[2].dat->set->size;
  double bytes = 16.0 * E + (double)rb * (2.0 * N + 13.0 * C);
  if (r.opt_fuse && r.opt_inc_mode == OP2B_INC_GATHER &&
      (r.opt_gather_kernel == OP2B_GATHER_CORNER || r.opt_gather_kernel == OP2B_GATHER_RING) &&
      r.opt_bres_kernel == 1) {
    const SlotRecords *cr = get_corner_records(pecell, pedge);
    if (!cr) return -1;
    bool ok = true;
    if (cr->corners) {
      // deferred: fused with a following bres_calc on the same res, or
      // launched alone before any other call
      PendingLoop &pd = r.pend;
      pd = PendingLoop{};
      pd.kind = 2;
      pd.set = set;
      pd.pedge = pedge;
      pd.pecell = pecell;
      pd.x = a[0].dat;
      pd.q = a[2].dat;
      pd.adt = a[4].dat;
      pd.res = a[6].dat;
      pd.rb = rb;
      pd.bytes = bytes;
      if (rb == 8) pd.kd = air_consts<double>(ok);
      else pd.kf = air_consts<float>(ok);
      if (!ok) {
        pd = PendingLoop{};
        return -1;
      }
      return 0;
    }
  }
  // launched now: a res known to be zero gets its zeros first
  if (r.res_zero && touches(a, nargs, r.res_zero) && !r.materialize_res()) return -1;
  Plan *plan = nullptr;
  const InvMap *inv = nullptr;
  const SlotRecords *slots = nullptr;
  if (r.opt_inc_mode == OP2B_INC_GATHER) {
    if (r.opt_gather_kernel == OP2B_GATHER_CORNER || r.opt_gather_kernel == OP2B_GATHER_RING) {
      slots = get_corner_records(pecell, pedge);
      if (!slots) return -1;
    } else if (r.opt_gather_kernel != OP2B_GATHER_CSR) {
      slots = get_slot_records(pecell, pedge);
      if (!slots) return -1;
    }
    if (!slots || !slots->usable) {  // CSR walk (also when a cell has more than 4 edges)
      slots = nullptr;
      inv = get_inverse_map(pecell);
      if (!inv) return -1;
    }
  } else if (r.opt_inc_mode != OP2B_INC_ATOMIC) {
    plan = get_res_plan(name, set, nargs, a);
    if (!plan) return -1;
  }
  bool ok;
  cudaError_t e;
  if (rb == 8) {
    AirConst<double> k = air_consts<double>(ok);
    if (!ok) return -1;
    ResCalcArgs<double> p{E, pedge->map_d, pecell->map_d, (const double *)a[0].dat->data_d,
                          (const double *)a[2].dat->data_d, (const double *)a[4].dat->data_d,
                          (double *)a[6].dat->data_d, k};
    r.begin_loop(name);
    e = slots ? res_gather_slots<double>(r, *slots, p, k)
        : inv ? launch_res_calc_gather<double>(r.ctx(), *inv, p.pedge, p.pecell, p.x, p.q,
                                               p.adt, p.res, k)
              : run_res_calc<double>(r.ctx(), p, plan, r.opt_inc_mode);
  } else {
    AirConst<float> k = air_consts<float>(ok);
    if (!ok) return -1;
    ResCalcArgs<float> p{E, pedge->map_d, pecell->map_d, (const float *)a[0].dat->data_d,
                         (const float *)a[2].dat->data_d, (const float *)a[4].dat->data_d,
                         (float *)a[6].dat->data_d, k};
    r.begin_loop(name);
    e = slots ? res_gather_slots<float>(r, *slots, p, k)
        : inv ? launch_res_calc_gather<float>(r.ctx(), *inv, p.pedge, p.pecell, p.x, p.q,
                                              p.adt, p.res, k)
              : run_res_calc<float>(r.ctx(), p, plan, r.opt_inc_mode);
  }
  r.end_loop(bytes);
  return finish(e, name);
}

// ---------------------------------------------------------------- bres_calc
int loop_bres_calc(const char *name, op_set set, int nargs, op_arg *a) {
  Sig s{name, set, a, nargs};
  if (nargs != 6) return s.fail(nargs, "bres_calc takes 6 arguments"), kSigMismatch;
  op_map pbedge = a[0].map, pbecell = a[2].map;
  if (!pbedge || pbedge->dim != 2) return s.fail(0, "expected a dim-2 map (bedges -> nodes)"), kSigMismatch;
  if (!pbecell || pbecell->dim != 1) return s.fail(2, "expected a dim-1 map (bedges -> cells)"), kSigMismatch;
  s.dat(0, 2, OP_READ, pbedge, 0);
  s.dat(1, 2, OP_READ, pbedge, 1);
  s.dat(2, 4, OP_READ, pbecell, 0);
  s.dat(3, 1, OP_READ, pbecell, 0);
  s.dat(4, 4, OP_INC, pbecell, 0);
  s.dat(5, 1, OP_READ, nullptr, -1);
  if (s.ok && a[1].dat != a[0].dat) return s.fail(1, "arguments 0 and 1 must be the same dat"), kSigMismatch;
  if (s.ok && (type_bytes(a[5].dat->type) != 4 || std::string(a[5].dat->type).rfind("int", 0) != 0))
    return s.fail(5, "the boundary flag must be an int dat"), kSigMismatch;
  int rb = s.real_bytes({0, 2, 3, 4});
  if (!s.ok) return kSigMismatch;
  Runtime &r = rt();
  {
    const ResLearn &L = r.rlearn;
    if (r.sres_stage == 2 && set == L.bset && pbedge == L.pbedge && pbecell == L.pbecell &&
        a[0].dat == L.x && a[2].dat == L.q && a[3].dat == L.adt && a[4].dat == L.res &&
        a[5].dat == L.bound && rb == L.rb && consts_are(L.kd, L.kf, rb)) {
      r.sres_stage = 0;  // the pair the update launched is the program's
      if (r.res_zero == L.res) r.res_zero = nullptr;  // it wrote every element of res
      r.count_call("bres_calc(speculated)");
      return 0;
    }
    // not the learned pair: res back to zero (and res_calc deferred again)
    if (r.sres_stage && !r.settle_res()) return -1;
  }
  if (r.spec.inplace && !r.restore_spec()) return -1;
  int B = set->size;
  double bytes = 16.0 * B + (double)rb * (2.0 + 4.0 + 1.0 + 8.0) * B;
  PendingLoop &pd = r.pend;
  bool same_consts = false;  // bres_calc would use the constants res_calc was called with
  if (pd.kind == 2) {
    bool ok;
    if (rb == 8) {
      AirConst<double> k = air_consts<double>(ok);
      same_consts = ok && memcmp(&k, &pd.kd, sizeof(k)) == 0;
    } else {
      AirConst<float> k = air_consts<float>(ok);
      same_consts = ok && memcmp(&k, &pd.kf, sizeof(k)) == 0;
    }
  }
  if (pd.kind == 2 && same_consts && pd.res == a[4].dat && pd.q == a[2].dat &&
      pd.adt == a[3].dat && pd.x == a[0].dat && pd.rb == rb &&
      r.opt_inc_mode == OP2B_INC_GATHER && r.opt_bres_kernel == 1) {
    if (r.lazy.src && !save_compatible(r, a, nargs) && !r.materialize_save()) return -1;
    const SlotRecords *cr = get_corner_records(pd.pecell, pd.pedge);
    const BresRecords *br = cr ? get_bres_records(pbecell, pbedge) : nullptr;
    if (cr && br && link_boundary_records(cr, br, pbecell)) {
      // res_calc's and this bres_calc's increments in one launch, in the order
      // of the two loops run one after the other; beyond res_calc's bytes the
      // fused call reads the boundary maps, flags and nodes (q, adt and res of
      // the boundary cells move with res_calc's)
      const double fused = pd.bytes + 16.0 * B + 4.0 * rb * B;
      const double res_read = 4.0 * rb * (double)pd.res->set->size;
      const int *bound = (const int *)a[5].dat->data_d;
      const bool zero = r.res_zero == pd.res;  // start from 0: the update left res zero
      cudaError_t e;
      r.begin_loop("res_calc+bres_calc");
      if (rb == 8)
        e = launch_fused_pair<double>(r, *cr, *br, bound, (const double *)pd.x->data_d,
                                      (const double *)pd.q->data_d,
                                      (const double *)pd.adt->data_d, (double *)pd.res->data_d,
                                      pd.kd, zero);
      else
        e = launch_fused_pair<float>(r, *cr, *br, bound, (const float *)pd.x->data_d,
                                     (const float *)pd.q->data_d, (const float *)pd.adt->data_d,
                                     (float *)pd.res->data_d, pd.kf, zero);
      r.end_loop(fused - (zero ? res_read : 0.0));
      if (zero && e == cudaSuccess) r.res_zero = nullptr;  // every element rewritten
      if (e == cudaSuccess) {  // the pair the next update may launch ahead
        ResLearn &L = r.rlearn;
        L.valid = true;
        L.eset = pd.set;
        L.bset = set;
        L.pedge = pd.pedge;
        L.pecell = pd.pecell;
        L.pbedge = pbedge;
        L.pbecell = pbecell;
        L.x = pd.x;
        L.q = pd.q;
        L.adt = pd.adt;
        L.res = pd.res;
        L.bound = a[5].dat;
        L.rb = rb;
        L.res_bytes = pd.bytes;
        L.fused_bytes = fused;
        L.res_read_bytes = res_read;
        L.kd = pd.kd;
        L.kf = pd.kf;
      }
      pd = PendingLoop{};
      return finish(e, name);
    }
    if (!cr || (r.opt_bres_kernel == 1 && !br)) return -1;
  }
  if (!flush_for(r, a, nargs)) return -1;
  Plan *plan = nullptr;
  const InvMap *inv = nullptr;
  const BresRecords *brec = nullptr;
  if (r.opt_inc_mode == OP2B_INC_GATHER && r.opt_bres_kernel == 1) {
    brec = get_bres_records(pbecell, pbedge);
    if (!brec) return -1;
  } else if (r.opt_inc_mode == OP2B_INC_GATHER) {
    inv = get_inverse_map(pbecell);
    if (!inv) return -1;
  } else if (r.opt_inc_mode == OP2B_INC_COLOR) {
    plan = get_bres_plan(name, set, nargs, a);
    if (!plan) return -1;
  }
  bool ok;
  cudaError_t e;
  if (rb == 8) {
    AirConst<double> k = air_consts<double>(ok);
    if (!ok) return -1;
    BresCalcArgs<double> p{B, pbedge->map_d, pbecell->map_d, (const int *)a[5].dat->data_d,
                           (const double *)a[0].dat->data_d, (const double *)a[2].dat->data_d,
                           (const double *)a[3].dat->data_d, (double *)a[4].dat->data_d, k};
    r.begin_loop(name);
    e = brec ? launch_bres_calc_records<double>(r.ctx(), *brec, p.bound, p.x, p.q, p.adt, p.res, k)
        : inv ? launch_bres_calc_gather<double>(r.ctx(), *inv, p.pbedge, p.bound, p.x, p.q,
                                                p.adt, p.res, k)
              : run_bres_calc<double>(r.ctx(), p, plan, r.opt_inc_mode);
  } else {
    AirConst<float> k = air_consts<float>(ok);
    if (!ok) return -1;
    BresCalcArgs<float> p{B, pbedge->map_d, pbecell->map_d, (const int *)a[5].dat->data_d,
                          (const float *)a[0].dat->data_d, (const float *)a[2].dat->data_d,
                          (const float *)a[3].dat->data_d, (float *)a[4].dat->data_d, k};
    r.begin_loop(name);
    e = brec ? launch_bres_calc_records<float>(r.ctx(), *brec, p.bound, p.x, p.q, p.adt, p.res, k)
        : inv ? launch_bres_calc_gather<float>(r.ctx(), *inv, p.pbedge, p.bound, p.x, p.q,
                                               p.adt, p.res, k)
              : run_bres_calc<float>(r.ctx(), p, plan, r.opt_inc_mode);
  }
  r.end_loop(bytes);
  return finish(e, name);
}

// ---------------------------------------------------------------- update
// 8-argument form of airfoil_plain/dp/update.h (rms INC, maxerr MAX,
// op_arg_idx, op_arg_info of arg 5) or the 5-argument rms-only form of
// airfoil_tempdats/dp/update.h.
int loop_update(const char *name, op_set set, int nargs, op_arg *a) {
  Sig s{name, set, a, nargs};
  if (nargs != 5 && nargs != 8) return s.fail(nargs, "update takes 5 or 8 arguments"), kSigMismatch;
  s.dat(0, 4, OP_READ, nullptr, -1);
  s.dat(1, 4, OP_WRITE, nullptr, -1);
  s.dat(2, 4, OP_RW, nullptr, -1);
  s.dat(3, 1, OP_READ, nullptr, -1);
  s.gbl(4, 1, OP_INC, 8);
  if (nargs == 8) {
    s.gbl(5, 1, OP_MAX, 8);
    if (s.ok && (a[6].argtype != OP_ARG_IDX || a[6].idx != -1 || a[6].map != nullptr))
      s.fail(6, "expected op_arg_idx(-1, OP_ID)");
    if (s.ok && (a[7].argtype != OP_ARG_INFO || a[7].idx != 5 || a[7].dim != 1 ||
                 a[7].size != 4 || !a[7].data))
      s.fail(7, "expected op_arg_info(&int, 1, \"int\", 5)");
  }
  int rb = s.real_bytes({0, 1, 2, 3});
  if (!s.ok) return kSigMismatch;
  if (a[4].type && strcmp(a[4].type, "double") != 0) return s.fail(4, "rms must be double"), kSigMismatch;
  Runtime &r = rt();
  // a renamed save_soln of exactly this q into this qold: read q's array as
  // qold, write the new q into qold's array, then swap the two
  const bool rename = r.lazy.src == a[1].dat && r.lazy.dst == a[0].dat && a[2].dat != a[0].dat &&
                      a[2].dat != a[1].dat && a[3].dat != a[0].dat && a[3].dat != a[1].dat;
  if (r.sres_stage && !r.settle_res()) return -1;  // update reads res
  if (r.res_zero && !r.materialize_res()) return -1;
  if (rename ? (r.pend.kind && !r.flush_loop()) : (r.outstanding() && !r.flush_pending())) return -1;
  int C = set->size;
  double bytes = (double)rb * 17.0 * C;
  char *qin = rename ? a[1].dat->data_d : a[0].dat->data_d;
  char *qout = rename ? a[0].dat->data_d : a[1].dat->data_d;
  // res: read, and recorded as zero instead of written (res_zero)
  cudaStreamCaptureStatus rcap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(r.stream, &rcap);
  const bool keep_res = r.opt_lazy_res && rcap == cudaStreamCaptureStatusNone &&
                        !r.exposed.count(a[2].dat) && r.overlays.empty() &&
                        a[2].dat != a[0].dat && a[2].dat != a[1].dat && a[2].dat != a[3].dat;
  if (keep_res) bytes -= 4.0 * rb * C;
  r.red.seq = ++r.red_seq;
  // speculation: this update's q is the q the last adt_calc read, and adt
  // is what it wrote -- compute the next adt_calc's result now, into the
  // shadow buffer, in the same pass over the cells
  SpecAdt &sp = r.spec;
  if (sp.inplace && !r.restore_spec()) return -1;  // update reads the program's adt
  bool spec = r.opt_speculate && sp.pcell && sp.q == a[1].dat && sp.adt == a[3].dat &&
              sp.rb == rb && sp.pcell->from == set && sp.x && sp.pcell->to == sp.x->set &&
              !r.exposed.count(sp.x) && !r.exposed.count(sp.q) && !r.exposed.count(sp.adt) &&
              r.overlays.empty();
  const size_t abytes = ((size_t)C * rb + 255) & ~(size_t)255;
  if (spec && sp.shadow_bytes < abytes) {
    cudaFree(sp.shadow);
    sp.shadow = nullptr;
    sp.shadow_bytes = 0;
    if (cudaMalloc(&sp.shadow, abytes) == cudaSuccess) sp.shadow_bytes = abytes;
    else spec = false, cudaGetLastError();
  }
  bool ok = true;
  if (spec) {
    if (rb == 8) sp.kd = air_consts<double>(ok);
    else sp.kf = air_consts<float>(ok);
    spec = ok;
  }
  const int N = spec ? sp.x->set->size : 0;
  r.begin_loop(spec ? "update+adt_calc" : name);
  cudaError_t e;
  if (rb == 8)
    e = launch_update<double>(r.ctx(), C, (const double *)qin, (double *)qout,
                              (double *)a[2].dat->data_d,
                              (const double *)a[3].dat->data_d, r.red,
                              spec ? sp.pcell->map_d : nullptr,
                              spec ? (const double *)sp.x->data_d : nullptr,
                              spec ? (double *)sp.shadow : nullptr, &sp.kd, keep_res,
                              r.opt_update_rev != 0);
  else
    e = launch_update<float>(r.ctx(), C, (const float *)qin, (float *)qout,
                             (float *)a[2].dat->data_d,
                             (const float *)a[3].dat->data_d, r.red,
                             spec ? sp.pcell->map_d : nullptr,
                             spec ? (const float *)sp.x->data_d : nullptr,
                             spec ? (float *)sp.shadow : nullptr, &sp.kf, keep_res,
                             r.opt_update_rev != 0);
  // with the speculation the pass also reads pcell and x and writes adt
  r.end_loop(spec ? bytes + 16.0 * C + (double)rb * (2.0 * N + C) : bytes);
  sp.inplace = spec && e == cudaSuccess;
  if (finish(e, name)) return -1;
  if (keep_res) r.res_zero = a[2].dat;
  if (rename) {
    std::swap(a[0].dat->data_d, a[1].dat->data_d);
    r.lazy = LazySave{};
  }
  // queue the res_calc + bres_calc that usually follow before waiting
  launch_speculative_res(r, a, rb);
  // gbl results are valid when op_par_loop returns: the kernel's last block
  // publishes them in the mapped page, sequence number last
  volatile RedSlot *h = reinterpret_cast<volatile RedSlot *>(r.pinned);
  if (!wait_for_sequence(&h->pad, r.red.seq, "op_par_loop(update): reduction read-back"))
    return -1;
  if (C == 0) return 0;
  *reinterpret_cast<double *>(a[4].data) += h->sum;
  if (nargs == 8) {
    double *mx = reinterpret_cast<double *>(a[5].data);
    if (h->maxv > *mx) {
      *mx = h->maxv;
      *reinterpret_cast<int *>(a[7].data) = (int)h->idx;
    }
  }
  return 0;
}

struct Entry {
  const char *name;
  int (*fn)(const char *, op_set, int, op_arg *);
};
const Entry kLoops[] = {{"save_soln", loop_save_soln},
                        {"adt_calc", loop_adt_calc},
                        {"res_calc", loop_res_calc},
                        {"bres_calc", loop_bres_calc},
                        {"update", loop_update}};

}  // namespace

// Launch the deferred loop on its own (the calls it could have been fused
// with did not follow).  Errors are reported by the call that triggered it.
// Put the program's adt back: the update before wrote the next adt_calc's
// result into adt early, and something other than that adt_calc came first.
bool op2b::Runtime::restore_spec() {
  // the adt dat's array still holds the program's adt: drop the early values
  if (spec.inplace) count_call("adt ahead dropped");
  spec.inplace = false;
  return true;
}

bool op2b::Runtime::flush_pending() {
  bool ok = settle_res();
  ok = flush_loop() && ok;
  ok = materialize_save() && ok;
  return materialize_res() && ok;
}

bool op2b::Runtime::materialize_res() {
  if (!res_zero) return true;
  op_dat d = res_zero;
  res_zero = nullptr;
  count_call("res zeroed");
  cudaError_t e = cudaMemsetAsync(d->data_d, 0, (size_t)d->set->size * d->size, stream);
  return finish(e, "res zeroed") == 0;
}

// Undo a speculative res_calc + bres_calc: the update before it left res
// zero.  At stage 2 the program has called res_calc (and not bres_calc):
// that call is deferred again, to be fused or launched as usual.
bool op2b::Runtime::settle_res() {
  if (!sres_stage) return true;
  const int st = sres_stage;
  sres_stage = 0;
  const ResLearn &L = rlearn;
  count_call("res_calc+bres_calc undone");
  if (res_zero != L.res) {  // (with res recorded as zero, nothing to undo in memory)
    cudaError_t e = cudaMemsetAsync(L.res->data_d, 0, (size_t)L.res->set->size * L.res->size,
                                    stream);
    if (e != cudaSuccess) return finish(e, "res_calc+bres_calc undo") == 0;
  }
  if (st == 2) {
    bool ok = pend.kind == 0 || flush_loop();
    pend = PendingLoop{};
    pend.kind = 2;
    pend.set = L.eset;
    pend.pedge = L.pedge;
    pend.pecell = L.pecell;
    pend.x = L.x;
    pend.q = L.q;
    pend.adt = L.adt;
    pend.res = L.res;
    pend.rb = L.rb;
    pend.bytes = L.res_bytes;
    pend.kd = L.kd;
    pend.kf = L.kf;
    return ok;
  }
  return true;
}

bool op2b::Runtime::materialize_save() {
  if (!lazy.src) return true;
  LazySave ls = lazy;
  lazy = LazySave{};
  const size_t bytes = (size_t)ls.src->set->size * (size_t)ls.src->size;
  begin_loop("save_soln");
  cudaError_t e = launch_copy(ctx(), ls.src->data_d, ls.dst->data_d, bytes);
  end_loop(2.0 * (double)bytes);
  return finish(e, "save_soln") == 0;
}

bool op2b::Runtime::flush_loop() {
  PendingLoop pd = pend;
  pend = PendingLoop{};
  cudaError_t e = cudaSuccess;
  if (pd.kind == 1) {
    size_t bytes = (size_t)pd.set->size * (size_t)pd.src->size;
    begin_loop("save_soln");
    e = launch_copy(ctx(), pd.src->data_d, pd.dst->data_d, bytes);
    end_loop(pd.bytes);
    return finish(e, "save_soln") == 0;
  }
  if (pd.kind == 2) {
    const SlotRecords *cr = get_corner_records(pd.pecell, pd.pedge);
    if (!cr) return false;
    if (res_zero == pd.res && !materialize_res()) return false;
    begin_loop("res_calc");
    ring_used = opt_gather_kernel == OP2B_GATHER_RING && build_ring_records(cr, nsm, 256);
    if (pd.rb == 8)
      e = ring_used
              ? launch_res_ring<double>(ctx(), *cr, nullptr, (const double *)pd.x->data_d,
                                        (const double *)pd.q->data_d,
                                        (const double *)pd.adt->data_d, (double *)pd.res->data_d,
                                        pd.kd, false)
              : launch_res_calc_gather_corner<double>(ctx(), *cr, (const double *)pd.x->data_d,
                                                      (const double *)pd.q->data_d,
                                                      (const double *)pd.adt->data_d,
                                                      (double *)pd.res->data_d, pd.kd,
                                                      opt_pipe_block, opt_gather_minb);
    else
      e = ring_used
              ? launch_res_ring<float>(ctx(), *cr, nullptr, (const float *)pd.x->data_d,
                                       (const float *)pd.q->data_d, (const float *)pd.adt->data_d,
                                       (float *)pd.res->data_d, pd.kf, false)
              : launch_res_calc_gather_corner<float>(ctx(), *cr, (const float *)pd.x->data_d,
                                                     (const float *)pd.q->data_d,
                                                     (const float *)pd.adt->data_d,
                                                     (float *)pd.res->data_d, pd.kf,
                                                     opt_pipe_block, opt_gather_minb);
    end_loop(pd.bytes);
    return finish(e, "res_calc") == 0;
  }
  return true;
}

extern "C" {

int op_par_loop_c(char const *name, op_set set, int nargs, op_arg *args) {
  Runtime &r = rt();
  if (!r.initialised) {
    set_error("op_init has not been called");
    return -1;
  }
  if (!name || !set || (nargs > 0 && !args)) {
    set_error("op_par_loop: needs a name, a set and the argument list");
    return -1;
  }
  for (const Entry &e : kLoops)
    if (strcmp(e.name, name) == 0) {
      // with a kernel source to fall back on, a signature mismatch is not
      // reported: the application's own loop of that name runs instead
      const bool fallback = jit_has_kernel(name);
      r.quiet_errors = fallback;
      int rc = e.fn(name, set, nargs, args);
      r.quiet_errors = false;
      if (rc != kSigMismatch) {
        if (rc != 0 && fallback) set_error("%s", op2b_last_error());  // report it now
        return rc;
      }
      // an application's own loop that shares a name with an Airfoil loop
      // but not its arguments: run its kernel source if it has one
      if (!jit_has_kernel(name)) return -1;
      break;
    }
  if (r.outstanding() && !r.flush_pending()) return -1;
  if (r.spec.inplace && !r.restore_spec()) return -1;
  // no hand-written kernel: the application's own kernel source, compiled at
  // run time, if it has one
  if (jit_has_kernel(name)) return jit_par_loop(name, set, nargs, args);
  set_error("op_par_loop(%s): no device implementation of this loop is registered "
            "(libop2b runs loops on the GPU only)",
            name);
  return -1;
}

static void stub(const char *name, op_set set, std::initializer_list<op_arg> args) {
  std::vector<op_arg> v(args);
  if (op_par_loop_c(name, set, (int)v.size(), v.data()) != 0 && !rt().opt_abort)
    fprintf(stderr, "op2b: %s\n", op2b_last_error());
}

void op_par_loop_save_soln(char const *name, op_set set, op_arg a0, op_arg a1) {
  stub(name, set, {a0, a1});
}
void op_par_loop_adt_calc(char const *name, op_set set, op_arg a0, op_arg a1, op_arg a2,
                          op_arg a3, op_arg a4, op_arg a5) {
  stub(name, set, {a0, a1, a2, a3, a4, a5});
}
void op_par_loop_res_calc(char const *name, op_set set, op_arg a0, op_arg a1, op_arg a2,
                          op_arg a3, op_arg a4, op_arg a5, op_arg a6, op_arg a7) {
  stub(name, set, {a0, a1, a2, a3, a4, a5, a6, a7});
}
void op_par_loop_bres_calc(char const *name, op_set set, op_arg a0, op_arg a1, op_arg a2,
                           op_arg a3, op_arg a4, op_arg a5) {
  stub(name, set, {a0, a1, a2, a3, a4, a5});
}
void op_par_loop_update(char const *name, op_set set, op_arg a0, op_arg a1, op_arg a2,
                        op_arg a3, op_arg a4, op_arg a5, op_arg a6, op_arg a7) {
  stub(name, set, {a0, a1, a2, a3, a4, a5, a6, a7});
}

}  // extern "C"
