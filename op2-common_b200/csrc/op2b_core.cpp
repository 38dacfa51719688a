// Host runtime of libop2b: the OP2 C API (include/op2b.h) on one B200.
//
// Semantics follow the reference core (op2/src/core/op_lib_core.cpp):
//  * op_decl_set/map/dat copy the caller's arrays (op_lib_core.cpp:420-576);
//    the caller may free them afterwards.  Maps are range-checked on
//    declaration (check_map, :146-164) and stored on the device AoS.
//  * dats live only in device memory; op_fetch_data* copy them out.
//  * op_par_loop runs the device loop registered under the loop's name after
//    checking the argument list against that loop's signature (dats, dims,
//    maps, indices, access modes); gbl reductions are written back into the
//    caller's variables before the call returns, INC adding to the initial
//    value and MAX keeping the larger (translator-v2/resources/templates/cpp/
//    cuda/loop_host.hpp.jinja:405-415).
//  * there is no host execution path: an unknown loop name, a signature
//    mismatch or a CUDA error is reported through op2b_last_error() and, for
//    the void-returning reference entry points, printed (and fatal when
//    OP2B_ABORT_ON_ERROR / option "abort_on_error" is set).
#include "op2b.h"
#include "op2b_runtime.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <thread>

#include <sys/mman.h>
#include <vector>

namespace op2b {

Runtime &rt() {
  static Runtime r;
  return r;
}

static thread_local std::string g_last_error;

void set_error(const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  if (rt().quiet_errors) return;  // a tentative call: the caller decides
  if (rt().opt_diags > 0 || rt().opt_abort)
    fprintf(stderr, "op2b error: %s\n", buf);
  if (rt().opt_abort)
    exit(1);
}

bool cuda_ok(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return true;
  set_error("%s: CUDA error %d (%s)", what, (int)e, cudaGetErrorString(e));
  return false;
}

// A pool of host threads for large memcpys, started at the first use and
// kept for the process: copying into freshly allocated memory is bound by
// its page faults, which the kernel serves in parallel, and a staged
// download copies many chunks in a row (starting threads per chunk would
// cost more than some of the copies).
namespace {
struct CopyPool {
  std::mutex user;  // one job at a time (callers on several host threads wait their turn)
  std::mutex mu;
  std::condition_variable go, done;
  std::vector<std::thread> workers;
  // the current job: worker i copies part i + 1 (the caller part 0)
  char *dst = nullptr;
  const char *src = nullptr;
  size_t bytes = 0, part = 0;
  unsigned parts = 0, pending = 0;
  unsigned long long gen = 0;
  bool quit = false;

  void start(unsigned n) {
    for (unsigned i = (unsigned)workers.size(); i < n; i++)
      workers.emplace_back([this, i] {
        unsigned long long seen = 0;
        for (;;) {
          char *d;
          const char *sp;
          size_t b, e;
          {
            std::unique_lock<std::mutex> lk(mu);
            go.wait(lk, [&] { return quit || gen != seen; });
            if (quit) return;
            seen = gen;
            if (i + 1 >= parts) continue;  // not part of this job
            d = dst;
            sp = src;
            b = (i + 1) * part;
            e = std::min(bytes, b + part);
          }
          if (b < e) memcpy(d + b, sp + b, e - b);
          std::lock_guard<std::mutex> lk(mu);
          if (--pending == 0) done.notify_one();
        }
      });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lk(mu);
      quit = true;
    }
    go.notify_all();
    for (auto &t : workers) t.join();
  }
  void copy(void *d, const void *sp, size_t n, unsigned nt) {
    std::lock_guard<std::mutex> one(user);
    start(nt - 1);
    {
      std::lock_guard<std::mutex> lk(mu);
      dst = (char *)d;
      src = (const char *)sp;
      bytes = n;
      parts = nt;
      part = ((n + nt - 1) / nt + 4095) & ~(size_t)4095;
      pending = nt - 1;
      gen++;
    }
    go.notify_all();
    memcpy(d, sp, std::min(part, n));
    std::unique_lock<std::mutex> lk(mu);
    done.wait(lk, [&] { return pending == 0; });
  }
};

CopyPool &copy_pool() {
  static CopyPool p;
  return p;
}
}  // namespace

// memcpy of a large host array by up to `host_threads` threads (option,
// default 8, at most the host's)
static void host_copy(void *dst, const void *src, size_t bytes) {
  const size_t kParallel = (size_t)2 << 20;
  unsigned nt = std::min((unsigned)std::max(1, rt().opt_host_threads),
                         std::max(1u, std::thread::hardware_concurrency()));
  if (bytes < kParallel || nt < 2) {
    memcpy(dst, src, bytes);
    return;
  }
  copy_pool().copy(dst, src, bytes, nt);
}

// Device -> host copies of several arrays, one pipeline through the pinned
// staging buffers: chunk k of the whole list goes through buffer k % 2, its
// DMA under way while the host threads empty the other buffer; a pinned
// destination takes its DMA directly.  Synchronous.
// The pinned staging buffers of large device -> host copies: pinning them
// takes tens of milliseconds, so op_renumber has a thread do it while the
// device orders the mesh (the first copy that needs them, or op_exit, waits
// for it); without a renumbering the first large copy pins them itself.
void stage_in_background() {
  Runtime &r = rt();
  if (!r.opt_host_staging || r.stage || r.stage_alloc.joinable()) return;
  const int dev = r.device;
  r.stage_alloc = std::thread([&r, dev] {
    char *p = nullptr;
    if (cudaSetDevice(dev) == cudaSuccess &&
        cudaHostAlloc((void **)&p, 2 * kStageChunk, cudaHostAllocDefault) == cudaSuccess)
      r.stage = p;
    else
      cudaGetLastError();
  });
}

bool download_host_many(const std::vector<HostDownload> &jobs, const char *what) {
  Runtime &r = rt();
  const size_t kChunk = kStageChunk;
  struct Piece {
    char *dst;
    const char *src;
    size_t len;
  };
  std::vector<Piece> pieces;
  for (const auto &j : jobs) {
    if (!j.bytes) continue;
    cudaPointerAttributes pa{};
    const bool pinned = cudaPointerGetAttributes(&pa, j.dst) == cudaSuccess &&
                        pa.type == cudaMemoryTypeHost;
    cudaGetLastError();
    if (pinned || j.bytes <= ((size_t)1 << 20)) {  // straight DMA, on the stream in order
      if (!cuda_ok(cudaMemcpyAsync(j.dst, j.src_d, j.bytes, cudaMemcpyDeviceToHost, r.stream),
                   what))
        return false;
      continue;
    }
    for (size_t off = 0; off < j.bytes; off += kChunk)
      pieces.push_back({(char *)j.dst + off, (const char *)j.src_d + off,
                        std::min(kChunk, j.bytes - off)});
  }
  if (pieces.empty()) return cuda_ok(cudaStreamSynchronize(r.stream), what);
  if (!r.opt_host_staging) {  // the driver's own copies into pageable memory
    const auto t0 = std::chrono::steady_clock::now();
    size_t total = 0;
    for (const auto &p : pieces) {
      if (!cuda_ok(cudaMemcpyAsync(p.dst, p.src, p.len, cudaMemcpyDeviceToHost, r.stream), what))
        return false;
      total += p.len;
    }
    const bool ok = cuda_ok(cudaStreamSynchronize(r.stream), what);
    if (r.opt_diags > 2) {
      const double ms = std::chrono::duration<double, std::milli>(
                            std::chrono::steady_clock::now() - t0).count();
      fprintf(stderr, "%s: %.1f MB by the driver's pageable copies in %.2f ms (%.1f GB/s)\n",
              what, total / 1e6, ms, total / 1e6 / ms);
    }
    return ok;
  }
  const auto t0 = std::chrono::steady_clock::now();
  if (r.stage_alloc.joinable()) r.stage_alloc.join();
  if (!r.stage &&
      !cuda_ok(cudaHostAlloc((void **)&r.stage, 2 * kChunk, cudaHostAllocDefault), what))
    return false;
  for (auto &e : r.stage_ev)
    if (!e && !cuda_ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), what)) return false;
  const auto t1 = std::chrono::steady_clock::now();
  size_t total = 0;
  for (const auto &p : pieces) total += p.len;
  auto issue = [&](size_t k) {
    return cuda_ok(cudaMemcpyAsync(r.stage + (k % 2) * kChunk, pieces[k].src, pieces[k].len,
                                   cudaMemcpyDeviceToHost, r.stream),
                   what) &&
           cuda_ok(cudaEventRecord(r.stage_ev[k % 2], r.stream), what);
  };
  if (!issue(0)) return false;
  for (size_t i = 0; i < pieces.size(); i++) {
    if (i + 1 < pieces.size() && !issue(i + 1)) return false;
    if (!cuda_ok(cudaEventSynchronize(r.stage_ev[i % 2]), what)) return false;
    host_copy(pieces[i].dst, r.stage + (i % 2) * kChunk, pieces[i].len);
  }
  const bool ok = cuda_ok(cudaStreamSynchronize(r.stream), what);
  if (r.opt_diags > 2) {
    const auto t2 = std::chrono::steady_clock::now();
    const double a_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    const double c_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
    fprintf(stderr, "%s: %.1f MB through staging in %.2f ms (%.1f GB/s), staging set up in "
            "%.2f ms\n", what, total / 1e6, c_ms, total / 1e6 / c_ms, a_ms);
  }
  return ok;
}

bool download_host(void *dst, const void *src_d, size_t bytes, const char *what) {
  return download_host_many({HostDownload{dst, src_d, bytes}}, what);
}

// Host memory for large copies: 2 MiB aligned with a transparent-huge-page
// hint, so that filling it takes few page faults (free() releases it).
static void *host_alloc(size_t bytes) {
  const size_t kHuge = (size_t)2 << 20;
  if (bytes < 2 * kHuge) return malloc(bytes);
  void *p = nullptr;
  if (posix_memalign(&p, kHuge, bytes) != 0) return nullptr;
  madvise(p, (bytes + kHuge - 1) & ~(kHuge - 1), MADV_HUGEPAGE);
  return p;
}

static char *copy_str(const char *s) {
  if (!s) s = "";
  size_t n = strlen(s);
  char *d = (char *)malloc(n + 1);
  memcpy(d, s, n + 1);
  return d;
}

int type_bytes(const char *type) {
  if (!type) return 0;
  std::string t(type);
  size_t c = t.find(':');
  if (c != std::string::npos) t = t.substr(0, c);
  if (t == "double") return 8;
  if (t == "float") return 4;
  if (t == "int" || t == "uint") return 4;
  if (t == "ll" || t == "ull" || t == "long") return 8;
  if (t == "bool") return 1;
  return 0;
}

bool is_real(const char *type, int bytes) {
  if (!type) return false;
  std::string t(type);
  size_t c = t.find(':');
  if (c != std::string::npos) t = t.substr(0, c);
  return (bytes == 8 && t == "double") || (bytes == 4 && t == "float");
}

LaunchCtx Runtime::ctx() { return LaunchCtx{stream, nsm, &launches, opt_pdl != 0}; }

// launch a deferred loop before a call that observes the library's state
// (restore: also put adt back if an update wrote it early -- for calls that
// hand out access to the data; bookkeeping calls only launch deferred loops)
static void flush_quiet(bool restore = true) {
  Runtime &r = rt();
  if (r.initialised && r.outstanding()) r.flush_pending();
  if (restore && r.initialised && r.spec.inplace) r.restore_spec();
}

bool Runtime::ready() {
  if (!initialised) {
    set_error("op_init has not been called");
    return false;
  }
  return (!outstanding() || flush_pending()) && (!spec.inplace || restore_spec());
}

// ------------------------------------------------------------------ timing

// Device time per loop by CUDA events around its launches: one call in
// opt_timing_stride of each loop (every call inside a profiled region), so
// that the events, which keep consecutive kernels from overlapping their
// launch, stay off most calls.  Totals are the sampled mean times the calls.
void Runtime::begin_loop(const char *name) {
  cur_loop = name;
  cur_ev0 = cur_ev1 = nullptr;
  if (!opt_timing) return;
  const long calls = stats[cur_loop].calls;
  if (opt_timing_stride > 1 && calls % opt_timing_stride != 0 && !profile_times_loops()) return;
  if (ev_free.size() < 2) {
    for (int i = 0; i < 64; i++) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) == cudaSuccess) ev_free.push_back(e);
    }
  }
  cur_ev0 = ev_free.back();
  ev_free.pop_back();
  cur_ev1 = ev_free.back();
  ev_free.pop_back();
  cudaEventRecord(cur_ev0, stream);
}

void Runtime::end_loop(double bytes) {
  LoopStat &s = stats[cur_loop];
  s.calls++;
  s.bytes_per_call = bytes;
  if (!opt_timing || !cur_ev0) return;
  cudaEventRecord(cur_ev1, stream);
  pending.push_back(PendingTime{cur_loop, cur_ev0, cur_ev1, profile_loop_node(cur_loop)});
  if (pending.size() > 4096) resolve_timing();
}

void Runtime::resolve_timing() {
  if (pending.empty()) return;
  cudaStreamSynchronize(stream);
  for (auto &p : pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.e0, p.e1) == cudaSuccess) {
      if (!p.name.empty()) {
        LoopStat &s = stats[p.name];
        s.total_ms += ms;
        s.last_ms = ms;
        s.timed++;
      }
      if (p.node >= 0) profile_submit(p.node, ms);
    }
    ev_free.push_back(p.e0);
    ev_free.push_back(p.e1);
  }
  pending.clear();
}

const double *Runtime::const_ptr(const char *name, int dim) {
  auto it = consts.find(name);
  if (it == consts.end() || (int)it->second.size() < dim) {
    set_error("constant '%s' (dim %d) was not declared with op_decl_const", name, dim);
    return nullptr;
  }
  return it->second.data();
}

}  // namespace op2b

using namespace op2b;

// ====================================================================== C API

extern "C" {

const char *op2b_last_error(void) { return g_last_error.c_str(); }

int op2b_status(void) { return rt().initialised ? 0 : -1; }

static void parse_args(int argc, char **argv) {
  Runtime &r = rt();
  for (int i = 0; i < argc; i++) {
    if (!argv || !argv[i]) continue;
    const char *a = argv[i];
    const char *p;
    if ((p = strstr(a, "OP_BLOCK_SIZE="))) r.opt_block_size = atoi(p + 14);
    if ((p = strstr(a, "OP_PART_SIZE="))) r.opt_part_size = atoi(p + 13);
    if ((p = strstr(a, "OP_CACHE_LINE_SIZE="))) r.opt_cache_line = atoi(p + 19);
    if ((p = strstr(a, "OP_MAPS_BASE_INDEX="))) {
      int v = atoi(p + 19);
      if (v == 0 || v == 1) r.opt_maps_base = v;
    }
  }
}

void op_init(int argc, char **argv, int diags) {
  Runtime &r = rt();
  if (r.initialised) return;
  r.opt_diags = diags;
  if (const char *e = getenv("OP2B_ABORT_ON_ERROR")) r.opt_abort = atoi(e) != 0;
  if (const char *e = getenv("OP2B_INC_MODE")) r.opt_inc_mode = atoi(e);
  if (const char *e = getenv("OP2B_JIT_EXACT")) r.opt_jit_exact = atoi(e) != 0;
  parse_args(argc, argv);
  int dev = 0;
  if (const char *e = getenv("OP2B_DEVICE")) dev = atoi(e);
  if (!cuda_ok(cudaSetDevice(dev), "op_init: cudaSetDevice")) return;
  cudaDeviceProp prop;
  if (!cuda_ok(cudaGetDeviceProperties(&prop, dev), "op_init: cudaGetDeviceProperties")) return;
  r.device = dev;
  r.nsm = prop.multiProcessorCount;
  r.cc_major = prop.major;
  r.cc_minor = prop.minor;
  if (r.cc_major != 10) {
    set_error("op_init: device %d is sm_%d%d; libop2b is built for sm_100a (B200) only", dev,
              r.cc_major, r.cc_minor);
    return;
  }
  if (!cuda_ok(cudaStreamCreateWithFlags(&r.own_stream, cudaStreamNonBlocking),
               "op_init: stream"))
    return;
  r.stream = r.own_stream;
  // update-reduction scratch: partial slots + ticket + final slot
  r.red.capacity = 8192;
  void *p = nullptr;
  size_t bytes = sizeof(RedSlot) * (size_t)(r.red.capacity + 1) + 256;
  if (!cuda_ok(cudaMalloc(&p, bytes), "op_init: reduction scratch")) return;
  cudaMemset(p, 0, bytes);
  r.red_base = p;
  r.red.parts = reinterpret_cast<RedSlot *>(p);
  r.red.out = r.red.parts + r.red.capacity;
  r.red.counter = reinterpret_cast<unsigned *>(reinterpret_cast<char *>(r.red.out + 1));
  // mapped pinned page: the update kernel writes its reduction result here
  if (!cuda_ok(cudaHostAlloc(&r.pinned, 4096, cudaHostAllocMapped), "op_init: pinned buffer"))
    return;
  memset(r.pinned, 0, 4096);
  if (!cuda_ok(cudaHostGetDevicePointer(&r.pinned_dev, r.pinned, 0), "op_init: mapped pointer"))
    return;
  r.red.host_out = reinterpret_cast<RedSlot *>(r.pinned_dev);
  if (!cuda_ok(cudaMalloc((void **)&r.check_d, 256), "op_init: map check word")) return;
  // setup temporaries (renumbering, inverse maps, records) come from the
  // device's stream-ordered pool: kept in the pool between uses instead of
  // returned to the driver, so repeated setup makes no driver calls
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  r.initialised = true;
  if (diags > 1)
    printf(" op2b: device %d (%s, %d SMs), stream %p\n", dev, prop.name, r.nsm,
           (void *)r.stream);
}

void op_exit(void) {
  Runtime &r = rt();
  if (!r.initialised) return;
  if (r.outstanding()) r.flush_pending();
  cudaStreamSynchronize(r.stream);
  release_plans();
  release_inverse_maps();
  release_renumbering();
  for (auto &d : r.dats)
    if (d) {
      if (!r.overlays.count(d.get())) {  // overlays share their dat's storage
        cudaFree(d->data_d);
        free(d->data);
      }
      free((void *)d->name);
      free((void *)d->type);
    }
  for (auto &m : r.maps)
    if (m) {
      cudaFree(m->map_d);
      free(m->map);
      free((void *)m->name);
    }
  for (auto &s : r.sets)
    if (s) free((void *)s->name);
  r.dats.clear();
  r.maps.clear();
  r.sets.clear();
  r.consts.clear();
  r.const_types.clear();
  release_jit();
  r.map_ptrs.clear();
  r.resolve_timing();  // the loop table and the profiler keep their last times
  profile_on_exit();
  for (auto &p : r.pending) {
    cudaEventDestroy(p.e0);
    cudaEventDestroy(p.e1);
  }
  r.pending.clear();
  for (auto e : r.ev_free) cudaEventDestroy(e);
  r.ev_free.clear();
  cudaFree(r.spec.shadow);
  r.spec = SpecAdt{};
  cudaFree(r.red_base);
  cudaFree(r.check_d);
  r.check_d = nullptr;
  cudaFreeHost(r.pinned);
  if (r.stage_alloc.joinable()) r.stage_alloc.join();
  cudaFreeHost(r.stage);
  r.stage = nullptr;
  for (auto &e : r.stage_ev) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
  cudaStreamSynchronize(r.own_stream);
  cudaStreamDestroy(r.own_stream);
  cudaMemPool_t pool;  // give the pooled setup memory back
  if (cudaDeviceGetDefaultMemPool(&pool, r.device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
  r.red_base = nullptr;
  r.pinned = nullptr;
  r.stream = r.own_stream = nullptr;
  r.stats.clear();
  r.exposed.clear();
  r.zero_mirror.clear();
  r.overlays.clear();
  r.orig_ptrs.clear();
  r.launches = 0;
  r.initialised = false;
  // options return to their defaults: a later op_init starts from a clean state
  const Runtime d{};
  r.opt_diags = d.opt_diags;
  r.opt_abort = d.opt_abort;
  r.opt_timing = d.opt_timing;
  r.opt_block_size = d.opt_block_size;
  r.opt_part_size = d.opt_part_size;
  r.opt_cache_line = d.opt_cache_line;
  r.opt_maps_base = d.opt_maps_base;
  r.opt_inc_mode = d.opt_inc_mode;
  r.opt_gather_kernel = d.opt_gather_kernel;
  r.opt_gather_minb = d.opt_gather_minb;
  r.opt_bres_kernel = d.opt_bres_kernel;
  r.opt_adt_minb = d.opt_adt_minb;
  r.opt_fuse = d.opt_fuse;
  r.opt_speculate = d.opt_speculate;
  r.opt_host_mirror = d.opt_host_mirror;
  r.opt_rename_save = d.opt_rename_save;
  r.opt_speculate_res = d.opt_speculate_res;
  r.opt_lazy_res = d.opt_lazy_res;
  r.opt_host_threads = d.opt_host_threads;
  r.res_zero = nullptr;
  r.lazy = LazySave{};
  r.rlearn = ResLearn{};
  r.sres_stage = 0;
  r.pend = PendingLoop{};
  r.opt_pipe_block = d.opt_pipe_block;
  r.opt_pipe_hints = d.opt_pipe_hints;
  r.opt_plan_mode = d.opt_plan_mode;
  r.opt_atomic_seg = d.opt_atomic_seg;
  r.opt_jit_warp = d.opt_jit_warp;
  r.opt_jit_exact = d.opt_jit_exact;
  r.opt_update_rev = d.opt_update_rev;
  r.opt_atomic_blocks = d.opt_atomic_blocks;
  r.ring_used = 0;
  r.opt_gemm_tma = d.opt_gemm_tma;
  r.opt_gemm_ws = d.opt_gemm_ws;
  r.opt_gemm_rows = d.opt_gemm_rows;
  r.opt_pdl = d.opt_pdl;
  r.opt_timing_stride = d.opt_timing_stride;
  r.opt_host_staging = d.opt_host_staging;
  r.opt_check_plans = d.opt_check_plans;
}

op_set op_decl_set(int size, char const *name) {
  if (!rt().ready()) return nullptr;
  if (size < 0) {
    set_error("op_decl_set: negative size for set %s", name ? name : "");
    return nullptr;
  }
  auto s = std::make_unique<op_set_core>();
  s->index = (int)rt().sets.size();
  s->size = size;
  s->name = copy_str(name);
  s->core_size = size;
  s->exec_size = 0;
  s->nonexec_size = 0;
  rt().sets.push_back(std::move(s));
  return rt().sets.back().get();
}

op_map op_decl_map(op_set from, op_set to, int dim, int *imap, char const *name) {
  Runtime &r = rt();
  if (!r.ready()) return nullptr;
  if (!from || !to) {
    set_error("op_decl_map: invalid 'from'/'to' set for map %s", name ? name : "");
    return nullptr;
  }
  if (dim <= 0) {
    set_error("op_decl_map: non-positive dimension for map %s", name ? name : "");
    return nullptr;
  }
  size_t n = (size_t)from->size * (size_t)dim;
  if (n > 0 && !imap) {
    set_error("op_decl_map: NULL data for map %s", name ? name : "");
    return nullptr;
  }
  int *h = (int *)host_alloc(sizeof(int) * (n ? n : 1));
  int *map_d = nullptr;
  auto bad_entry = [&](size_t i) {
    set_error("op_decl_map: invalid data for map %s: element %zu, dimension %zu, value %d "
              "outside [0, %d)",
              name ? name : "", i / dim, i % dim, imap[i], to->size);
    free(h);
    cudaFree(map_d);
    return nullptr;
  };
  if (n > 0 && !cuda_ok(cudaMalloc((void **)&map_d, n * sizeof(int)), "op_decl_map: cudaMalloc")) {
    free(h);
    return nullptr;
  }
  if (r.opt_maps_base == 0) {
    // upload the caller's array as it is (a pinned array goes by DMA), check
    // the range on the device and take the host copy while the copy runs
    unsigned long long bad = ~0ull;
    if (n > 0) {
      if (!cuda_ok(cudaMemsetAsync(r.check_d, 0xff, sizeof(bad), r.stream), "op_decl_map") ||
          !cuda_ok(cudaMemcpyAsync(map_d, imap, n * sizeof(int), cudaMemcpyHostToDevice,
                                   r.stream),
                   "op_decl_map: upload") ||
          !cuda_ok(launch_map_check(r.ctx(), map_d, (long long)n, to->size, r.check_d),
                   "op_decl_map: range check")) {
        free(h);
        cudaFree(map_d);
        return nullptr;
      }
      host_copy(h, imap, sizeof(int) * n);
      if (!cuda_ok(cudaMemcpyAsync(&bad, r.check_d, sizeof(bad), cudaMemcpyDeviceToHost,
                                   r.stream),
                   "op_decl_map: range check") ||
          !cuda_ok(cudaStreamSynchronize(r.stream), "op_decl_map: upload")) {
        free(h);
        cudaFree(map_d);
        return nullptr;
      }
    }
    if (bad != ~0ull) return bad_entry((size_t)bad);
  } else {
    for (size_t i = 0; i < n; i++) {
      int v = imap[i] - r.opt_maps_base;
      if (v < 0 || v >= to->size) return bad_entry(i);
      h[i] = v;
    }
    if (n > 0 && !cuda_ok(cudaMemcpy(map_d, h, n * sizeof(int), cudaMemcpyHostToDevice),
                          "op_decl_map: upload")) {
      free(h);
      cudaFree(map_d);
      return nullptr;
    }
  }
  auto m = std::make_unique<op_map_core>();
  m->index = (int)r.maps.size();
  m->from = from;
  m->to = to;
  m->dim = dim;
  m->map = h;
  m->map_d = map_d;
  m->name = copy_str(name);
  if (imap) r.map_ptrs[imap] = m.get();  // op_register_map_ptr (op_lib_core.cpp:493-495)
  r.maps.push_back(std::move(m));
  return r.maps.back().get();
}

op_dat op_decl_dat_char(op_set set, int dim, char const *type, int type_size, char *data,
                        char const *name) {
  Runtime &r = rt();
  if (!r.ready()) return nullptr;
  if (!set) {
    set_error("op_decl_dat: invalid set for data %s", name ? name : "");
    return nullptr;
  }
  if (dim <= 0 || type_size <= 0) {
    set_error("op_decl_dat: non-positive dimension or type size for data %s",
              name ? name : "");
    return nullptr;
  }
  int tb = type_bytes(type);
  if (tb != 0 && tb != type_size) {
    set_error("op_decl_dat: type '%s' does not have size %d (data %s)", type, type_size,
              name ? name : "");
    return nullptr;
  }
  auto d = std::make_unique<op_dat_core>();
  d->index = (int)r.dats.size();
  d->set = set;
  d->dim = dim;
  d->size = dim * type_size;
  d->data = nullptr;
  d->data_d = nullptr;
  d->type = copy_str(type);
  d->name = copy_str(name);
  size_t bytes = (size_t)set->size * (size_t)d->size;
  if (bytes > 0) {
    // 256-byte aligned allocation rounded up to 32 bytes so every element
    // record and 16/32-byte vector access stays in bounds
    size_t alloc = (bytes + 255) & ~(size_t)255;
    if (!cuda_ok(cudaMalloc((void **)&d->data_d, alloc), "op_decl_dat: cudaMalloc")) return nullptr;
    // the host copy behind dat->data, as op_decl_dat_core keeps one
    // (op_lib_core.cpp:581-680; zeros for a NULL source), taken by host
    // threads while this one uploads the same source
    std::thread mirror;
    if (r.opt_host_mirror) {
      d->data = (char *)(data ? host_alloc(bytes) : calloc(bytes, 1));
      if (!d->data) {
        cudaFree(d->data_d);
        set_error("op_decl_dat: out of host memory for data %s", d->name);
        return nullptr;
      }
      if (data) mirror = std::thread([&] { host_copy(d->data, data, bytes); });
    }
    cudaError_t e = data ? cudaMemcpyAsync(d->data_d, data, bytes, cudaMemcpyHostToDevice, r.stream)
                         : cudaMemsetAsync(d->data_d, 0, alloc, r.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(r.stream);
    if (mirror.joinable()) mirror.join();
    if (!cuda_ok(e, "op_decl_dat: upload")) {
      cudaFree(d->data_d);
      free(d->data);
      return nullptr;
    }
  }
  if (d->data && !data) r.zero_mirror.insert(d.get());
  if (data) r.orig_ptrs[data] = d.get();  // for op_decl_dat_overlay_ptr
  r.dats.push_back(std::move(d));
  return r.dats.back().get();
}

// op_decl_dat_temp_core (op_lib_core.cpp:638-651): a dat of the same set,
// dim, type, size and name must not exist yet.
op_dat op_decl_dat_temp_char(op_set set, int dim, char const *type, int type_size,
                             char const *name) {
  Runtime &r = rt();
  for (auto &d : r.dats)
    if (d && d->set == set && d->dim == dim && d->size == dim * type_size &&
        strcmp(d->type, type ? type : "") == 0 && strcmp(d->name, name ? name : "") == 0) {
      set_error("op_dat with name %s already exists, cannot create temporary op_dat",
                name ? name : "");
      return nullptr;
    }
  return op_decl_dat_char(set, dim, type, type_size, nullptr, name);
}

// op_free_dat_temp_core (op_lib_core.cpp:653-680): 1 when the dat was
// found and freed, -1 otherwise.
int op_free_dat_temp_char(op_dat dat) {
  Runtime &r = rt();
  flush_quiet();
  // forget the learned arguments (flush_quiet put adt back), keep the buffer
  r.spec = SpecAdt{nullptr, nullptr, nullptr, nullptr, 0, false, r.spec.shadow,
                   r.spec.shadow_bytes};
  for (auto &d : r.dats)
    if (d.get() == dat) {
      cudaStreamSynchronize(r.stream);
      if (!r.overlays.count(dat)) {
        cudaFree(d->data_d);
        free(d->data);
      }
      free((void *)d->name);
      free((void *)d->type);
      if (r.rlearn.x == dat || r.rlearn.q == dat || r.rlearn.adt == dat || r.rlearn.res == dat ||
          r.rlearn.bound == dat)
        r.rlearn = ResLearn{};
      r.overlays.erase(dat);
      r.zero_mirror.erase(dat);
      r.exposed.erase(dat);
      for (auto it = r.orig_ptrs.begin(); it != r.orig_ptrs.end();)
        it = it->second == dat ? r.orig_ptrs.erase(it) : std::next(it);
      d.reset();
      return 1;
    }
  set_error("op_free_dat_temp: unknown dat");
  return -1;
}

// op_decl_dat_overlay (op_lib_core.cpp:581-636, op_cuda_decl.cpp:101-123):
// a dat on another set that shares `dat`'s storage, host and device; the
// set may not be larger than the dat's.
op_dat op_decl_dat_overlay(op_set set, op_dat dat) {
  Runtime &r = rt();
  if (!r.ready()) return nullptr;
  if (!set || !dat) {
    set_error("op_decl_dat_overlay error -- invalid set or dat");
    return nullptr;
  }
  if (set->size > dat->set->size) {
    set_error("op_decl_dat_overlay error -- new set size bigger than overlayed size (%d > %d)",
              set->size, dat->set->size);
    return nullptr;
  }
  if (r.opt_diags > 1)
    op_printf("op_decl_dat_overlay: dat: %s, set %s (%d elems) -> %s (%d elems)\n", dat->name,
              dat->set->name, dat->set->size, set->name, set->size);
  flush_quiet();
  auto d = std::make_unique<op_dat_core>(*dat);
  d->index = (int)r.dats.size();
  d->set = set;
  d->name = copy_str(dat->name);
  d->type = copy_str(dat->type);
  r.overlays.insert(d.get());
  r.dats.push_back(std::move(d));
  return r.dats.back().get();
}

op_dat op_decl_dat_overlay_ptr(op_set set, char *dat) {
  Runtime &r = rt();
  auto it = r.orig_ptrs.find(dat);
  if (it == r.orig_ptrs.end()) {
    set_error("op_decl_dat_overlay_ptr: op_dat not found for dat with %p pointer", (void *)dat);
    return nullptr;
  }
  return op_decl_dat_overlay(set, it->second);
}

void op_decl_const_char(int dim, char const *type, int type_size, char *dat, char const *name) {
  Runtime &r = rt();
  if (!name || !dat || dim <= 0) {
    set_error("op_decl_const: needs a name, data and a positive dimension");
    return;
  }
  std::vector<double> v((size_t)dim);
  std::string t = type ? type : "";
  for (int i = 0; i < dim; i++) {
    if (t == "double" && type_size == 8)
      v[i] = reinterpret_cast<double *>(dat)[i];
    else if (t == "float" && type_size == 4)
      v[i] = reinterpret_cast<float *>(dat)[i];
    else if (t == "int" && type_size == 4)
      v[i] = reinterpret_cast<int *>(dat)[i];
    else {
      set_error("op_decl_const: unsupported type '%s' for constant %s", type ? type : "", name);
      return;
    }
  }
  std::string n(name);
  while (!n.empty() && (n[0] == '&' || n[0] == ' ')) n.erase(0, 1);
  r.consts[n] = v;
  r.const_types[n] = t;
  r.const_version++;
}

// ------------------------------------------------------------------ op_arg

// op_arg keeps the type string beyond the call (the reference keeps the
// caller's pointer, normally a literal); interning makes callers whose
// strings are temporaries (e.g. other language bindings) safe too.
static const char *intern_type(const char *t) {
  static const char *known[] = {"double", "float", "int", "uint", "ll", "ull", "bool",
                                "double:soa", "float:soa", "int:soa", "error"};
  static std::vector<std::unique_ptr<std::string>> extra;
  if (!t) return nullptr;
  for (const char *k : known)
    if (strcmp(k, t) == 0) return k;
  for (auto &e : extra)
    if (*e == t) return e->c_str();
  extra.push_back(std::make_unique<std::string>(t));
  return extra.back()->c_str();
}

static op_arg blank_arg() {
  op_arg a;
  memset(&a, 0, sizeof(a));
  a.idx = -1;
  a.opt = 1;
  return a;
}

op_arg op_arg_dat(op_dat dat, int idx, op_map map, int dim, char const *type, op_access acc) {
  op_arg a = blank_arg();
  a.argtype = OP_ARG_DAT;
  a.dat = dat;
  a.map = map;
  a.dim = dim;
  a.idx = idx;
  a.type = intern_type(type);
  a.acc = acc;
  if (dat) {
    a.size = dat->size;
    a.data = dat->data;
    a.data_d = dat->data_d;
  }
  if (map) {
    a.map_data = map->map;
    a.map_data_d = map->map_d;
  }
  return a;
}

op_arg op_opt_arg_dat(int opt, op_dat dat, int idx, op_map map, int dim, char const *type,
                      op_access acc) {
  op_arg a = op_arg_dat(dat, idx, map, dim, type, acc);
  a.opt = opt;
  return a;
}

op_arg op_arg_gbl_char(char *data, int dim, const char *type, int type_size, op_access acc) {
  op_arg a = blank_arg();
  a.argtype = OP_ARG_GBL;
  a.data = data;
  a.dim = dim;
  a.size = dim * type_size;
  a.type = intern_type(type);
  a.acc = acc;
  return a;
}

op_arg op_opt_arg_gbl_char(int opt, char *data, int dim, const char *type, int type_size,
                           op_access acc) {
  op_arg a = op_arg_gbl_char(data, dim, type, type_size, acc);
  a.opt = opt;
  return a;
}

// op_arg_info_char (op_lib_core.cpp:973-1015): payload written at the
// winning element of the MIN/MAX argument `ref`.
op_arg op_arg_info_char(char *data, int dim, const char *type, int type_size, int ref) {
  op_arg a = blank_arg();
  a.argtype = OP_ARG_INFO;
  a.data = data;
  a.dim = dim;
  a.size = dim * type_size;
  a.type = intern_type(type);
  a.acc = ref;  // the reference keeps the referenced argument's position here too
  a.idx = ref;
  return a;
}

op_arg op_arg_idx(int idx, op_map map) {
  op_arg a = blank_arg();
  a.argtype = OP_ARG_IDX;
  a.idx = idx;
  a.map = map;
  a.acc = OP_READ;
  a.type = "int";
  a.size = sizeof(int);
  return a;
}

// ------------------------------------------------------------------ data out

static bool fetch_range(op_dat dat, char *dst, size_t first, size_t count) {
  Runtime &r = rt();
  if (!r.ready()) return false;
  if (!dat || !dat->data_d) {
    if (dat && count == 0) return true;
    set_error("op_fetch_data: invalid dat");
    return false;
  }
  resolve_renumbering_for_fetch(dat);
  size_t bytes = count * (size_t)dat->size;
  return download_host(dst, dat->data_d + first * dat->size, bytes, "op_fetch_data");
}

void op_fetch_data_char(op_dat dat, char *usr_ptr) {
  if (!dat) {
    set_error("op_fetch_data: NULL dat");
    return;
  }
  fetch_range(dat, usr_ptr, 0, (size_t)dat->set->size);
}

// op_fetch_data_idx_char: elements low..high (inclusive) in the order the
// application declared them, i.e. with any renumbering undone.
void op_fetch_data_idx_char(op_dat dat, char *usr_ptr, int low, int high) {
  if (!dat || low < 0 || high >= dat->set->size || low > high + 1) {
    set_error("op_fetch_data_idx: invalid dat or range [%d, %d]", low, high);
    return;
  }
  fetch_original_order(dat, usr_ptr, low, high);
}

static std::vector<char> host_copy(op_dat dat) {
  std::vector<char> buf((size_t)dat->set->size * (size_t)dat->size);
  if (!buf.empty()) fetch_original_order(dat, buf.data(), 0, dat->set->size - 1);
  return buf;
}

// op_print_dat_to_binfile_core (op_lib_core.cpp:1283-1307): int count,
// int dim, then the raw AoS elements.
void op_print_dat_to_binfile(op_dat dat, const char *file_name) {
  if (!dat) return;
  std::vector<char> buf = host_copy(dat);
  FILE *fp = fopen(file_name, "wb");
  if (!fp) {
    set_error("op_print_dat_to_binfile: cannot open %s", file_name);
    return;
  }
  int count = dat->set->size, dim = dat->dim;
  fwrite(&count, sizeof(int), 1, fp);
  fwrite(&dim, sizeof(int), 1, fp);
  if (!buf.empty()) fwrite(buf.data(), 1, buf.size(), fp);
  fclose(fp);
}

// op_print_dat_to_txtfile_core (op_lib_core.cpp:1309-1370): "size dim" then
// one line per element, " %+2.15lE" per double (-0.0 printed as +0.0),
// " %+f" per float, " %+d" per int.
void op_print_dat_to_txtfile(op_dat dat, const char *file_name) {
  if (!dat) return;
  std::vector<char> buf = host_copy(dat);
  FILE *fp = fopen(file_name, "w");
  if (!fp) {
    set_error("op_print_dat_to_txtfile: cannot open %s", file_name);
    return;
  }
  fprintf(fp, "%d %d\n", dat->set->size, dat->dim);
  int tb = type_bytes(dat->type);
  std::string t(dat->type);
  if (t.find(':') != std::string::npos) t = t.substr(0, t.find(':'));
  for (int i = 0; i < dat->set->size; i++) {
    for (int j = 0; j < dat->dim; j++) {
      size_t k = (size_t)i * dat->dim + j;
      if (t == "double" && tb == 8) {
        double v = reinterpret_cast<double *>(buf.data())[k];
        if (v == -0.0) v = +0.0;
        fprintf(fp, " %+2.15lE", v);
      } else if (t == "float") {
        fprintf(fp, " %+f", reinterpret_cast<float *>(buf.data())[k]);
      } else if (t == "int") {
        fprintf(fp, " %+d", reinterpret_cast<int *>(buf.data())[k]);
      } else {
        fclose(fp);
        set_error("op_print_dat_to_txtfile: unknown type %s", dat->type);
        return;
      }
    }
    fprintf(fp, "\n");
  }
  fclose(fp);
}

// ------------------------------------------------------------------ misc

int op_get_size(op_set set) { return set ? set->size : 0; }

void op_printf(const char *format, ...) {
  va_list ap;
  va_start(ap, format);
  vprintf(format, ap);
  va_end(ap);
}

void *op_malloc(size_t size) { return size ? malloc(size) : nullptr; }
void *op_calloc(size_t num, size_t size) { return calloc(num, size); }
void *op_realloc(void *ptr, size_t size) { return realloc(ptr, size); }
void op_free(void *ptr) { free(ptr); }

void op_rank(int *rank) {
  if (rank) *rank = 0;
}

// One rank owns every set: partitioning has nothing to do, as in the
// reference's single-node builds (op2/src/core/op_dummy_singlenode.cpp:
// 144-200).
void op_partition(const char *, const char *, op_set, op_map, op_dat) {}
void op_partition_ptr(const char *, const char *, op_set, int *, double *) {}
void op_partition_reverse(void) {}
void op_partition_destroy(void) {}
int op_is_root(void) { return 1; }

void op_timers(double *cpu, double *et) {
  using namespace std::chrono;
  double t = duration<double>(steady_clock::now().time_since_epoch()).count();
  if (cpu) *cpu = (double)clock() / CLOCKS_PER_SEC;
  if (et) *et = t;
}

void op_diagnostic_output(void) {
  Runtime &r = rt();
  if (r.opt_diags <= 1) return;
  printf("\n  OP diagnostic output\n  --------------------\n\n       set       size\n"
         "  -------------------\n");
  for (auto &s : r.sets)
    if (s) printf("%10s %10d\n", s->name, s->size);
  printf("\n       map        dim       from         to\n  ------------------------------\n");
  for (auto &m : r.maps)
    if (m) printf("%10s %10d %10s %10s\n", m->name, m->dim, m->from->name, m->to->name);
  printf("\n       dat        dim        set\n  ------------------------------\n");
  for (auto &d : r.dats)
    if (d) printf("%10s %10d %10s\n", d->name, d->dim, d->set->name);
  printf("\n");
}

// op_timing_output_core (op_lib_core.cpp:1096-1167): count, plan time, device
// time and GB/s per loop, sorted by time.  Times are CUDA-event device times;
// GB/s uses each loop's algorithmic bytes per call.
void op_timing_output(void) {
  Runtime &r = rt();
  flush_quiet(false);
  r.resolve_timing();
  std::vector<std::pair<std::string, LoopStat>> v(r.stats.begin(), r.stats.end());
  std::sort(v.begin(), v.end(),
            [](auto &a, auto &b) { return a.second.total_ms > b.second.total_ms; });
  printf("\n  count   plan time     device time      GB/s   kernel name\n"
         " -----------------------------------------------------------\n");
  for (auto &kv : v) {
    const LoopStat &s = kv.second;
    const double sampled = s.total_ms * 1e-3;  // over the s.timed sampled calls
    double sec = s.timed > 0 ? sampled * (double)s.calls / (double)s.timed : 0.0;
    double gbs = sampled > 0 ? s.bytes_per_call * (double)s.timed / sampled * 1e-9 : 0.0;
    printf(" %6ld;  %8.4f;  %12.6f;  %8.2f;   %s\n", s.calls, s.plan_ms * 1e-3, sec, gbs,
           kv.first.c_str());
  }
}

// ------------------------------------------------------------------ extensions

int op2b_dat_upload(op_dat dat, const char *src, size_t bytes) {
  Runtime &r = rt();
  if (!r.ready()) return -1;
  if (!dat || !src || bytes != (size_t)dat->set->size * (size_t)dat->size) {
    set_error("op2b_dat_upload: invalid dat or size");
    return -1;
  }
  if (bytes == 0) return 0;
  if (!cuda_ok(cudaMemcpyAsync(dat->data_d, src, bytes, cudaMemcpyHostToDevice, r.stream),
               "op2b_dat_upload"))
    return -1;
  return cuda_ok(cudaStreamSynchronize(r.stream), "op2b_dat_upload") ? 0 : -1;
}

void *op2b_dat_device_ptr(op_dat dat) {
  flush_quiet();
  // the caller may read or write through the pointer at any later time: no
  // speculation on this dat from now on
  if (dat) rt().exposed.insert(dat);
  return dat ? dat->data_d : nullptr;
}
void *op2b_map_device_ptr(op_map map) {
  flush_quiet();
  return map ? map->map_d : nullptr;
}

int op2b_set_option(const char *key, long value) {
  Runtime &r = rt();
  if (r.initialised && r.outstanding() && !r.flush_pending()) return -1;
  if (r.initialised && r.spec.inplace && !r.restore_spec()) return -1;
  std::string k = key ? key : "";
  if (k == "inc_mode") {
    if (value < 0 || value > 3) {
      set_error("op2b_set_option: inc_mode must be 0, 1, 2 or 3");
      return -1;
    }
    r.opt_inc_mode = (int)value;
  } else if (k == "timing") {
    r.opt_timing = value != 0;
  } else if (k == "diags") {
    r.opt_diags = (int)value;
  } else if (k == "abort_on_error") {
    r.opt_abort = value != 0;
  } else if (k == "part_size") {
    r.opt_part_size = (int)value;
  } else if (k == "block_size") {
    r.opt_block_size = (int)value;
  } else if (k == "plan_mode") {
    if (value < 0 || value > 2) {
      set_error("op2b_set_option: plan_mode must be 0, 1 or 2");
      return -1;
    }
    r.opt_plan_mode = (int)value;
  } else if (k == "atomic_segmented") {
    r.opt_atomic_seg = value != 0;
  } else if (k == "jit_warp") {
    r.opt_jit_warp = value != 0;
  } else if (k == "jit_exact") {
    r.opt_jit_exact = value != 0;
  } else if (k == "update_reverse") {
    r.opt_update_rev = value != 0;
  } else if (k == "atomic_blocks") {
    if (value < 1 || value > 4096) {
      set_error("op2b_set_option: atomic_blocks must be between 1 and 4096");
      return -1;
    }
    r.opt_atomic_blocks = (int)value;
  } else if (k == "gemm_tma") {
    r.opt_gemm_tma = value != 0;
  } else if (k == "timing_stride") {
    if (value < 1) {
      set_error("op2b_set_option: timing_stride must be at least 1");
      return -1;
    }
    r.opt_timing_stride = (int)value;
  } else if (k == "pdl") {
    r.opt_pdl = value != 0;
  } else if (k == "gemm_rows") {
    r.opt_gemm_rows = value != 0;
  } else if (k == "host_staging") {
    r.opt_host_staging = value != 0;
  } else if (k == "gemm_persistent") {
    if (value < 0 || value > 2) {
      set_error("op2b_set_option: gemm_persistent must be 0 (a CTA per tile), 1 (persistent, "
                "8 epilogue warps) or 2 (persistent, 16 epilogue warps)");
      return -1;
    }
    r.opt_gemm_ws = (int)value;

  } else if (k == "gather_kernel") {
    if (value < 1 || value > 7) {
      set_error("op2b_set_option: gather_kernel must be 1 (csr), 2 (lanes), 3 (cell4), 4 "
                "(shared-memory pipeline), 5 (register pipeline), 6 (register pipeline "
                "over corner records) or 7 (corner records, each flux computed once)");
      return -1;
    }
    r.opt_gather_kernel = (int)value;
  } else if (k == "pipe_block") {
    if (value != 64 && value != 96 && value != 128 && value != 256) {
      set_error("op2b_set_option: pipe_block must be 64, 96, 128 or 256");
      return -1;
    }
    r.opt_pipe_block = (int)value;
  } else if (k == "pipe_hints") {
    r.opt_pipe_hints = value != 0;
  } else if (k == "gather_minblocks") {
    r.opt_gather_minb = (int)value;
  } else if (k == "bres_kernel") {
    if (value != 0 && value != 1) {
      set_error("op2b_set_option: bres_kernel must be 0 (inverse-map walk) or 1 (records)");
      return -1;
    }
    r.opt_bres_kernel = (int)value;
  } else if (k == "fuse") {
    r.opt_fuse = value != 0;
  } else if (k == "speculate_adt") {
    r.opt_speculate = value != 0;
  } else if (k == "adt_minblocks") {
    if (value < 0 || value > 8) {
      set_error("op2b_set_option: adt_minblocks must be 0..8");
      return -1;
    }
    r.opt_adt_minb = (int)value;
  } else if (k == "check_plans") {
    r.opt_check_plans = value != 0;
  } else if (k == "host_mirror") {
    r.opt_host_mirror = value != 0;
  } else if (k == "rename_save") {
    r.opt_rename_save = value != 0;
  } else if (k == "speculate_res") {
    r.opt_speculate_res = value != 0;
  } else if (k == "lazy_res") {
    r.opt_lazy_res = value != 0;
  } else if (k == "host_threads") {
    if (value < 1 || value > 64) {
      set_error("op2b_set_option: host_threads must be 1..64");
      return -1;
    }
    r.opt_host_threads = (int)value;
  } else {
    set_error("op2b_set_option: unknown option '%s'", k.c_str());
    return -1;
  }
  return 0;
}

long op2b_get_option(const char *key) {
  Runtime &r = rt();
  std::string k = key ? key : "";
  if (k == "inc_mode") return r.opt_inc_mode;
  if (k == "timing") return r.opt_timing;
  if (k == "diags") return r.opt_diags;
  if (k == "abort_on_error") return r.opt_abort;
  if (k == "part_size") return r.opt_part_size;
  if (k == "block_size") return r.opt_block_size;
  if (k == "plan_mode") return r.opt_plan_mode;
  if (k == "atomic_segmented") return r.opt_atomic_seg;
  if (k == "jit_warp") return r.opt_jit_warp;
  if (k == "jit_exact") return r.opt_jit_exact;
  if (k == "update_reverse") return r.opt_update_rev;
  if (k == "atomic_blocks") return r.opt_atomic_blocks;
  if (k == "ring_used") return r.ring_used;  // read-only
  if (k == "gemm_tma") return r.opt_gemm_tma;
  if (k == "gemm_persistent") return r.opt_gemm_ws;
  if (k == "host_staging") return r.opt_host_staging;
  if (k == "gemm_rows") return r.opt_gemm_rows;
  if (k == "pdl") return r.opt_pdl;
  if (k == "timing_stride") return r.opt_timing_stride;
  if (k == "gather_kernel") return r.opt_gather_kernel;
  if (k == "pipe_block") return r.opt_pipe_block;
  if (k == "pipe_hints") return r.opt_pipe_hints;
  if (k == "check_plans") return r.opt_check_plans;
  if (k == "gather_minblocks") return r.opt_gather_minb;
  if (k == "bres_kernel") return r.opt_bres_kernel;
  if (k == "adt_minblocks") return r.opt_adt_minb;
  if (k == "fuse") return r.opt_fuse;
  if (k == "speculate_adt") return r.opt_speculate;
  if (k == "host_mirror") return r.opt_host_mirror;
  if (k == "rename_save") return r.opt_rename_save;
  if (k == "speculate_res") return r.opt_speculate_res;
  if (k == "lazy_res") return r.opt_lazy_res;
  if (k == "host_threads") return r.opt_host_threads;
  if (k == "nsm") return r.nsm;
  return -1;
}

int op2b_loop_stats(const char *name, double *total_ms, long *calls, double *bytes_per_call,
                    double *last_ms) {
  Runtime &r = rt();
  flush_quiet(false);
  r.resolve_timing();
  auto it = r.stats.find(name ? name : "");
  if (it == r.stats.end()) return -1;
  const LoopStat &st = it->second;
  if (total_ms)  // the sampled calls' mean times every call
    *total_ms = st.timed > 0 ? st.total_ms * (double)st.calls / (double)st.timed : 0.0;
  if (calls) *calls = st.calls;
  if (bytes_per_call) *bytes_per_call = it->second.bytes_per_call;
  if (last_ms) *last_ms = it->second.last_ms;
  return 0;
}

void op2b_reset_stats(void) {
  Runtime &r = rt();
  flush_quiet(false);
  r.resolve_timing();
  for (auto &kv : r.stats) {
    double plan = kv.second.plan_ms;
    kv.second = LoopStat();
    kv.second.plan_ms = plan;
  }
}

long op2b_kernel_launches(void) {
  flush_quiet(false);
  return rt().launches;
}

int op2b_set_stream(void *stream) {
  Runtime &r = rt();
  if (!r.ready()) return -1;
  cudaStreamSynchronize(r.stream);
  r.stream = stream ? (cudaStream_t)stream : r.own_stream;
  return 0;
}

void *op2b_get_stream(void) {
  flush_quiet(false);
  return (void *)rt().stream;
}

int op2b_synchronize(void) {
  Runtime &r = rt();
  if (!r.initialised) {
    set_error("op_init has not been called");
    return -1;
  }
  flush_quiet(false);  // waiting observes no dat
  cudaError_t e = cudaStreamSynchronize(r.stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) cuda_ok(e, "op2b_synchronize");
  return (int)e;
}

}  // extern "C"
