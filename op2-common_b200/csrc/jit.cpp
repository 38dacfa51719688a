// Loops without a hand-written kernel: the application's own kernel function,
// compiled for sm_100a at run time (NVRTC) inside a generated loop.
//
// OP2's code generator turns each op_par_loop's user kernel into a device
// loop at build time (translator-v2/resources/templates/cuda/*.jinja); this
// file does the same at run time from the kernel's source text:
//   * the source is the one registered with op2b_register_kernel, or the file
//     <name>.h on OP2B_KERNEL_PATH (default: the working directory) -- the
//     reference's applications keep each kernel in a header of that name
//     (apps/c/jac1/dp/res.h, update.h); preludes (op2b_register_prelude, or
//     user_types.h where it exists) come first; quoted includes are inlined
//     and system includes dropped (NVRTC provides the device math and printf);
//   * constants declared with op_decl_const become __constant__ variables of
//     the same name, type and dimension, refreshed when they change;
//   * the generated kernel runs the user function once per set element
//     (grid-stride): direct dats by pointer, indirect OP_READ through the map,
//     indirect OP_INC into a per-element local added atomically, op_arg_idx
//     as the element's (or its target's) index, op_arg_gbl OP_READ from a
//     device copy, OP_INC/MIN/MAX into per-thread partials reduced by warp
//     shuffles and device atomics, then combined with the caller's value;
//   * a loop with an indirect OP_WRITE or OP_RW argument runs colour by
//     colour over the device-built OP_COLOR2 plan (op_plan_get_stage, the
//     reference's flat element colouring, op_rt_support.cpp:684-754), one
//     launch per colour, so that no two elements of a launch share a target;
//     the colouring covers indirect OP_INC, OP_RW and OP_WRITE arguments;
//   * vector map arguments (idx = -k) get k pointers; switched-off optional
//     arguments a pointer to zeroed scratch; an OP_WORK global a thread's own
//     copy of the caller's values (scratch, not written back);
//   * op_arg_info: the payload the kernel writes where its OP_MIN/OP_MAX
//     global improves, kept per thread with the element of the improvement;
//     the best value over the loop wins, the lowest element on ties (the
//     reference's CUDA reductions take the argmin/argmax with CUB); not in a
//     loop that runs colour by colour;
//   * compiled with --fmad=false (each operation rounded once, like the
//     reference's strictly compiled sequential build); modules are cached per
//     loop signature and source until op_exit.
// Summation order of OP_INC increments and gbl reductions is that of the
// atomics, so results equal the sequential reference's to rounding, not bit
// for bit (the hand-written Airfoil loops keep the reference's order).  In a
// coloured loop the indirect increments of one launch reach distinct
// targets, so they are deterministic; only the gbl reductions are not.
#include <cuda_runtime.h>
#include <nvrtc.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "gather.h"
#include "op2b_plan.h"
#include "op2b_runtime.h"
#include "plan.h"

namespace op2b {
namespace {

struct Sources {
  std::map<std::string, std::string> kernels;
  std::vector<std::string> preludes;
};
Sources &sources() {
  static Sources s;
  return s;
}

bool read_file(const std::string &path, std::string &out) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  std::ostringstream ss;
  ss << f.rdbuf();
  out = ss.str();
  return true;
}

std::vector<std::string> search_path() {
  std::vector<std::string> dirs;
  const char *p = getenv("OP2B_KERNEL_PATH");
  std::string s = p ? p : ".";
  size_t b = 0;
  while (b <= s.size()) {
    size_t e = s.find(':', b);
    if (e == std::string::npos) e = s.size();
    if (e > b) dirs.push_back(s.substr(b, e - b));
    b = e + 1;
  }
  return dirs;
}

// a registered source or a file on the search path
bool find_file(const std::string &name, std::string &out) {
  auto it = sources().kernels.find(name);
  if (it != sources().kernels.end()) {
    out = it->second;
    return true;
  }
  for (const std::string &d : search_path())
    if (read_file(d + "/" + name, out)) return true;
  return false;
}

// inline quoted includes (once each), drop system includes
std::string expand(const std::string &src, std::vector<std::string> &seen, int depth) {
  std::istringstream in(src);
  std::ostringstream out;
  std::string line;
  while (std::getline(in, line)) {
    size_t p = line.find_first_not_of(" \t");
    if (p != std::string::npos && line.compare(p, 8, "#include") == 0) {
      size_t q1 = line.find('"', p), q2 = q1 == std::string::npos ? q1 : line.find('"', q1 + 1);
      if (q1 != std::string::npos && q2 != std::string::npos && depth < 8) {
        std::string inc = line.substr(q1 + 1, q2 - q1 - 1), text;
        bool done = false;
        for (auto &s : seen) done |= s == inc;
        if (!done && find_file(inc, text)) {
          seen.push_back(inc);
          out << expand(text, seen, depth + 1) << "\n";
        }
      }
      out << "\n";  // keep line numbers close for compiler messages
      continue;
    }
    out << line << "\n";
  }
  return out.str();
}

// OFF: an optional argument switched off (op_opt_arg_dat / op_opt_arg_gbl
// with opt = 0): the kernel gets a pointer to zeroed scratch it must not use.
// INFO: op_arg_info, the payload the kernel writes where its MIN/MAX global
// (argument `idx`) improves; kept per thread with the element index of the
// improvement, and the lowest index among equal best values wins.
enum ArgKind { DIRECT, INDIRECT, GBL, IDX, OFF, INFO };

struct ArgPlan {
  ArgKind kind;
  std::string ctype;
  int dim = 1, acc = OP_READ, mdim = 0, idx = -1, bytes = 8;
  int vec = 0;  // vector map argument (idx = -vec): the kernel gets vec pointers
  // stage 1: a direct dat moved through the warp's shared memory in whole
  // rows (coalesced), the kernel working on registers; stage 2: an indirect
  // OP_READ gathered by `vw`-element vector loads into registers
  int stage = 0, vw = 0;
  bool seg = false;  // indirect OP_INC combined per warp before the atomics
};

std::string base_type(const char *t) {
  std::string s = t ? t : "";
  size_t c = s.find(':');
  if (c != std::string::npos) s = s.substr(0, c);
  return s;
}

int type_size(const std::string &t) {
  if (t == "double") return 8;
  if (t == "float" || t == "int") return 4;
  return 0;
}

struct Jit {
  cudaLibrary_t lib = nullptr;
  cudaKernel_t fn = nullptr;
  std::vector<std::string> cnames, clowered;
  long const_version = -1;
  void *gbl_d = nullptr;
  size_t gbl_cap = 0;
};

std::map<std::string, Jit> &cache() {
  static std::map<std::string, Jit> c;
  return c;
}

std::string identity(const std::string &t, int acc) {
  if (acc == OP_INC) return "0";
  const bool mn = acc == OP_MIN;
  if (t == "double") return mn ? "__longlong_as_double(0x7ff0000000000000LL)"
                               : "__longlong_as_double((long long)0xfff0000000000000ULL)";
  if (t == "float") return mn ? "__int_as_float(0x7f800000)" : "__int_as_float((int)0xff800000u)";
  return mn ? "2147483647" : "(-2147483647 - 1)";
}

// NVRTC has no C++ standard library: the std:: names kernels written for a
// host compiler use (std::min in apps/c/min/min_direct.cpp:9-11, the math
// functions), mapped onto the device's own.
const char *kStd = R"(
namespace std {
template <typename T> __device__ const T &min(const T &a, const T &b) { return b < a ? b : a; }
template <typename T> __device__ const T &max(const T &a, const T &b) { return a < b ? b : a; }
using ::abs; using ::fabs; using ::sqrt; using ::cbrt; using ::pow; using ::exp; using ::log;
using ::log10; using ::sin; using ::cos; using ::tan; using ::atan; using ::atan2; using ::tanh;
using ::floor; using ::ceil; using ::fmin; using ::fmax; using ::hypot;
}
)";

const char *kHelpers = R"(
// a vector map argument's pointer array, passed to a kernel parameter
// declared T ** or const T ** (op_seq.h hands the kernel a T ** it typed
// from the kernel's own signature)
template <typename T> struct op2b_vec {
  T **p;
  __device__ operator T **() const { return p; }
  __device__ operator const T **() const { return (const T **)p; }
  __device__ operator const T *const *() const { return p; }
};
__device__ void op2b_amin(double *a, double v) {
  unsigned long long *p = (unsigned long long *)a, old = *p, as;
  do { as = old; if (__longlong_as_double((long long)as) <= v) return;
       old = atomicCAS(p, as, (unsigned long long)__double_as_longlong(v)); } while (old != as);
}
__device__ void op2b_amax(double *a, double v) {
  unsigned long long *p = (unsigned long long *)a, old = *p, as;
  do { as = old; if (__longlong_as_double((long long)as) >= v) return;
       old = atomicCAS(p, as, (unsigned long long)__double_as_longlong(v)); } while (old != as);
}
__device__ void op2b_amin(float *a, float v) {
  int *p = (int *)a, old = *p, as;
  do { as = old; if (__int_as_float(as) <= v) return;
       old = atomicCAS(p, as, __float_as_int(v)); } while (old != as);
}
__device__ void op2b_amax(float *a, float v) {
  int *p = (int *)a, old = *p, as;
  do { as = old; if (__int_as_float(as) >= v) return;
       old = atomicCAS(p, as, __float_as_int(v)); } while (old != as);
}
__device__ void op2b_amin(int *a, int v) { atomicMin(a, v); }
__device__ void op2b_amax(int *a, int v) { atomicMax(a, v); }
template <typename T> __device__ T op2b_min(T a, T b) { return b < a ? b : a; }
template <typename T> __device__ T op2b_max(T a, T b) { return b > a ? b : a; }
)";

// own >= 0: the owner-computes loop (option jit_exact) for the increments of
// argument own's dat; the others of its increment arguments share its map
std::string generate(const char *name, const std::vector<ArgPlan> &ap, const std::string &body,
                     bool coloured, int own = -1) {
  Runtime &r = rt();
  std::ostringstream s;
  s << "// libop2b: generated loop for the user kernel '" << name << "'\n";
  for (auto &kv : r.consts) {
    const std::string &t = r.const_types[kv.first];
    s << "__constant__ " << (t.empty() ? "double" : t) << " " << kv.first;
    if (kv.second.size() > 1) s << "[" << kv.second.size() << "]";
    s << ";\n";
  }
  // the min/max macros kernels find in OP2's headers (op_lib_core.h:246-249)
  s << "#ifndef MIN\n#define MIN(a, b) ((a < b) ? (a) : (b))\n#endif\n"
       "#ifndef MAX\n#define MAX(a, b) ((a > b) ? (a) : (b))\n#endif\n";
  s << kStd << "\n";
  s << kHelpers << "\n" << body << "\n";
  s << "extern \"C\" __global__ void op2b_loop(int op2b_n";
  for (size_t i = 0; i < ap.size(); i++) {
    const ArgPlan &a = ap[i];
    if (a.kind == DIRECT || a.kind == INDIRECT || a.kind == GBL || a.kind == OFF)
      s << ", " << a.ctype << " *op2b_d" << i;
    if (a.kind == INDIRECT || (a.kind == IDX && a.mdim > 0)) s << ", const int *op2b_m" << i;
    if (a.kind == INFO)  // per block: best value, its element, its payload; the caller's payload
      s << ", double *op2b_iv" << i << ", long long *op2b_ix" << i << ", " << a.ctype
        << " *op2b_ip" << i << ", const " << a.ctype << " *op2b_ic" << i;
  }
  // coloured: this launch runs the elements op2b_perm[op2b_first, +op2b_n)
  if (coloured) s << ", const int *op2b_perm, int op2b_first";
  // owner computes: op2b_n targets, each with its (element, slot) entries
  if (own >= 0) s << ", const long long *op2b_ioff, const int *op2b_ient, const int *op2b_rows";
  s << ") {\n";
  for (size_t i = 0; i < ap.size(); i++) {
    const ArgPlan &a = ap[i];
    if (a.kind == INFO) {
      const ArgPlan &g = ap[(size_t)a.idx];
      // each thread's payload starts as the caller's (as the sequential
      // build's info temp is a copy of the caller's data)
      s << "  " << a.ctype << " op2b_l" << i << "[" << a.dim << "];\n  for (int k = 0; k < "
        << a.dim << "; k++) op2b_l" << i << "[k] = op2b_ic" << i << "[k];\n  long long op2b_e" << i
        << " = 0x7fffffffffffffffLL;\n  " << g.ctype << " op2b_pv" << i << " = "
        << identity(g.ctype, g.acc) << ";\n";
    }
  }
  for (size_t i = 0; i < ap.size(); i++) {
    const ArgPlan &a = ap[i];
    if (a.kind == GBL && a.acc == OP_WORK)  // a thread's own scratch, reloaded every element
      s << "  " << a.ctype << " op2b_l" << i << "[" << a.dim << "];\n";
    else if (a.kind == GBL && a.acc != OP_READ)
      s << "  " << a.ctype << " op2b_l" << i << "[" << a.dim << "];\n  for (int k = 0; k < "
        << a.dim << "; k++) op2b_l" << i << "[k] = " << identity(a.ctype, a.acc) << ";\n";
  }
  // warp mode: the loop advances a warp at a time (32 consecutive elements,
  // every lane reaching each warp-wide step) when a direct dat is staged
  // through shared memory or an increment is combined per warp
  bool warp = false;
  size_t wbytes = 0;  // shared memory a lane needs: the widest staged row (+ padding)
  for (const ArgPlan &a : ap) {
    if (a.stage == 1) wbytes = std::max(wbytes, (size_t)(a.dim + 1) * a.bytes);
    if (a.seg) wbytes = std::max(wbytes, (size_t)a.dim * a.bytes);
    warp |= a.stage == 1 || a.seg;
  }
  wbytes = (wbytes + 15) & ~(size_t)15;
  if (own >= 0) {
    // a thread per target: the elements that increment it, in element order
    // (each slot in slot order), the kernel adding straight into the target's
    // own sum -- the additions of the sequential loop, in its order
    const ArgPlan &o = ap[(size_t)own];
    // (op2b_rows, when given, lists the targets that have entries)
    s << "  for (int op2b_i = blockIdx.x * blockDim.x + threadIdx.x; op2b_i < op2b_n;"
         " op2b_i += gridDim.x * blockDim.x) {\n"
      << "  const int op2b_t = op2b_rows ? op2b_rows[op2b_i] : op2b_i;\n"
      << "  " << o.ctype << " op2b_acc[" << o.dim << "];\n"
      << "  for (int k = 0; k < " << o.dim << "; k++) op2b_acc[k] = op2b_d" << own
      << "[(size_t)op2b_t * " << o.dim << " + k];\n"
      << "  for (long long op2b_k = op2b_ioff[op2b_t]; op2b_k < op2b_ioff[op2b_t + 1]; op2b_k++) {\n"
      << "    const int op2b_e = op2b_ient[op2b_k] / " << o.mdim << ";\n"
      << "    const int op2b_s = op2b_ient[op2b_k] % " << o.mdim << ";\n";
  } else if (warp) {
    s << "  __shared__ __align__(16) unsigned char op2b_sh[" << 256 * wbytes << "];\n"
      << "  const int op2b_lane = threadIdx.x & 31;\n"
      << "  unsigned char *op2b_w = op2b_sh + (threadIdx.x >> 5) * " << 32 * wbytes << ";\n"
      << "  for (int op2b_b = blockIdx.x * blockDim.x + (threadIdx.x & ~31); op2b_b < op2b_n;"
         " op2b_b += gridDim.x * blockDim.x) {\n"
      // the element (loads of lanes past the end repeat the last element's;
      // only lanes with op2b_ok call the kernel and store)
      << "    const bool op2b_ok = op2b_b + op2b_lane < op2b_n;\n"
      << "    const int op2b_e = op2b_ok ? op2b_b + op2b_lane : op2b_n - 1;\n"
      << "    const int op2b_cnt = op2b_n - op2b_b < 32 ? op2b_n - op2b_b : 32;\n";
    for (size_t i = 0; i < ap.size(); i++) {
      const ArgPlan &a = ap[i];
      if (a.stage == 1) {
        // the warp's rows as whole words, all loads issued before any is used
        s << "    " << a.ctype << " op2b_y" << i << "[" << a.dim << "];\n#pragma unroll\n"
          << "    for (int k = 0; k < " << a.dim << "; k++) {\n      const int w = k * 32 + op2b_lane;\n"
          << "      op2b_y" << i << "[k] = w < op2b_cnt * " << a.dim << " ? op2b_d" << i
          << "[(size_t)op2b_b * " << a.dim << " + w] : (" << a.ctype << ")0;\n    }\n";
      }
      if (a.seg) {
        const int nv = std::max(a.vec, 1);
        s << "    " << a.ctype << " op2b_l" << i << "[" << nv * a.dim << "];\n    for (int k = 0; k < "
          << nv * a.dim << "; k++) op2b_l" << i << "[k] = 0;\n    int op2b_t" << i << "[" << nv
          << "];\n";
      }
    }
  } else if (coloured) {
    s << "  for (int op2b_i = blockIdx.x * blockDim.x + threadIdx.x; op2b_i < op2b_n;"
         " op2b_i += gridDim.x * blockDim.x) {\n"
         "    const int op2b_e = op2b_perm[op2b_first + op2b_i];\n";
  } else {
    s << "  for (int op2b_e = blockIdx.x * blockDim.x + threadIdx.x; op2b_e < op2b_n;"
         " op2b_e += gridDim.x * blockDim.x) {\n";
  }
  // OP_WORK: every element starts from the caller's values
  for (size_t i = 0; i < ap.size(); i++)
    if (ap[i].kind == GBL && ap[i].acc == OP_WORK)
      s << "    for (int k = 0; k < " << ap[i].dim << "; k++) op2b_l" << i << "[k] = op2b_d" << i
        << "[k];\n";
  // op_arg_info: a copy of the payload before the call, to see whether the
  // kernel wrote it (a write on a tie changes the payload, not the value)
  for (size_t i = 0; i < ap.size(); i++)
    if (ap[i].kind == INFO)
      s << "    " << ap[i].ctype << " op2b_s" << i << "[" << ap[i].dim << "];\n    for (int k = 0; k < "
        << ap[i].dim << "; k++) op2b_s" << i << "[k] = op2b_l" << i << "[k];\n";
  static const char *comp[4] = {".x", ".y", ".z", ".w"};
  std::ostringstream call;
  call << "    " << name << "(";
  for (size_t i = 0; i < ap.size(); i++) {
    const ArgPlan &a = ap[i];
    if (i) call << ", ";
    switch (a.kind) {
      case DIRECT:
        if (a.stage == 1)
          call << "op2b_r" << i;
        else
          call << "op2b_d" << i << " + (size_t)op2b_e * " << a.dim;
        break;
      case OFF:
        if (a.vec) {
          s << "    " << a.ctype << " *op2b_v" << i << "[" << a.vec << "];\n    for (int j = 0; j < "
            << a.vec << "; j++) op2b_v" << i << "[j] = op2b_d" << i << ";\n";
          call << "op2b_vec<" << a.ctype << ">{op2b_v" << i << "}";
        } else {
          call << "op2b_d" << i;
        }
        break;
      case INDIRECT:
        if (own >= 0 && a.acc == OP_INC) {
          // the owner's slot adds into its sum, the element's other slots
          // into scratch
          const int nv = std::max(a.vec, 1);
          s << "    " << a.ctype << " op2b_l" << i << "[" << nv * a.dim << "];\n"
            << "    for (int k = 0; k < " << nv * a.dim << "; k++) op2b_l" << i << "[k] = 0;\n";
          if (a.vec) {
            s << "    " << a.ctype << " *op2b_v" << i << "[" << a.vec << "];\n    for (int j = 0; j < "
              << a.vec << "; j++) op2b_v" << i << "[j] = op2b_s == j ? op2b_acc : op2b_l" << i
              << " + j * " << a.dim << ";\n";
            call << "op2b_vec<" << a.ctype << ">{op2b_v" << i << "}";
          } else {
            call << "(op2b_s == " << a.idx << " ? op2b_acc : op2b_l" << i << ")";
          }
          break;
        }
        if (a.vec) {
          // one pointer per map entry (op_seq.h op_arg_copy_in); increments
          // into locals added atomically after the call
          s << "    " << a.ctype << " *op2b_v" << i << "[" << a.vec << "];\n";
          if (a.acc == OP_INC && !a.seg)
            s << "    " << a.ctype << " op2b_l" << i << "[" << a.vec * a.dim << "];\n"
              << "    for (int k = 0; k < " << a.vec * a.dim << "; k++) op2b_l" << i << "[k] = 0;\n";
          if (a.seg)
            s << "    for (int j = 0; j < " << a.vec << "; j++) op2b_t" << i << "[j] = op2b_ok ? op2b_m"
              << i << "[(size_t)op2b_e * " << a.mdim << " + j] : -1 - op2b_lane;\n";
          s << "    for (int j = 0; j < " << a.vec << "; j++) op2b_v" << i << "[j] = ";
          if (a.acc == OP_INC)
            s << "op2b_l" << i << " + j * " << a.dim << ";\n";
          else
            s << "op2b_d" << i << " + (size_t)op2b_m" << i << "[(size_t)op2b_e * " << a.mdim
              << " + j] * " << a.dim << ";\n";
          call << "op2b_vec<" << a.ctype << ">{op2b_v" << i << "}";
          break;
        }
        if (a.seg) {
          s << "    op2b_t" << i << "[0] = op2b_ok ? op2b_m" << i << "[(size_t)op2b_e * " << a.mdim
            << " + " << a.idx << "] : -1 - op2b_lane;\n";
          call << "op2b_l" << i;
          break;
        }
        s << "    const int op2b_t" << i << " = op2b_m" << i << "[(size_t)op2b_e * " << a.mdim
          << " + " << a.idx << "];\n";
        if (a.acc == OP_INC) {
          s << "    " << a.ctype << " op2b_l" << i << "[" << a.dim << "];\n    for (int k = 0; k < "
            << a.dim << "; k++) op2b_l" << i << "[k] = 0;\n";
          call << "op2b_l" << i;
        } else if (a.stage == 2) {
          // the row by vector loads into registers
          const std::string vt = (a.ctype == "double" ? "double" : a.ctype) + std::to_string(a.vw);
          s << "    " << a.ctype << " op2b_r" << i << "[" << a.dim << "];\n    {\n      const " << vt
            << " *op2b_p = (const " << vt << " *)(op2b_d" << i << " + (size_t)op2b_t" << i
            << " * " << a.dim << ");\n";
          for (int v = 0; v < a.dim / a.vw; v++) {
            s << "      { const " << vt << " op2b_x = op2b_p[" << v << "];";
            for (int c = 0; c < a.vw; c++)
              s << " op2b_r" << i << "[" << v * a.vw + c << "] = op2b_x" << comp[c] << ";";
            s << " }\n";
          }
          s << "    }\n";
          call << "op2b_r" << i;
        } else {
          call << "op2b_d" << i << " + (size_t)op2b_t" << i << " * " << a.dim;
        }
        break;
      case GBL:
        if (a.acc == OP_READ) call << "op2b_d" << i;
        else call << "op2b_l" << i;
        break;
      case INFO:
        call << "op2b_l" << i;
        break;
      case IDX:
        if (a.mdim > 0)
          s << "    int op2b_x" << i << " = op2b_m" << i << "[(size_t)op2b_e * " << a.mdim
            << " + " << a.idx << "];\n";
        else
          s << "    int op2b_x" << i << " = op2b_e;\n";
        call << "&op2b_x" << i;
        break;
    }
  }
  call << ");\n";
  if (warp) {
    // staged rows from the loaded words through the warp's shared memory
    // (rows padded by one element against bank conflicts) into registers
    for (size_t i = 0; i < ap.size(); i++) {
      const ArgPlan &a = ap[i];
      if (a.stage != 1) continue;
      const int P = a.dim + 1;
      s << "    " << a.ctype << " op2b_r" << i << "[" << a.dim << "];\n    {\n      " << a.ctype
        << " *op2b_q = (" << a.ctype << " *)op2b_w;\n#pragma unroll\n"
        << "      for (int k = 0; k < " << a.dim << "; k++) {\n        const int w = k * 32 + op2b_lane;\n"
        << "        op2b_q[(w / " << a.dim << ") * " << P << " + w % " << a.dim << "] = op2b_y" << i
        << "[k];\n      }\n      __syncwarp();\n#pragma unroll\n"
        << "      for (int k = 0; k < " << a.dim << "; k++) op2b_r" << i << "[k] = op2b_q[op2b_lane * "
        << P << " + k];\n      __syncwarp();\n    }\n";
    }
    s << "    if (op2b_ok) {\n";
  }
  s << call.str();
  // the thread's candidate: its best value, and the element whose call last
  // wrote the payload (an improvement, or a write on a tie)
  for (size_t i = 0; i < ap.size(); i++)
    if (ap[i].kind == INFO) {
      s << "    {\n      bool w = op2b_l" << ap[i].idx << "[0] != op2b_pv" << i << ";\n"
        << "      for (int k = 0; k < " << ap[i].dim << "; k++) w |= op2b_s" << i
        << "[k] != op2b_l" << i << "[k];\n"
        << "      if (w) { op2b_pv" << i << " = op2b_l" << ap[i].idx << "[0]; op2b_e" << i
        << " = op2b_e; }\n    }\n";
    }
  for (size_t i = 0; i < ap.size(); i++) {
    const ArgPlan &a = ap[i];
    if (a.seg || own >= 0) continue;
    if (a.kind == INDIRECT && a.acc == OP_INC && a.vec)
      s << "    for (int j = 0; j < " << a.vec << "; j++) {\n      const size_t t = (size_t)op2b_m"
        << i << "[(size_t)op2b_e * " << a.mdim << " + j] * " << a.dim << ";\n"
        << "      for (int k = 0; k < " << a.dim << "; k++) atomicAdd(op2b_d" << i
        << " + t + k, op2b_l" << i << "[j * " << a.dim << " + k]);\n    }\n";
    else if (a.kind == INDIRECT && a.acc == OP_INC)
      s << "    for (int k = 0; k < " << a.dim << "; k++) atomicAdd(op2b_d" << i
        << " + (size_t)op2b_t" << i << " * " << a.dim << " + k, op2b_l" << i << "[k]);\n";
  }
  if (own >= 0) {
    const ArgPlan &o = ap[(size_t)own];
    s << "  }\n  for (int k = 0; k < " << o.dim << "; k++) op2b_d" << own << "[(size_t)op2b_t * "
      << o.dim << " + k] = op2b_acc[k];\n";
  }
  if (warp) {
    s << "    }\n";  // if (op2b_ok)
    for (size_t i = 0; i < ap.size(); i++) {
      const ArgPlan &a = ap[i];
      if (a.stage != 1 || a.acc == OP_READ) continue;
      // written rows back through shared memory, whole rows per store
      const int P = a.dim + 1;
      s << "    {\n      " << a.ctype << " *op2b_q = (" << a.ctype << " *)op2b_w;\n"
        << "      for (int k = 0; k < " << a.dim << "; k++) op2b_q[op2b_lane * " << P
        << " + k] = op2b_r" << i << "[k];\n      __syncwarp();\n#pragma unroll\n"
        << "      for (int k = 0; k < " << a.dim << "; k++) {\n        const int w = k * 32 + op2b_lane;\n"
        << "        if (w < op2b_cnt * " << a.dim << ") op2b_d" << i << "[(size_t)op2b_b * " << a.dim
        << " + w] = op2b_q[(w / " << a.dim << ") * " << P << " + w % " << a.dim << "];\n      }\n"
        << "      __syncwarp();\n    }\n";
    }
    for (size_t i = 0; i < ap.size(); i++) {
      const ArgPlan &a = ap[i];
      if (!a.seg) continue;
      // lanes with the same target combine their increments (lowest lane
      // sums them in lane order) and that lane adds the sum atomically
      s << "    for (int j = 0; j < " << std::max(a.vec, 1) << "; j++) {\n      " << a.ctype
        << " *op2b_q = (" << a.ctype << " *)op2b_w;\n      const int op2b_k = op2b_t" << i
        << "[j];\n      for (int k = 0; k < " << a.dim << "; k++) op2b_q[k * 32 + op2b_lane] = op2b_l"
        << i << "[j * " << a.dim << " + k];\n      __syncwarp();\n"
        << "      const unsigned op2b_g = __match_any_sync(0xffffffffu, op2b_k);\n"
        << "      if (op2b_k >= 0 && op2b_lane == __ffs(op2b_g) - 1)\n"
        << "        for (int k = 0; k < " << a.dim << "; k++) {\n          " << a.ctype
        << " op2b_a = op2b_q[k * 32 + op2b_lane];\n"
        << "          for (unsigned op2b_m = op2b_g & (op2b_g - 1); op2b_m; op2b_m &= op2b_m - 1)\n"
        << "            op2b_a += op2b_q[k * 32 + __ffs(op2b_m) - 1];\n"
        << "          atomicAdd(op2b_d" << i << " + (size_t)op2b_k * " << a.dim << " + k, op2b_a);\n"
        << "        }\n      __syncwarp();\n    }\n";
    }
  }
  s << "  }\n";
  for (size_t i = 0; i < ap.size(); i++) {
    const ArgPlan &a = ap[i];
    if (a.kind != INFO) continue;
    const bool mx = ap[(size_t)a.idx].acc == OP_MAX;
    // the block's best: thread 0 walks the block's candidates in order
    s << "  {\n    __shared__ double sv[256];\n    __shared__ long long se[256];\n"
      << "    __shared__ " << a.ctype << " sp[256 * " << a.dim << "];\n"
      << "    sv[threadIdx.x] = (double)op2b_pv" << i << ";\n    se[threadIdx.x] = op2b_e" << i
      << ";\n    for (int k = 0; k < " << a.dim << "; k++) sp[threadIdx.x * " << a.dim
      << " + k] = op2b_l" << i << "[k];\n    __syncthreads();\n"
      << "    if (threadIdx.x == 0) {\n      int b = -1;\n"
      << "      for (int t = 0; t < (int)blockDim.x; t++) {\n"
      << "        if (se[t] == 0x7fffffffffffffffLL) continue;\n"
      << "        if (b < 0 || sv[t] " << (mx ? ">" : "<") << " sv[b] || (sv[t] == sv[b] && se[t] < se[b])) b = t;\n"
      << "      }\n      op2b_ix" << i << "[blockIdx.x] = b < 0 ? 0x7fffffffffffffffLL : se[b];\n"
      << "      if (b >= 0) {\n        op2b_iv" << i << "[blockIdx.x] = sv[b];\n"
      << "        for (int k = 0; k < " << a.dim << "; k++) op2b_ip" << i << "[blockIdx.x * "
      << a.dim << " + k] = sp[b * " << a.dim << " + k];\n      }\n    }\n  }\n";
  }
  for (size_t i = 0; i < ap.size(); i++) {
    const ArgPlan &a = ap[i];
    if (a.kind != GBL || a.acc == OP_READ || a.acc == OP_WORK) continue;
    const char *op = a.acc == OP_INC ? "v + w" : a.acc == OP_MIN ? "op2b_min(v, w)" : "op2b_max(v, w)";
    s << "  for (int k = 0; k < " << a.dim << "; k++) {\n    " << a.ctype << " v = op2b_l" << i
      << "[k];\n    for (int o = 16; o > 0; o >>= 1) { " << a.ctype
      << " w = __shfl_down_sync(0xffffffffu, v, o); v = " << op << "; }\n"
      << "    if ((threadIdx.x & 31) == 0) ";
    if (a.acc == OP_INC) s << "atomicAdd(op2b_d" << i << " + k, v);\n";
    else s << (a.acc == OP_MIN ? "op2b_amin" : "op2b_amax") << "(op2b_d" << i << " + k, v);\n";
    s << "  }\n";
  }
  s << "}\n";
  return s.str();
}

bool compile(const char *name, const std::string &src, Jit &j) {
  Runtime &r = rt();
  nvrtcProgram prog;
  if (nvrtcCreateProgram(&prog, src.c_str(), (std::string(name) + "_op2b.cu").c_str(), 0,
                         nullptr, nullptr) != NVRTC_SUCCESS) {
    set_error("op_par_loop(%s): NVRTC could not create the program", name);
    return false;
  }
  for (auto &kv : r.consts) {
    j.cnames.push_back(kv.first);
    nvrtcAddNameExpression(prog, ("&" + kv.first).c_str());
  }
  const char *opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "-default-device",
                        "--fmad=false"};
  nvrtcResult rc = nvrtcCompileProgram(prog, 4, opts);
  if (rc != NVRTC_SUCCESS) {
    size_t n = 0;
    nvrtcGetProgramLogSize(prog, &n);
    std::string log(n, '\0');
    if (n) nvrtcGetProgramLog(prog, &log[0]);
    set_error("op_par_loop(%s): compiling the kernel failed:\n%s", name, log.c_str());
    nvrtcDestroyProgram(&prog);
    return false;
  }
  for (auto &c : j.cnames) {
    const char *low = nullptr;
    nvrtcGetLoweredName(prog, ("&" + c).c_str(), &low);
    j.clowered.push_back(low ? low : c);
  }
  size_t cubin_size = 0;
  nvrtcGetCUBINSize(prog, &cubin_size);
  std::vector<char> cubin(cubin_size);
  nvrtcGetCUBIN(prog, cubin.data());
  nvrtcDestroyProgram(&prog);
  if (!cuda_ok(cudaLibraryLoadData(&j.lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr,
                                   0),
               "op_par_loop: loading the compiled kernel"))
    return false;
  return cuda_ok(cudaLibraryGetKernel(&j.fn, j.lib, "op2b_loop"), "op_par_loop: kernel entry");
}

bool upload_constants(Jit &j) {
  Runtime &r = rt();
  if (j.const_version == r.const_version) return true;
  if (!cuda_ok(cudaStreamSynchronize(r.stream), "op_par_loop: constants")) return false;
  for (size_t i = 0; i < j.cnames.size(); i++) {
    auto it = r.consts.find(j.cnames[i]);
    if (it == r.consts.end()) continue;
    void *p = nullptr;
    size_t bytes = 0;
    if (!cuda_ok(cudaLibraryGetGlobal(&p, &bytes, j.lib, j.clowered[i].c_str()),
                 "op_par_loop: constant lookup"))
      return false;
    const std::string &t = r.const_types[j.cnames[i]];
    std::vector<char> buf(bytes, 0);
    for (size_t k = 0; k < it->second.size(); k++) {
      if (t == "float" && (k + 1) * 4 <= bytes) {
        float v = (float)it->second[k];
        memcpy(&buf[k * 4], &v, 4);
      } else if (t == "int" && (k + 1) * 4 <= bytes) {
        int v = (int)it->second[k];
        memcpy(&buf[k * 4], &v, 4);
      } else if ((k + 1) * 8 <= bytes) {
        memcpy(&buf[k * 8], &it->second[k], 8);
      }
    }
    if (!cuda_ok(cudaMemcpyAsync(p, buf.data(), bytes, cudaMemcpyHostToDevice, r.stream),
                 "op_par_loop: constant upload") ||
        !cuda_ok(cudaStreamSynchronize(r.stream), "op_par_loop: constant upload"))
      return false;
  }
  j.const_version = r.const_version;
  return true;
}

}  // namespace

bool jit_has_kernel(const char *name) {
  std::string src;
  return name && find_file(std::string(name) + ".h", src);
}

void release_jit() {
  for (auto &kv : cache()) {
    if (kv.second.lib) cudaLibraryUnload(kv.second.lib);
    cudaFree(kv.second.gbl_d);
  }
  cache().clear();
}

// The OP_COLOR2 plan of a loop with indirect OP_WRITE/OP_RW arguments: every
// indirect dat is one indirection (the reference's generated stubs number
// them the same way), and OP_WRITE is planned as OP_RW so that the colouring,
// which the reference restricts to OP_INC and OP_RW (op_rt_support.cpp:
// 716-739), keeps writers of one target apart as well.
const Plan *colour_plan(const char *name, op_set set, int nargs, const op_arg *args) {
  // the plan sees one argument per map entry a vector argument reaches, and
  // none for a switched-off one
  std::vector<op_arg> pa;
  std::vector<int> inds;
  std::vector<op_dat> seen;
  for (int i = 0; i < nargs; i++) {
    op_arg x = args[i];
    if (x.argtype == OP_ARG_DAT && !x.opt) continue;
    if (x.argtype != OP_ARG_DAT || x.map == nullptr) {
      pa.push_back(x);
      inds.push_back(-1);
      continue;
    }
    if (x.acc == OP_WRITE) x.acc = OP_RW;
    auto it = std::find(seen.begin(), seen.end(), x.dat);
    const int ind = (int)(it - seen.begin());
    if (it == seen.end()) seen.push_back(x.dat);
    const int k = x.idx < -1 ? -x.idx : 1;
    for (int j = 0; j < k; j++) {
      if (k > 1) x.idx = j;
      pa.push_back(x);
      inds.push_back(ind);
    }
  }
  // colours by parallel rounds (no reference integers to match here) unless
  // plan_mode 2 asks for the serial greedy walk
  const std::string pname = std::string(name) + "#coloured";
  Plan *bp = build_plan(pname.c_str(), set, 0, (int)pa.size(), pa.data(), (int)seen.size(),
                        inds.data(), OP_COLOR2,
                        rt().opt_plan_mode == 2 ? OP2B_COLOUR_GREEDY : OP2B_COLOUR_JP);
  op_plan *o = bp ? &bp->pub : nullptr;
  const Plan *pl = o ? find_plan(o) : nullptr;
  if (!pl || !pl->col_reord_d || !o->color2_offsets) {
    if (op2b_last_error()[0] == 0) set_error("op_par_loop(%s): colouring the loop failed", name);
    return nullptr;
  }
  return pl;
}

int jit_par_loop(const char *name, op_set set, int nargs, op_arg *args) {
  Runtime &r = rt();
  std::vector<ArgPlan> ap((size_t)nargs);
  bool coloured = false;
  std::ostringstream key;
  key << name;
  for (int i = 0; i < nargs; i++) {
    const op_arg &x = args[i];
    ArgPlan &a = ap[(size_t)i];
    if (!x.opt && (x.argtype == OP_ARG_DAT || x.argtype == OP_ARG_GBL)) {
      // switched off: typed scratch of the argument's shape
      a.kind = OFF;
      a.ctype = base_type(x.argtype == OP_ARG_DAT && x.dat ? x.dat->type : x.type);
      a.bytes = type_size(a.ctype);
      if (!a.bytes) a.ctype = "double", a.bytes = 8;
      a.dim = std::max(x.argtype == OP_ARG_DAT && x.dat ? x.dat->dim : x.dim, 1);
      a.vec = x.argtype == OP_ARG_DAT && x.map && x.idx < -1 ? -x.idx : 0;
      key << "|off:" << a.ctype << ":" << a.dim << ":" << a.vec;
      continue;
    }
    if (x.argtype == OP_ARG_DAT) {
      if (!x.dat) return set_error("op_par_loop(%s): argument %d: no dat", name, i), -1;
      a.ctype = base_type(x.dat->type);
      a.bytes = type_size(a.ctype);
      a.dim = x.dat->dim;
      a.acc = x.acc;
      if (!a.bytes || a.bytes * a.dim != x.dat->size) {
        set_error("op_par_loop(%s): argument %d: dat type '%s' is not double, float or int",
                  name, i, x.dat->type);
        return -1;
      }
      if (x.map == nullptr) {
        if (x.dat->set != set) return set_error("op_par_loop(%s): argument %d: dat is not on the loop's set", name, i), -1;
        a.kind = DIRECT;
      } else {
        if (x.idx >= x.map->dim || x.idx == -1 || -x.idx > x.map->dim) {
          set_error("op_par_loop(%s): argument %d: map index %d does not fit a map of dimension "
                    "%d", name, i, x.idx, x.map->dim);
          return -1;
        }
        a.vec = x.idx < -1 ? -x.idx : 0;
        if (x.map->from != set || x.map->to != x.dat->set)
          return set_error("op_par_loop(%s): argument %d: map does not match the loop's set and the dat", name, i), -1;
        if (x.acc != OP_READ && x.acc != OP_INC && x.acc != OP_WRITE && x.acc != OP_RW)
          return set_error("op_par_loop(%s): argument %d: indirect dats are OP_READ, OP_WRITE, OP_RW or OP_INC", name, i), -1;
        coloured |= x.acc == OP_WRITE || x.acc == OP_RW;
        a.kind = INDIRECT;
        a.mdim = x.map->dim;
        a.idx = x.idx;
      }
    } else if (x.argtype == OP_ARG_GBL) {
      a.kind = GBL;
      a.ctype = base_type(x.type);
      a.bytes = type_size(a.ctype);
      a.dim = x.dim;
      a.acc = x.acc;
      if (!a.bytes || !x.data || a.dim <= 0)
        return set_error("op_par_loop(%s): argument %d: global of unsupported type '%s'", name, i, x.type ? x.type : ""), -1;
      if (a.acc != OP_READ && a.acc != OP_INC && a.acc != OP_MIN && a.acc != OP_MAX &&
          a.acc != OP_WORK)
        return set_error("op_par_loop(%s): argument %d: globals are OP_READ, OP_INC, OP_MIN, "
                         "OP_MAX or OP_WORK", name, i), -1;
    } else if (x.argtype == OP_ARG_IDX) {
      a.kind = IDX;
      a.ctype = "int";
      if (x.map) {
        if (x.map->from != set || x.idx < 0 || x.idx >= x.map->dim)
          return set_error("op_par_loop(%s): argument %d: op_arg_idx map or index does not fit the loop", name, i), -1;
        a.mdim = x.map->dim;
        a.idx = x.idx;
      }
    } else if (x.argtype == OP_ARG_INFO) {
      a.kind = INFO;
      a.ctype = base_type(x.type);
      a.bytes = type_size(a.ctype);
      a.dim = x.dim;
      a.idx = x.idx;  // the MIN/MAX global it follows
      const int g = x.idx;
      if (!a.bytes || a.dim <= 0 || !x.data || g < 0 || g >= nargs ||
          args[g].argtype != OP_ARG_GBL || args[g].dim != 1 || !args[g].opt ||
          (args[g].acc != OP_MIN && args[g].acc != OP_MAX))
        return set_error("op_par_loop(%s): argument %d: op_arg_info must follow a dim-1 "
                         "OP_MIN or OP_MAX global", name, i), -1;
    } else {
      return set_error("op_par_loop(%s): argument %d: unknown argument kind", name, i), -1;
    }
    key << "|" << a.kind << ":" << a.ctype << ":" << a.dim << ":" << a.acc << ":" << a.mdim
        << ":" << a.idx << ":" << a.vec;
  }
  // option jit_exact: a loop whose only effect is to increment one dat
  // through one map (no other writes, no global reductions, the dat read by
  // no other argument, each slot of the map incremented by at most one
  // argument) runs owner-computes: a thread per target walks the inverse map
  // and re-runs the kernel for each element that increments the target, in
  // element order, the target's argument pointing at its own sum.  The sum
  // then sees the sequential loop's additions in its order: bit for bit.
  int own = -1;
  if (r.opt_jit_exact && !coloured) {
    bool ok = true;
    std::vector<int> slots;
    for (int i = 0; i < nargs && ok; i++) {
      const ArgPlan &a = ap[(size_t)i];
      if (a.kind == INDIRECT && a.acc == OP_INC) {
        if (own < 0) own = i;
        else ok = args[i].dat == args[own].dat && args[i].map == args[own].map && !a.vec &&
                  !ap[(size_t)own].vec;
        slots.push_back(a.vec ? -1 : a.idx);
      } else if ((a.kind == DIRECT || a.kind == INDIRECT) && a.acc != OP_READ) {
        ok = false;
      } else if ((a.kind == GBL && a.acc != OP_READ && a.acc != OP_WORK) || a.kind == INFO) {
        ok = false;
      }
    }
    for (int i = 0; i < nargs && ok && own >= 0; i++)
      if ((ap[(size_t)i].kind == DIRECT || ap[(size_t)i].kind == INDIRECT) &&
          args[i].dat == args[own].dat && ap[(size_t)i].acc != OP_INC)
        ok = false;
    std::sort(slots.begin(), slots.end());
    ok = ok && std::adjacent_find(slots.begin(), slots.end()) == slots.end();
    if (!ok || own < 0 || (long long)args[own].map->from->size * args[own].map->dim >= INT32_MAX)
      own = -1;
    if (own >= 0) key << "|own" << own;
  }
  // option jit_warp: a direct dat that no other argument of the loop names
  // moves through the warp's shared memory in whole rows (coalesced) and the
  // kernel works on registers; an indirect dat the loop only reads is
  // gathered by vector loads; indirect increments are combined per warp
  // before the atomics.  Not for loops that run colour by colour (their
  // elements come permuted) except the gathers; rows up to 128 bytes, and
  // fewer where op_arg_info's reduction takes shared memory as well.
  bool has_info = false, has_red = false;
  for (auto &a : ap) {
    has_info |= a.kind == INFO;
    has_red |= a.kind == INFO || (a.kind == GBL && a.acc != OP_READ && a.acc != OP_WORK);
  }
  if (r.opt_jit_warp && own < 0) {
    std::map<op_dat, int> uses, writes;
    for (int i = 0; i < nargs; i++)
      if (ap[(size_t)i].kind == DIRECT || ap[(size_t)i].kind == INDIRECT) {
        uses[args[i].dat]++;
        if (ap[(size_t)i].acc != OP_READ) writes[args[i].dat]++;
      }
    // the warp buffer (256 threads x the widest row, 16-byte padded) shares
    // the 48 KB of static shared memory with op_arg_info's block reduction
    size_t info_bytes = 0;
    for (auto &a : ap)
      if (a.kind == INFO) info_bytes += 256 * (16 + (size_t)a.dim * a.bytes);
    const size_t budget = info_bytes < 46 * 1024 ? 46 * 1024 - info_bytes : 0;
    auto fits = [&](size_t row_bytes) {
      return row_bytes <= 128 && 256 * ((row_bytes + 15) & ~(size_t)15) <= budget;
    };
    bool gathers = false;
    for (auto &a : ap) gathers |= a.kind == INDIRECT && a.acc == OP_READ;
    for (int i = 0; i < nargs; i++) {
      ArgPlan &a = ap[(size_t)i];
      const int row = a.dim * a.bytes;
      // staged: rows the kernel reads (OP_READ, OP_RW, direct OP_INC), a
      // write-only row is stored by the kernel itself (loading it first cost
      // more than the scattered stores); read-only rows only in loops without
      // gathers, whose latency the staging would otherwise add to
      if (a.kind == DIRECT && !coloured && a.dim > 1 && uses[args[i].dat] == 1 &&
          fits((size_t)row + a.bytes) && a.acc != OP_WRITE && (a.acc != OP_READ || !gathers))
        a.stage = 1;
      if (a.kind == INDIRECT && !a.vec && a.acc == OP_READ && writes[args[i].dat] == 0) {
        const uintptr_t base = (uintptr_t)args[i].dat->data_d;
        const int vw = (row % 16 == 0 && base % 16 == 0) ? 16 / a.bytes
                       : (row % 8 == 0 && base % 8 == 0 && a.bytes < 8) ? 8 / a.bytes : 0;
        if (vw >= 2) {
          a.stage = 2;
          a.vw = vw;
        }
      }
      if (a.kind == INDIRECT && a.acc == OP_INC && !coloured && fits((size_t)row)) a.seg = true;
      key << "|w" << a.stage << a.vw << a.seg;
    }
  }
  std::string body;
  std::vector<std::string> seen;
  for (auto &p : sources().preludes) body += expand(p, seen, 0) + "\n";
  std::string types;
  if (sources().preludes.empty() && find_file("user_types.h", types)) {
    seen.push_back("user_types.h");
    body += expand(types, seen, 0) + "\n";
  }
  std::string ksrc;
  if (!find_file(std::string(name) + ".h", ksrc)) {
    set_error("op_par_loop(%s): no device implementation of this loop is registered, and no "
              "kernel source %s.h was registered or found on OP2B_KERNEL_PATH", name, name);
    return -1;
  }
  seen.push_back(std::string(name) + ".h");
  body += expand(ksrc, seen, 0);
  for (auto &kv : r.consts) key << "|c:" << kv.first << ":" << r.const_types[kv.first] << ":" << kv.second.size();
  key << "|s:" << std::hash<std::string>()(body) << "|col:" << coloured;
  // each op_arg_info's block reduction keeps every thread's value, element and
  // payload in static shared memory (256 threads a block)
  size_t info_smem = 0;
  for (auto &a : ap) {
    if (coloured && a.kind == INFO)
      return set_error("op_par_loop(%s): op_arg_info in a loop that runs colour by colour is "
                       "not supported", name), -1;
    if (a.kind == INFO) info_smem += 256 * (16 + (size_t)a.dim * a.bytes);
  }
  if (info_smem > 40 * 1024)
    return set_error("op_par_loop(%s): the op_arg_info payloads take %zu bytes of shared memory "
                     "for a 256-thread block's reduction, above the 40960 bytes allowed: use "
                     "fewer or smaller payloads (at most 144 bytes for one)", name, info_smem), -1;
  // the colouring (built once per loop signature and cached with the plans)
  const Plan *plan = nullptr;
  if (coloured && set->size > 0 && !(plan = colour_plan(name, set, nargs, args))) return -1;
  Jit &j = cache()[key.str()];
  if (!j.fn) {
    const std::string src = generate(name, ap, body, coloured, own);
    if (!compile(name, src, j)) {
      cache().erase(key.str());
      return -1;
    }
  }
  if (!upload_constants(j)) return -1;
  // globals: device copies (OP_READ values, reduction identities)
  std::vector<size_t> goff((size_t)nargs, 0);
  size_t gbytes = 0;
  for (int i = 0; i < nargs; i++)
    if (ap[(size_t)i].kind == GBL || ap[(size_t)i].kind == OFF) {  // OFF: zeroed scratch
      goff[(size_t)i] = gbytes;
      gbytes += ((size_t)ap[(size_t)i].dim * ap[(size_t)i].bytes + 15) & ~(size_t)15;
    }
  // INFO: per launched block, best value (double), its element, its payload
  const long long max_grid = (long long)r.nsm * 8;
  for (int i = 0; i < nargs; i++)
    if (ap[(size_t)i].kind == INFO) {
      goff[(size_t)i] = gbytes;
      gbytes += ((size_t)(max_grid + 1) * (16 + (size_t)ap[(size_t)i].dim * ap[(size_t)i].bytes) +
                 15) & ~(size_t)15;
    }
  std::vector<char> gh(gbytes, 0);
  for (int i = 0; i < nargs; i++) {  // INFO: the caller's payload after the per-block ones
    const ArgPlan &a = ap[(size_t)i];
    if (a.kind == INFO)
      memcpy(gh.data() + goff[(size_t)i] + 16 * max_grid + (size_t)max_grid * a.dim * a.bytes,
             args[i].data, (size_t)a.dim * a.bytes);
  }
  for (int i = 0; i < nargs; i++) {
    const ArgPlan &a = ap[(size_t)i];
    if (a.kind != GBL) continue;
    char *dst = gh.data() + goff[(size_t)i];
    if (a.acc == OP_READ || a.acc == OP_INC || a.acc == OP_WORK) {
      if (a.acc != OP_INC) memcpy(dst, args[i].data, (size_t)a.dim * a.bytes);
      continue;  // OP_INC starts from zero
    }
    for (int k = 0; k < a.dim; k++) {  // MIN / MAX start from the identity
      const bool mn = a.acc == OP_MIN;
      if (a.ctype == "double") {
        double v = mn ? HUGE_VAL : -HUGE_VAL;
        memcpy(dst + 8 * k, &v, 8);
      } else if (a.ctype == "float") {
        float v = mn ? HUGE_VALF : -HUGE_VALF;
        memcpy(dst + 4 * k, &v, 4);
      } else {
        int v = mn ? 2147483647 : (-2147483647 - 1);
        memcpy(dst + 4 * k, &v, 4);
      }
    }
  }
  if (gbytes > j.gbl_cap) {
    cudaStreamSynchronize(r.stream);
    cudaFree(j.gbl_d);
    j.gbl_d = nullptr;
    j.gbl_cap = 0;
    if (!cuda_ok(cudaMalloc(&j.gbl_d, gbytes), "op_par_loop: globals")) return -1;
    j.gbl_cap = gbytes;
  }
  if (gbytes && !cuda_ok(cudaMemcpyAsync(j.gbl_d, gh.data(), gbytes, cudaMemcpyHostToDevice,
                                         r.stream),
                         "op_par_loop: globals"))
    return -1;
  // parameters
  std::vector<void *> ptrs;
  ptrs.reserve((size_t)nargs * 4 + 1);  // kp keeps pointers into ptrs: no reallocation
  std::vector<void *> kp;
  int n = set->size;
  kp.push_back(&n);
  double bytes = 0.0;
  for (int i = 0; i < nargs; i++) {
    const ArgPlan &a = ap[(size_t)i];
    const op_arg &x = args[i];
    if (a.kind == DIRECT || a.kind == INDIRECT) {
      ptrs.push_back(x.dat->data_d);
      bytes += (double)x.dat->size * (a.kind == DIRECT ? n : x.dat->set->size);
    } else if (a.kind == GBL) {
      ptrs.push_back((char *)j.gbl_d + goff[(size_t)i]);
    } else if (a.kind == OFF) {
      ptrs.push_back((char *)j.gbl_d + goff[(size_t)i]);
    }
    if (a.kind == DIRECT || a.kind == INDIRECT || a.kind == GBL || a.kind == OFF)
      kp.push_back(&ptrs.back());
    if (a.kind == INDIRECT || (a.kind == IDX && a.mdim > 0)) {
      ptrs.push_back(x.map->map_d);
      kp.push_back(&ptrs.back());
      bytes += 4.0 * n;
    }
    if (a.kind == INFO) {
      char *base = (char *)j.gbl_d + goff[(size_t)i];
      ptrs.push_back(base);
      kp.push_back(&ptrs.back());
      ptrs.push_back(base + 8 * max_grid);
      kp.push_back(&ptrs.back());
      ptrs.push_back(base + 16 * max_grid);
      kp.push_back(&ptrs.back());
      ptrs.push_back(base + 16 * max_grid + (size_t)max_grid * a.dim * a.bytes);
      kp.push_back(&ptrs.back());
    }
  }
  // owner computes: the targets and the inverse of the increments' map
  const long long *ioff = nullptr;
  const int *ient = nullptr, *irows = nullptr;
  if (own >= 0) {
    const InvMap *inv = get_inverse_map(args[own].map);
    if (!inv) return -1;
    ioff = inv->off;
    ient = inv->ent;
    // every target, or only those that have entries (the others keep their values)
    irows = inv->all_rows ? nullptr : inv->rows;
    n = inv->all_rows ? inv->nto : inv->nrows;
    kp.push_back(&ioff);
    kp.push_back(&ient);
    kp.push_back(&irows);
  }
  r.begin_loop(name);
  // one launch over the set, or one per colour over its slice of col_reord
  const int ncol = plan ? plan->pub.ncolors : 1;
  const int *perm = plan ? plan->col_reord_d : nullptr;
  int first = 0;
  if (plan) {
    kp.push_back(&perm);
    kp.push_back(&first);
  }
  unsigned grid = 0;  // of the last launch (a loop with op_arg_info has one)
  for (int c = 0; c < ncol && set->size > 0 && n > 0; c++) {
    if (plan) {
      first = plan->pub.color2_offsets[c];
      n = plan->pub.color2_offsets[c + 1] - first;
    }
    if (n <= 0) continue;
    // a thread per element, unless per-block reduction partials bound the
    // grid (op_arg_info) or the global reductions' atomics should stay few
    grid = (unsigned)std::min<long long>(((long long)n + 255) / 256,
                                         has_red ? max_grid : (long long)INT32_MAX);
    if (!cuda_ok(cudaLaunchKernel((const void *)j.fn, dim3(grid), dim3(256), kp.data(), 0,
                                  r.stream),
                 "op_par_loop: launch")) {
      r.end_loop(bytes);
      return -1;
    }
    r.launches++;
  }
  n = set->size;
  r.end_loop(bytes);
  // reductions: combine with the caller's values once the loop has finished
  bool reduce = false;
  for (auto &a : ap) reduce |= a.kind == GBL && a.acc != OP_READ && a.acc != OP_WORK;
  if (!reduce) return 0;
  if (!cuda_ok(cudaMemcpyAsync(gh.data(), j.gbl_d, gbytes, cudaMemcpyDeviceToHost, r.stream),
               "op_par_loop: globals") ||
      !cuda_ok(cudaStreamSynchronize(r.stream), "op_par_loop: globals"))
    return -1;
  // op_arg_info first, against the caller's value of its global before the
  // loop: the payload of the best value over the blocks, lowest element on
  // ties, if that value improves on the caller's (else the kernel would
  // never have written it)
  for (int i = 0; i < nargs; i++) {
    const ArgPlan &a = ap[(size_t)i];
    if (a.kind != INFO || n == 0) continue;
    const ArgPlan &g = ap[(size_t)a.idx];
    const bool mx = g.acc == OP_MAX;
    const char *base = gh.data() + goff[(size_t)i];
    int best = -1;
    double bv = 0.0;
    long long be = 0;
    for (unsigned b = 0; b < grid; b++) {
      double v;
      long long e;
      memcpy(&v, base + 8 * b, 8);
      memcpy(&e, base + 8 * max_grid + 8 * b, 8);
      if (e == 0x7fffffffffffffffLL) continue;
      if (best < 0 || (mx ? v > bv : v < bv) || (v == bv && e < be)) {
        best = (int)b;
        bv = v;
        be = e;
      }
    }
    if (best < 0) continue;
    double u;  // the caller's value of the global
    const char *ud = args[a.idx].data;
    if (g.ctype == "double") memcpy(&u, ud, 8);
    else if (g.ctype == "float") {
      float f;
      memcpy(&f, ud, 4);
      u = f;
    } else {
      int k;
      memcpy(&k, ud, 4);
      u = k;
    }
    if (mx ? bv > u : bv < u)
      memcpy(args[i].data, base + 16 * max_grid + (size_t)best * a.dim * a.bytes,
             (size_t)a.dim * a.bytes);
  }
  for (int i = 0; i < nargs; i++) {
    const ArgPlan &a = ap[(size_t)i];
    if (a.kind != GBL || a.acc == OP_READ || a.acc == OP_WORK || n == 0) continue;
    const char *src = gh.data() + goff[(size_t)i];
    char *dst = args[i].data;
    for (int k = 0; k < a.dim; k++) {
      if (a.ctype == "double") {
        double v, u;
        memcpy(&v, src + 8 * k, 8);
        memcpy(&u, dst + 8 * k, 8);
        u = a.acc == OP_INC ? u + v : a.acc == OP_MIN ? (v < u ? v : u) : (v > u ? v : u);
        memcpy(dst + 8 * k, &u, 8);
      } else if (a.ctype == "float") {
        float v, u;
        memcpy(&v, src + 4 * k, 4);
        memcpy(&u, dst + 4 * k, 4);
        u = a.acc == OP_INC ? u + v : a.acc == OP_MIN ? (v < u ? v : u) : (v > u ? v : u);
        memcpy(dst + 4 * k, &u, 4);
      } else {
        int v, u;
        memcpy(&v, src + 4 * k, 4);
        memcpy(&u, dst + 4 * k, 4);
        u = a.acc == OP_INC ? u + v : a.acc == OP_MIN ? (v < u ? v : u) : (v > u ? v : u);
        memcpy(dst + 4 * k, &u, 4);
      }
    }
  }
  return 0;
}

}  // namespace op2b

extern "C" {

int op2b_register_kernel(const char *name, const char *source) {
  if (!name || !*name) {
    op2b::set_error("op2b_register_kernel: needs a kernel name");
    return -1;
  }
  std::string n(name);
  if (n.size() < 2 || n.compare(n.size() - 2, 2, ".h") != 0) n += ".h";
  if (source) op2b::sources().kernels[n] = source;
  else op2b::sources().kernels.erase(n);  // forget it
  op2b::release_jit();  // sources changed: compile afresh
  return 0;
}

int op2b_register_prelude(const char *source) {
  if (!source) {
    op2b::set_error("op2b_register_prelude: needs a source");
    return -1;
  }
  op2b::sources().preludes.push_back(source);
  op2b::release_jit();
  return 0;
}

}  // extern "C"
