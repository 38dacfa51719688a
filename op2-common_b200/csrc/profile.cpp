// Region profiling: the reference's op_profile tree (op2/src/externlib/
// op_profile.cpp:221-560, op2/include/op_profile.h) for applications on
// libop2b.
//
// An application brackets its phases with op_profile_start / enter / next /
// exit / end and prints the tree with op_profile_output.  Level
// (OP_PROFILE_LEVEL, read at op_profile_start, as in the reference):
//   0 disabled; 1 the application's regions only (the default);
//   2 regions plus one kernel node per op_par_loop under the region it runs
//     in; 3 as 2 (this library has no code-generated sections inside loops).
// OP_PROFILE_JSON_OUTPUT=<file> writes the tree as JSON at op_profile_output,
// with the reference's node fields (name, type, clock {n, total, min, max},
// num_ranks, children); durations are nanoseconds.
//
// The reference times regions with host clocks and a device-wide
// synchronisation at every boundary.  Here a region boundary records a CUDA
// event on the library's stream instead, so entering and leaving a region
// costs no synchronisation and the region's time is the device time between
// its boundaries (with the stream's work ordered as the calls were made).
// Event pairs are resolved together with the loops' own event pairs (at
// op_timing_output, op_profile_output, or when many are outstanding).  A
// loop's kernel node takes the same device time the per-loop table shows.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "op2b.h"
#include "op2b_runtime.h"

namespace op2b {

namespace {

struct ProfNode {
  std::string name;
  int type = 0;  // 0 standard, 1 kernel (a loop)
  long long n = 0;
  double total_ns = 0, min_ns = 0, max_ns = 0;
  int parent = -1;
  std::vector<int> children;
};

struct Profiler {
  int level = 1;
  bool started = false, finished = false;
  std::vector<ProfNode> nodes;        // nodes[0] is the root
  std::vector<int> scope;             // open regions, innermost last
  std::vector<cudaEvent_t> starts;    // their start events
  int extra_depth = 0;                // regions entered below the level's detail

  int child(int parent, const std::string &name, int type) {
    for (int c : nodes[(size_t)parent].children)
      if (nodes[(size_t)c].name == name) return c;
    ProfNode nd;
    nd.name = name;
    nd.type = type;
    nd.parent = parent;
    nodes.push_back(nd);
    const int id = (int)nodes.size() - 1;
    nodes[(size_t)parent].children.push_back(id);
    return id;
  }
};

Profiler &prof() {
  static Profiler p;
  return p;
}

cudaEvent_t take_event() {
  Runtime &r = rt();
  if (r.ev_free.empty()) {
    for (int i = 0; i < 64; i++) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) == cudaSuccess) r.ev_free.push_back(e);
    }
  }
  if (r.ev_free.empty()) return nullptr;
  cudaEvent_t e = r.ev_free.back();
  r.ev_free.pop_back();
  return e;
}

// a region's boundary: the stream's deferred work is launched first, so the
// region holds the work its calls asked for
cudaEvent_t boundary() {
  Runtime &r = rt();
  if (!r.ready()) return nullptr;
  if (r.outstanding()) r.flush_pending();
  cudaEvent_t e = take_event();
  if (e) cudaEventRecord(e, r.stream);
  return e;
}

void close_region() {
  Profiler &p = prof();
  const int id = p.scope.back();
  cudaEvent_t e0 = p.starts.back();
  p.scope.pop_back();
  p.starts.pop_back();
  cudaEvent_t e1 = boundary();
  if (e0 && e1) {
    Runtime &r = rt();
    r.pending.push_back(PendingTime{std::string(), e0, e1, id});
    if (r.pending.size() > 4096) r.resolve_timing();
  }
}

void json_node(FILE *f, const std::vector<ProfNode> &nodes, int id) {
  const ProfNode &n = nodes[(size_t)id];
  std::string esc;
  for (char c : n.name) {
    if (c == '"' || c == '\\') esc += '\\';
    esc += c;
  }
  fprintf(f, "{\"name\":\"%s\",\"type\":%d,\"clock\":{\"n\":%lld,\"total\":%.0f,\"min\":%.0f,"
             "\"max\":%.0f},\"num_ranks\":1,\"children\":[",
          esc.c_str(), n.type, n.n, n.total_ns, n.min_ns, n.max_ns);
  for (size_t i = 0; i < n.children.size(); i++) {
    if (i) fputc(',', f);
    json_node(f, nodes, n.children[i]);
  }
  fputs("]}", f);
}

void fmt(char *buf, size_t len, double ns) {
  if (ns >= 1e9) snprintf(buf, len, "%6.2fs", ns * 1e-9);
  else if (ns >= 1e6) snprintf(buf, len, "%5.1fms", ns * 1e-6);
  else if (ns >= 1e3) snprintf(buf, len, "%5.1fus", ns * 1e-3);
  else snprintf(buf, len, "%5.0fns", ns);
}

void print_tree(const std::vector<ProfNode> &nodes, int id, int indent) {
  const ProfNode &n = nodes[(size_t)id];
  char t[16], a[16], lo[16], hi[16];
  fmt(t, sizeof t, n.total_ns);
  fmt(a, sizeof a, n.n ? n.total_ns / (double)n.n : 0.0);
  fmt(lo, sizeof lo, n.min_ns);
  fmt(hi, sizeof hi, n.max_ns);
  printf("%*s%-*s %8lld  %s  %s  %s  %s\n", indent, "", 40 - indent, n.name.c_str(), n.n, t, a,
         lo, hi);
  // regions first, then the kernel nodes by descending total time
  std::vector<int> kern;
  for (int c : n.children) {
    if (nodes[(size_t)c].type == 1) kern.push_back(c);
    else print_tree(nodes, c, indent + 4);
  }
  std::sort(kern.begin(), kern.end(),
            [&](int x, int y) { return nodes[(size_t)x].total_ns > nodes[(size_t)y].total_ns; });
  for (int c : kern) print_tree(nodes, c, indent + 4);
}

}  // namespace

// a resolved event pair of the profiler: region node `id` took `ms`
void profile_submit(int id, float ms) {
  Profiler &p = prof();
  if (id < 0 || id >= (int)p.nodes.size()) return;
  ProfNode &n = p.nodes[(size_t)id];
  const double ns = (double)ms * 1e6;
  if (n.n == 0) {
    n.min_ns = n.max_ns = ns;
  } else {
    n.min_ns = std::min(n.min_ns, ns);
    n.max_ns = std::max(n.max_ns, ns);
  }
  n.n++;
  n.total_ns += ns;
}

// whether a loop called now is timed into a region of the profile
bool profile_times_loops() {
  Profiler &p = prof();
  return p.started && !p.finished && p.level >= 2 && !p.scope.empty();
}

// the kernel node a loop called now is timed into (-1: none)
int profile_loop_node(const std::string &loop) {
  Profiler &p = prof();
  if (!p.started || p.finished || p.level < 2 || p.scope.empty()) return -1;
  return p.child(p.scope.back(), loop + "/cuda/b200", 1);
}

// op_exit: the open regions' start events go back to the library (their
// times are lost); the tree, with every resolved time, stays for a later
// op_profile_output
void profile_on_exit() {
  Profiler &p = prof();
  if (!p.started || p.finished) return;
  for (cudaEvent_t e : p.starts)
    if (e) rt().ev_free.push_back(e);
  p.starts.clear();
  p.scope.clear();
  p.extra_depth = 0;
  p.finished = true;
}

}  // namespace op2b

using namespace op2b;

extern "C" {

void op_profile_start(const char *name) {
  Profiler &p = prof();
  if (p.started && !p.finished) return;
  p = Profiler{};
  if (const char *lv = getenv("OP_PROFILE_LEVEL")) {
    char *end = nullptr;
    long v = strtol(lv, &end, 10);
    if (end == lv || v < 0 || v > 3)
      printf("warning: OP_PROFILE_LEVEL set to unsupported value: %s\n", lv);
    else
      p.level = (int)v;
  }
  if (p.level == 0) return;
  p.started = true;
  ProfNode root;
  root.name = name ? name : "";
  p.nodes.push_back(root);
  p.scope.push_back(0);
  p.starts.push_back(boundary());
}

void op_profile_enter(const char *name) {
  Profiler &p = prof();
  if (!p.started || p.finished || p.scope.empty()) return;
  if (p.extra_depth > 0 || (p.level < 3 && p.nodes[(size_t)p.scope.back()].type == 1)) {
    p.extra_depth++;
    return;
  }
  const int id = p.child(p.scope.back(), name ? name : "", 0);
  p.scope.push_back(id);
  p.starts.push_back(boundary());
}

void op_profile_enter_kernel(const char *name, const char *target, const char *variant) {
  Profiler &p = prof();
  if (!p.started || p.finished || p.scope.empty()) return;
  if (p.level < 2) {
    p.extra_depth++;
    return;
  }
  std::string full = std::string(name ? name : "") + "/" + (target ? target : "") + "/" +
                     (variant ? variant : "");
  const int id = p.child(p.scope.back(), full, 1);
  p.scope.push_back(id);
  p.starts.push_back(boundary());
}

void op_profile_exit(void) {
  Profiler &p = prof();
  if (!p.started || p.finished) return;
  if (p.extra_depth > 0) {
    p.extra_depth--;
    return;
  }
  if (p.scope.size() > 1) close_region();
}

void op_profile_next(const char *name) {
  op_profile_exit();
  op_profile_enter(name);
}

void op_profile_end(void) {
  Profiler &p = prof();
  if (!p.started || p.finished) return;
  p.extra_depth = 0;
  while (!p.scope.empty()) close_region();
  p.finished = true;
}

void op_profile_output_json(const char *fn) {
  Profiler &p = prof();
  if (!p.started || !p.finished || !fn) return;
  Runtime &r = rt();
  if (r.initialised) r.resolve_timing();
  FILE *f = fopen(fn, "w");
  if (!f) {
    printf("Unable to open timing JSON output file: %s\n", fn);
    return;
  }
  printf("Writing timing JSON to: %s\n", fn);
  json_node(f, p.nodes, 0);
  fclose(f);
}

void op_profile_output(void) {
  Profiler &p = prof();
  if (!p.started || !p.finished) return;
  Runtime &r = rt();
  if (r.initialised) r.resolve_timing();
  printf("\n%-40s %8s  %7s  %7s  %7s  %7s\n", "region (device time)", "num", "total", "avg",
         "min", "max");
  print_tree(p.nodes, 0, 0);
  printf("\n");
  if (const char *fn = getenv("OP_PROFILE_JSON_OUTPUT")) op_profile_output_json(fn);
}

}  // extern "C"
