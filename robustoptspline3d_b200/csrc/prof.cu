// Launch accounting and per-kernel CUDA-event timing.
//
// Every kernel launch of the library bumps a process-wide counter
// (rso_launch_count).  With profiling switched on for a handle, the fine- and
// coarse-level operator kernels are bracketed by event pairs on the
// handle's stream; rso_profile_top reports the kernel class with the largest
// total device time together with its algorithmic bytes and flops per
// launch, which is what the roofline figures are computed from.
#include "rso_internal.cuh"
#include <atomic>
#include <cstring>

static std::atomic<long long> g_launches{0};

namespace rso {

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void note_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

struct ProfClassInfo {
  const char* name;
  double bytes_per_node;  // minimum algorithmic traffic (each array touched once)
  double flops_per_node;
};

// u/f/out vectors 3 components, rho^p one value per node (one element per node), node class 1 byte
static const ProfClassInfo kInfo[PC_N] = {
    {"fine_jacobi_fp32", 12 + 12 + 4 + 1 + 12, 1200 + 60},
    {"fine_residual_fp32", 12 + 12 + 4 + 1 + 12, 1200},
    {"fine_gs_fp32", 12 + 12 + 4 + 1 + 12, 1200 + 80},
    {"fine_applyK_fp64", 24 + 8 + 1 + 24, 1200},
    {"fine_residual_fp64", 24 + 24 + 8 + 1 + 24, 1200},
    {"fine_jacobi_fp64", 24 + 24 + 8 + 1 + 24, 1200 + 60},
    {"fine_gs_fp64", 24 + 24 + 8 + 1 + 24, 1200 + 80},
    {"coarse_stencil_fp32", 243 * 4 + 12 + 12 + 12 + 1, 486},
    {"coarse_stencil_fp64", 243 * 8 + 24 + 24 + 24 + 1, 486},
    // the same operator, four nodes per thread on 16-byte streams (large FP32 levels)
    {"coarse_stencil_fp32_streamed", 243 * 4 + 12 + 12 + 12 + 1, 486},
    // the whole bottom of a V-cycle in one launch (its levels' nodes counted
    // once; no per-node traffic figure)
    {"vcycle_bottom", 0, 0},
};

struct Prof {
  std::vector<cudaEvent_t> ev[PC_N];
  std::vector<double> nodes[PC_N];
  size_t used[PC_N] = {};
  // launches timed inside replayed V-cycle graphs
  double graph_ms[PC_N] = {}, graph_nodes[PC_N] = {};
  long long graph_n[PC_N] = {};
};

// Inside a stream capture the event pair of a launch is recorded as a graph
// node (cudaEventRecordExternal) from a pool made before the capture began;
// every replay re-records the same events, so they are read (prof_harvest)
// before the graph runs again.
struct ProfPair {
  int cls = 0;
  double nodes = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
};
struct ProfPairs {
  std::vector<ProfPair> pairs;
  size_t used = 0;
};

void* prof_pairs_new(int capacity) {
  ProfPairs* v = new ProfPairs();
  v->pairs.resize(capacity);
  for (auto& p : v->pairs) {
    cudaEventCreate(&p.e0);
    cudaEventCreate(&p.e1);
  }
  return v;
}

void prof_pairs_free(void* pairs) {
  ProfPairs* v = (ProfPairs*)pairs;
  if (!v) return;
  for (auto& p : v->pairs) {
    cudaEventDestroy(p.e0);
    cudaEventDestroy(p.e1);
  }
  delete v;
}

bool prof_pairs_used(const void* pairs) { return pairs && ((const ProfPairs*)pairs)->used > 0; }

void prof_harvest(rso_handle* h, void* pairs) {
  ProfPairs* v = (ProfPairs*)pairs;
  if (!v || v->used == 0) return;
  Prof* p = (Prof*)h->prof;
  if (!p) { p = new Prof(); h->prof = p; }
  for (size_t k = 0; k < v->used; k++) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, v->pairs[k].e0, v->pairs[k].e1) != cudaSuccess) continue;
    const int c = v->pairs[k].cls;
    p->graph_ms[c] += ms;
    p->graph_nodes[c] += v->pairs[k].nodes;
    p->graph_n[c]++;
  }
}

void prof_begin(rso_handle* h, int cls, double nodes) {
  if (!((h->prof_on >> cls) & 1)) return;
  if (h->cap_prof) {
    ProfPairs* v = (ProfPairs*)h->cap_prof;
    if (v->used >= v->pairs.size()) return;  // pool exhausted: launch left untimed
    ProfPair& pp = v->pairs[v->used];
    pp.cls = cls;
    pp.nodes = nodes;
    cudaEventRecordWithFlags(pp.e0, h->stream, cudaEventRecordExternal);
    return;
  }
  Prof* p = (Prof*)h->prof;
  if (!p) { p = new Prof(); h->prof = p; }
  size_t k = p->used[cls];
  while (p->ev[cls].size() < k + 2) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    p->ev[cls].push_back(e);
  }
  if (p->nodes[cls].size() < k / 2 + 1) p->nodes[cls].resize(k / 2 + 1);
  p->nodes[cls][k / 2] = nodes;
  cudaEventRecord(p->ev[cls][k], h->stream);
}

void prof_end(rso_handle* h, int cls) {
  if (!((h->prof_on >> cls) & 1)) return;
  if (h->cap_prof) {
    ProfPairs* v = (ProfPairs*)h->cap_prof;
    if (v->used >= v->pairs.size()) return;
    cudaEventRecordWithFlags(v->pairs[v->used].e1, h->stream, cudaEventRecordExternal);
    v->used++;
    return;
  }
  Prof* p = (Prof*)h->prof;
  size_t k = p->used[cls];
  cudaEventRecord(p->ev[cls][k + 1], h->stream);
  p->used[cls] = k + 2;
}

void prof_free(rso_handle* h) {
  Prof* p = (Prof*)h->prof;
  if (!p) return;
  for (int c = 0; c < PC_N; c++)
    for (auto e : p->ev[c]) cudaEventDestroy(e);
  delete p;
  h->prof = nullptr;
}

}  // namespace rso

using namespace rso;

extern "C" long long rso_launch_count(void) { return g_launches.load(); }

extern "C" rso_status rso_set_profiling(rso_handle* h, int on) {
  if (!h) return RSO_ERR_INVALID_ARG;
  h->prof_on = on ? (1u << PC_N) - 1 : 0u;
  return RSO_OK;
}

extern "C" rso_status rso_set_profiling_classes(rso_handle* h, unsigned mask) {
  if (!h) return RSO_ERR_INVALID_ARG;
  h->prof_on = mask & ((1u << PC_N) - 1);
  return RSO_OK;
}

extern "C" rso_status rso_profile_reset(rso_handle* h) {
  if (!h) return RSO_ERR_INVALID_ARG;
  vcycle_graphs_harvest(h);  // drop timings of replays still unread
  Prof* p = (Prof*)h->prof;
  if (p)
    for (int c = 0; c < PC_N; c++) {
      p->used[c] = 0;
      p->graph_ms[c] = p->graph_nodes[c] = 0;
      p->graph_n[c] = 0;
    }
  return RSO_OK;
}

extern "C" rso_status rso_profile_class(rso_handle* h, int cls, char* name, int name_len, long long* launches,
                                        double* total_ms, double* bytes_per_launch, double* flops_per_launch) {
  if (!h || cls < 0 || cls >= PC_N) return RSO_ERR_INVALID_ARG;
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  vcycle_graphs_harvest(h);
  Prof* p = (Prof*)h->prof;
  double tot = 0, nodes = 0;
  long long n = 0;
  if (p) {
    for (size_t k = 0; k + 1 < p->used[cls]; k += 2) {
      float ms = 0;
      cudaEventElapsedTime(&ms, p->ev[cls][k], p->ev[cls][k + 1]);
      tot += ms;
      nodes += p->nodes[cls][k / 2];
      n++;
    }
    tot += p->graph_ms[cls];
    nodes += p->graph_nodes[cls];
    n += p->graph_n[cls];
  }
  if (name && name_len > 0) {
    std::strncpy(name, kInfo[cls].name, name_len - 1);
    name[name_len - 1] = 0;
  }
  if (launches) *launches = n;
  if (total_ms) *total_ms = tot;
  const double avg_nodes = n ? nodes / n : 0;
  if (bytes_per_launch) *bytes_per_launch = avg_nodes * kInfo[cls].bytes_per_node;
  if (flops_per_launch) *flops_per_launch = avg_nodes * kInfo[cls].flops_per_node;
  return RSO_OK;
}

extern "C" rso_status rso_profile_top(rso_handle* h, char* name, int name_len, long long* launches, double* total_ms,
                                      double* bytes_per_launch, double* flops_per_launch) {
  if (!h) return RSO_ERR_INVALID_ARG;
  int best = 0;
  double best_ms = -1;
  for (int c = 0; c < PC_N; c++) {
    double t = 0;
    RSO_TRY(rso_profile_class(h, c, nullptr, 0, nullptr, &t, nullptr, nullptr));
    if (t > best_ms) { best_ms = t; best = c; }
  }
  return rso_profile_class(h, best, name, name_len, launches, total_ms, bytes_per_launch, flops_per_launch);
}
