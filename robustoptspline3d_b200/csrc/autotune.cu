// Launch-shape autotuner (rso_autotune).
//
// Three choices depend on the problem's size and shape more than on anything
// a fixed rule sees, so they are measured on the handle's own hierarchy with
// CUDA events, one after the other, and the fastest is kept in h->tune:
//   - thread rows of a CTA of the packed FP32 fine kernel (2, 4 or 8: 32 x 4,
//     32 x 8 or 32 x 16 element columns per CTA; the smaller tiles give small
//     grids more CTAs, the larger ones less halo per node) and the node planes
//     of its z chunks (32 down to 4: shorter chunks give small grids more CTAs
//     and each re-reads one plane),
//   - per coarse level, one thread per node (k_coarse4 / k_coarse), per
//     (node, row) (k_coarse_r) or nine per node (k_coarse_r9),
//   - the first level of the bottom kernel and its kind (or none).
// Each candidate is timed as whole solves (see solve_ms).
// The candidates compute the same arithmetic; only launch shapes differ.  The
// solver's work vectors are overwritten.
#include "rso_internal.cuh"

namespace rso {
namespace {

// random right-hand side at the active, unsupported fine nodes, zero elsewhere
__global__ void k_tune_rhs(const Level L, double* f, uint64_t seed) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= L.NP) return;
  const uint8_t c = L.vclass[i];
  const bool z = !(c & NC_ACTIVE) || (c & NC_SUPPORT);
#pragma unroll
  for (int k = 0; k < 3; k++) f[i + k * L.NP] = z ? 0.0 : rso_urand(seed, (uint64_t)(i + k * L.NP)) - 0.5;
}

struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  EventPair() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
  }
  ~EventPair() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

// mean device time of `reps` runs of body after `warm` untimed runs
template <typename F>
rso_status time_ms(rso_handle* h, int warm, int reps, F&& body, double* ms) {
  EventPair e;
  for (int r = 0; r < warm; r++) RSO_TRY(body());
  RSO_CHECK_CUDA(h, cudaEventRecord(e.a, h->stream));
  for (int r = 0; r < reps; r++) RSO_TRY(body());
  RSO_CHECK_CUDA(h, cudaEventRecord(e.b, h->stream));
  RSO_CHECK_CUDA(h, cudaEventSynchronize(e.b));
  float t = 0;
  RSO_CHECK_CUDA(h, cudaEventElapsedTime(&t, e.a, e.b));
  *ms = t / reps;
  return RSO_OK;
}


// Every candidate is timed as mixed-precision PCG solves to relative residual
// 1e-6 of a random load (the FP64 level vectors of the fine level hold it and
// the iterate; the mixed path does not use them): kernels then see the cache
// state and the graph replays they see in the solver.  One untimed solve
// captures the V-cycle graphs, two are timed; the result is per iteration.
rso_status solve_ms(rso_handle* h, double* ms) {
  Level& l0 = h->L[0];
  long long its = 0;
  bool timed = false;
  RSO_TRY(time_ms(h, 1, 2, [&]() -> rso_status {
    RSO_CHECK_CUDA(h, cudaMemsetAsync(l0.u64, 0, sizeof(double) * 3 * l0.NP, h->stream));
    rso_solve_info info;
    const rso_status st = solve_pcg(h, l0.f64, l0.u64, 1e-6, 100, &info);
    if (timed) its += info.iterations;
    timed = true;  // the first call is the untimed one
    return st == RSO_ERR_BUDGET_EXCEEDED ? RSO_OK : st;
  }, ms));
  // per PCG iteration: the candidates round differently, and a solve that
  // converges one iteration earlier says nothing about the launch shapes
  *ms = *ms * 2 / (double)(its > 0 ? its : 1);
  return RSO_OK;
}

// a candidate replaces the incumbent (the first value, the built-in rule's
// choice) only when it is faster by more than the run-to-run noise
constexpr double kTuneMargin = 0.97;

// tries the values of one choice in turn, keeps the fastest
template <typename Set>
rso_status pick(rso_handle* h, const std::vector<int>& values, Set&& set) {
  double best = 1e300;
  int keep = values.front();
  for (int v : values) {
    set(v);
    double ms = 0;
    RSO_TRY(solve_ms(h, &ms));
    if (ms < best * kTuneMargin || best == 1e300) { best = ms; keep = v; }
  }
  set(keep);
  return RSO_OK;
}

rso_status autotune(rso_handle* h) {
  const int nl = (int)h->L.size();
  Level& l0 = h->L[0];
  k_tune_rhs<<<cdiv(l0.NP, 256), 256, 0, h->stream>>>(l0, l0.f64, 4242); note_launch();
  RSO_TRY(launch_check(h, "autotune rhs"));
  // fine kernel tile, with the built-in rules for the rest
  RSO_TRY(pick(h, {4, 2, 8}, [&](int v) { h->tune.fine_rows = v; }));
  // its z chunk: the size rule's choice first, then the other lengths
  {
    h->tune.fine_zc = 0;
    std::vector<int> zc = {fine_zc(h)};
    for (int v = kFineZcMax; v >= kFineZcMin; v /= 2)
      if (v != zc.front()) zc.push_back(v);
    RSO_TRY(pick(h, zc, [&](int v) { h->tune.fine_zc = v; }));
  }
  // first level of the bottom kernel and its kind (2 level + kind: 1 the
  // persistent grid-wide kernel, 0 the cluster kernel), or none
  h->tune.bottom = 1;
  if (nl >= 3 && bottom_level(h) == 1) {
    // the built-in rule's choice first
    h->tune.bottom = -2;
    h->tune.bottom_kind = 1;
    const int rule = bottom_level(h);
    std::vector<int> cands = {rule > 0 ? 2 * rule + 1 : -1};
    if (rule > 0) cands.push_back(-1);
    for (int lb = nl - 2; lb >= 1; lb--) {
      bool small = true;
      for (int li = lb; li < nl; li++) small = small && h->L[li].nn <= kBottomMaxNodes;
      for (int kind = 1; small && kind >= 0; kind--)
        if (2 * lb + kind != cands.front()) cands.push_back(2 * lb + kind);
    }
    RSO_TRY(pick(h, cands, [&](int v) {
      h->tune.bottom = v < 0 ? -1 : v / 2;
      if (v >= 0) h->tune.bottom_kind = v % 2;
    }));
  } else {
    h->tune.bottom = -2;
  }
  // coarse kernel variant of each level the bottom kernel does not take
  const int lb = bottom_level(h);
  for (int li = 1; li < nl - 1 && li < 16 && (lb < 0 || li < lb); li++) {
    // the size rule's variant first, then the others
    h->tune.rowsplit[li] = -1;
    std::vector<int> v = {coarse_variant_of(h, li)};
    for (int k = 0; k <= 2; k++)
      if (k != v.front()) v.push_back(k);
    RSO_TRY(pick(h, v, [&](int x) { h->tune.rowsplit[li] = x; }));
  }
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  // graphs captured for the rejected candidates are never replayed again
  vcycle_graphs_free(h);
  return RSO_OK;
}

}  // namespace
}  // namespace rso

using namespace rso;

extern "C" rso_status rso_autotune(rso_handle* h, int* choices_host) {
  if (!h) return RSO_ERR_INVALID_ARG;
  if (!h->operators_ready) {
    h->err = "call rso_update_operators before rso_autotune";
    return RSO_ERR_STATE;
  }
  if (h->cfg.precision != RSO_MIXED || h->cfg.smoother == RSO_SMOOTH_GS) {
    h->err = "rso_autotune tunes the FP32 V-cycle with a Jacobi or Chebyshev smoother";
    return RSO_ERR_UNSUPPORTED;
  }
  const unsigned prof = h->prof_on;
  h->prof_on = 0;  // tuning runs stay out of the kernel profile
  const rso_status st = autotune(h);
  h->prof_on = prof;
  if (st != RSO_OK) {
    h->tune = rso_handle::Tune();
    return st;
  }
  if (choices_host) {
    choices_host[0] = h->tune.fine_rows;  // the z chunk is read with rso_fine_zchunk
    choices_host[1] = bottom_level(h);
    for (int li = 0; li < (int)h->L.size(); li++) choices_host[2 + li] = li > 0 && li < 16 ? h->tune.rowsplit[li] : -1;
  }
  return RSO_OK;
}

extern "C" rso_status rso_set_launch_shapes(rso_handle* h, const int* choices_host, int n) {
  if (!h || !choices_host || n < 2) return RSO_ERR_INVALID_ARG;
  const int nl = (int)h->L.size();
  if (choices_host[0] != 2 && choices_host[0] != 4 && choices_host[0] != 8) {
    h->err = "fine thread rows must be 2, 4 or 8";
    return RSO_ERR_INVALID_ARG;
  }
  const int b = choices_host[1];
  if (b < -2 || b == 0 || b > nl - 2) {
    h->err = "bottom level must be -2 (built-in rule), -1 (none) or a level from 1 to n_levels - 2";
    return RSO_ERR_INVALID_ARG;
  }
  rso_handle::Tune t;
  t.fine_zc = h->tune.fine_zc;  // set on their own (rso_set_fine_zchunk, rso_set_bottom_kernel)
  t.bottom_kind = h->tune.bottom_kind;
  t.fine_rows = choices_host[0];
  t.bottom = b;
  for (int li = 0; li < nl && 2 + li < n && li < 16; li++) {
    const int r = choices_host[2 + li];
    if (r < -1 || r > 2) {
      h->err = "coarse kernel choices are -1 (size rule), 0 (per node), 1 (per node and row) or 2 (nine per node)";
      return RSO_ERR_INVALID_ARG;
    }
    t.rowsplit[li] = li > 0 ? r : -1;
  }
  h->tune = t;
  return RSO_OK;
}
