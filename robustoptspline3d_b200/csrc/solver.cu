// Multigrid V-cycle (templated on the arithmetic type), the FP64 outer
// iterations (defect correction and V-cycle preconditioned CG) and the
// reference-sequenced V-cycle on a caller vector.
//
// HierarchyGrid::v_cycle (grid/Grid.cpp:2431-2476): down-sweep computes the
// finer residual, restricts it, zeroes u and pre-smooths; the coarsest level
// is solved directly; the up-sweep prolongates and post-smooths.  In mixed
// precision the V-cycle runs in FP32 on FP32 copies of rho^p and of the
// coarse stencils; the CG recurrence runs in FP32 too unless the handle's
// replacement factor is 0 (then the outer residual and the CG vectors are
// FP64), while the iterate, the sums, the residual replacements and the
// coarsest solve stay FP64.
#include "rso_internal.cuh"
#include <cmath>
#include <cstring>
#include <utility>

namespace rso {

template <typename T>
struct LV;
template <>
struct LV<double> {
  static double*& u(Level& l) { return l.u64; }
  static double*& f(Level& l) { return l.f64; }
  static double*& r(Level& l) { return l.r64; }
  static double*& t(Level& l) { return l.t64; }
  static const double* rp(rso_handle* h) { return h->rp64; }
};
template <>
struct LV<float> {
  static float*& u(Level& l) { return l.u32; }
  static float*& f(Level& l) { return l.f32; }
  static float*& r(Level& l) { return l.r32; }
  static float*& t(Level& l) { return l.t32; }
  static const float* rp(rso_handle* h) { return h->rp32; }
};

// Step coefficients of the stationary smoothers, out = u + c1 (u - u_prev) +
// om D^-1 (f - K u): damped Jacobi (om = omega * 2 / lambda_max, c1 = 0), or
// Chebyshev iteration for D^-1 K on [a, b] = [cheb_lower lambda_max,
// lambda_max] by the three-term recurrence: theta = (b + a) / 2,
// delta = (b - a) / 2, sigma = theta / delta, rho_0 = 1 / sigma,
// rho_k = 1 / (2 sigma - rho_{k-1}); step 0 has om = 1 / theta, step k has
// c1 = rho_k rho_{k-1} and om = 2 rho_k / delta.
void smoother_steps(const rso_handle* h, double lam, int m, double* om, double* c1) {
  if (h->cfg.smoother == RSO_SMOOTH_CHEBYSHEV) {
    const double b = lam, a = lam * h->cfg.cheb_lower, theta = 0.5 * (b + a), delta = 0.5 * (b - a),
                 sigma = theta / delta;
    double rho_prev = 1.0 / sigma;
    for (int k = 0; k < m; k++) {
      if (k == 0) { om[0] = 1.0 / theta; c1[0] = 0.0; continue; }
      const double rho = 1.0 / (2.0 * sigma - rho_prev);
      c1[k] = rho * rho_prev;
      om[k] = 2.0 * rho / delta;
      rho_prev = rho;
    }
  } else {
    for (int k = 0; k < m; k++) { om[k] = h->cfg.omega * 2.0 / lam; c1[k] = 0.0; }
  }
}

// zero: the iterate is known to be zero before the first sweep (the first
// sweep on the fine level then needs no operator application).  Jacobi and
// Chebyshev steps rotate three level vectors: u (current), t (next) and r
// (previous iterate; free while the level is being smoothed).
// last_dot (FP32 fine level only): the last step also sums f . u into it
template <typename T>
static rso_status smooth(rso_handle* h, int li, int sweeps, int reverse, bool zero = false, double* last_dot = nullptr) {
  Level& l = h->L[li];
  if (h->cfg.smoother == RSO_SMOOTH_GS) {
    for (int s = 0; s < sweeps; s++)
      for (int ci = 0; ci < 8; ci++) {
        const int c = reverse ? 7 - ci : ci;
        if (li == 0) RSO_TRY(fine_gs<T>(h, LV<T>::u(l), LV<T>::f(l), LV<T>::rp(h), c, reverse));
        else RSO_TRY(coarse_gs<T>(h, li, LV<T>::u(l), LV<T>::f(l), c, reverse));
      }
    return RSO_OK;
  }
  double om[kMaxSweeps], c1[kMaxSweeps];
  if (sweeps > kMaxSweeps) { h->err = "too many smoothing sweeps"; return RSO_ERR_INVALID_ARG; }
  smoother_steps(h, l.lam, sweeps, om, c1);
  const bool cheb = h->cfg.smoother == RSO_SMOOTH_CHEBYSHEV;
  for (int s = 0; s < sweeps; s++) {
    // previous iterate: none before the second step; zero when the smoothing started from zero
    const T* prev = (!cheb || s == 0 || (zero && s == 1)) ? nullptr : LV<T>::r(l);
    const bool dot_here = last_dot != nullptr && li == 0 && s == sweeps - 1 && !(zero && s == 0);
    if (li == 0 && zero && s == 0) RSO_TRY(fine_jacobi0<T>(h, LV<T>::f(l), LV<T>::t(l), LV<T>::rp(h), om[0]));
    else if (dot_here) {
      if constexpr (sizeof(T) == 4)
        RSO_TRY(fine_jacobi_dot32(h, LV<T>::u(l), LV<T>::f(l), LV<T>::t(l), om[s], prev, c1[s], last_dot,
                                  h->vc_zdot_stride));
    } else if (li == 0) RSO_TRY(fine_jacobi<T>(h, LV<T>::u(l), LV<T>::f(l), LV<T>::t(l), LV<T>::rp(h), om[s], prev, c1[s]));
    else RSO_TRY(coarse_jacobi<T>(h, li, LV<T>::u(l), LV<T>::f(l), LV<T>::t(l), om[s], prev, c1[s]));
    if (cheb) {  // previous <- current <- next
      T* old_prev = LV<T>::r(l);
      LV<T>::r(l) = LV<T>::u(l);
      LV<T>::u(l) = LV<T>::t(l);
      LV<T>::t(l) = old_prev;
    } else {
      std::swap(LV<T>::u(l), LV<T>::t(l));
    }
  }
  return RSO_OK;
}

template <typename T>
static rso_status level_residual(rso_handle* h, int li) {
  Level& l = h->L[li];
  if (li == 0) return fine_residual<T>(h, LV<T>::u(l), LV<T>::f(l), LV<T>::r(l), LV<T>::rp(h));
  return coarse_residual<T>(h, li, LV<T>::u(l), LV<T>::f(l), LV<T>::r(l));
}

// V-cycle on the level work vectors: L[0].f holds the right-hand side and
// L[0].u the initial iterate; the result is left in L[0].u.
template <typename T>
rso_status vcycle_levels(rso_handle* h, int pre, int post, int symmetric, bool u0_zero) {
  const int nl = (int)h->L.size();
  // levels from lb down run inside one bottom kernel (bottom_vcycle)
  const int lb = bottom_level(h, sizeof(T) == 4);
  const int top = lb > 0 ? lb : nl;
  for (int li = 0; li < top; li++) {
    Level& l = h->L[li];
    if (li > 0) {
      RSO_TRY(level_residual<T>(h, li - 1));
      RSO_TRY(restrict_<T>(h, li, LV<T>::r(h->L[li - 1]), LV<T>::f(l)));
      RSO_CHECK_CUDA(h, cudaMemsetAsync(LV<T>::u(l), 0, sizeof(T) * 3 * l.NP * l.nb, h->stream));
    }
    const bool zero = li > 0 || u0_zero;
    if (li < nl - 1) RSO_TRY(smooth<T>(h, li, pre, 0, zero));
    else if (nl > 1) RSO_TRY(coarsest_solve<T>(h, LV<T>::f(l), LV<T>::u(l)));
    else {  // single level: smoothing only, kept symmetric
      RSO_TRY(smooth<T>(h, li, pre, 0, zero));
      RSO_TRY(smooth<T>(h, li, post, symmetric ? 1 : 0));
    }
  }
  if (lb > 0) {
    RSO_TRY(level_residual<T>(h, lb - 1));
    RSO_TRY(restrict_<T>(h, lb, LV<T>::r(h->L[lb - 1]), LV<T>::f(h->L[lb])));
    RSO_TRY(bottom_vcycle<T>(h, lb, pre, post));
  }
  // up-sweep from the level above the coarsest (or above the cluster kernel's levels)
  // the FP32 V-cycle's last fine step may also sum f . u (h->vc_zdot)
  double* zdot = sizeof(T) == 4 ? h->vc_zdot : nullptr;
  for (int li = lb > 0 ? lb - 1 : nl - 2; li >= 0; li--) {
    RSO_TRY(prolong<T>(h, li + 1, LV<T>::u(h->L[li + 1]), LV<T>::u(h->L[li])));
    RSO_TRY(smooth<T>(h, li, post, symmetric ? 1 : 0, false, li == 0 ? zdot : nullptr));
  }
  return RSO_OK;
}

template rso_status vcycle_levels<double>(rso_handle*, int, int, int, bool);
template rso_status vcycle_levels<float>(rso_handle*, int, int, int, bool);

__global__ void k_d2f(const double* __restrict__ a, float* __restrict__ b, long long n) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}
__global__ void k_f2d(const float* __restrict__ a, double* __restrict__ b, long long n) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (double)a[i];
}

rso_status to_f32(rso_handle* h, const double* a, float* b, long long n) {
  k_d2f<<<cdiv(n, 256), 256, 0, h->stream>>>(a, b, n); rso::note_launch();
  return launch_check(h, "to_f32");
}
rso_status to_f64(rso_handle* h, const float* a, double* b, long long n) {
  k_f2d<<<cdiv(n, 256), 256, 0, h->stream>>>(a, b, n); rso::note_launch();
  return launch_check(h, "to_f64");
}

// z = M r: one V-cycle from a zero iterate (FP32 in mixed precision)
rso_status precondition(rso_handle* h, const double* r, double* z) {
  Level& l0 = h->L[0];
  const long long n3 = 3 * l0.NP;
  const int pre = h->cfg.pre, post = h->cfg.post;
  if (h->cfg.precision == RSO_MIXED) {
    k_d2f<<<cdiv(n3, 256), 256, 0, h->stream>>>(r, l0.f32, n3); rso::note_launch();
    RSO_CHECK_CUDA(h, cudaMemsetAsync(l0.u32, 0, sizeof(float) * n3, h->stream));
    RSO_TRY(vcycle_levels<float>(h, pre, post, 1, true));
    k_f2d<<<cdiv(n3, 256), 256, 0, h->stream>>>(l0.u32, z, n3); rso::note_launch();
  } else {
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(l0.f64, r, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->stream));
    RSO_CHECK_CUDA(h, cudaMemsetAsync(l0.u64, 0, sizeof(double) * n3, h->stream));
    RSO_TRY(vcycle_levels<double>(h, pre, post, 1, true));
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(z, l0.u64, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->stream));
  }
  return launch_check(h, "precondition");
}

// scalar updates on the device: s[0]=rz, s[1]=pq, s[2]=alpha, s[3]=rz_new, s[4]=beta
__global__ void k_cg_alpha(double* s) { s[2] = s[0] / s[1]; }
__global__ void k_cg_beta(double* s) {
  s[4] = s[3] / s[0];
  s[0] = s[3];
}

// x += alpha p (the step of the previous iteration); p = z + beta p
template <typename Z>
__global__ void k_cg_step_dir(long long n, const double* __restrict__ alpha, const double* __restrict__ beta,
                              const Z* __restrict__ z, double* __restrict__ p, double* __restrict__ x) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double pi = p[i];
  x[i] += (*alpha) * pi;
  p[i] = (double)z[i] + (*beta) * pi;
}
__global__ void k_cg_step(long long n, const double* __restrict__ alpha, const double* __restrict__ p,
                          double* __restrict__ x) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) x[i] += (*alpha) * p[i];
}

// mixed precision: one FP32 V-cycle from a zero iterate on L[0].f32 (already
// holding the FP32 residual); the result is left in L[0].u32
static rso_status vcycle_mixed_launches(rso_handle* h) {
  Level& l0 = h->L[0];
  // the first damped-Jacobi sweep from zero reads no iterate; Gauss-Seidel does
  if (h->cfg.smoother == RSO_SMOOTH_GS || h->cfg.pre == 0)
    RSO_CHECK_CUDA(h, cudaMemsetAsync(l0.u32, 0, sizeof(float) * 3 * l0.NP * l0.nb, h->stream));
  return vcycle_levels<float>(h, h->cfg.pre, h->cfg.post, 1, true);
}

// ---------------------------------------------------------------- captured V-cycles
// The FP32 V-cycle of the preconditioner is about forty launches per CG
// iteration.  It is captured once into a CUDA graph and replayed.  What a
// capture freezes is the launch arguments: level vectors (the smoothers
// rotate three per level, so successive V-cycles differ and repeat with a
// short period), level sizes, smoother step sizes (from lambda_max), scratch
// and coarsest-solve buffers, the configuration and the profiling mask.  All
// of them form the key a graph is looked up by; a V-cycle whose key was not
// seen before runs as plain launches, the second time it is captured.  A
// graph also records how the rotating vectors end, which the host state takes
// on after a replay.
namespace {
struct VcGraph {
  std::vector<uint64_t> key, after;
  cudaGraphExec_t exec = nullptr;
  long long kernels = 0;
  void* pairs = nullptr;  // profiling event pairs inside the graph
  bool unread = false;    // replayed with event pairs not yet read
};
struct VcCache {
  std::vector<VcGraph> graphs;
  std::vector<std::vector<uint64_t>> seen;
  bool broken = false;  // a capture failed: plain launches from now on
};
constexpr size_t kMaxGraphs = 8, kMaxSeen = 32;

template <typename X>
void push_bits(std::vector<uint64_t>& k, X v) {
  uint64_t b = 0;
  static_assert(sizeof(X) <= 8, "key entries are at most 8 bytes");
  std::memcpy(&b, &v, sizeof(X));
  k.push_back(b);
}

// rotating = false leaves the rotating level vectors (u32, r32, t32) out
std::vector<uint64_t> vc_key(const rso_handle* h, bool rotating = true) {
  std::vector<uint64_t> k;
  for (const Level& l : h->L) {
    push_bits(k, rotating ? l.u32 : nullptr); push_bits(k, l.f32);
    push_bits(k, rotating ? l.r32 : nullptr); push_bits(k, rotating ? l.t32 : nullptr);
    push_bits(k, l.st32); push_bits(k, l.vclass); push_bits(k, l.emask);
    push_bits(k, l.NP); push_bits(k, l.nn); push_bits(k, l.nb); push_bits(k, l.lam);
    push_bits(k, l.nx); push_bits(k, l.ny); push_bits(k, l.nz); push_bits(k, l.px); push_bits(k, l.py);
    push_bits(k, l.factor);
  }
  push_bits(k, h->rp32); push_bits(k, h->xfer); push_bits(k, h->xfer_n);
  push_bits(k, h->c_K); push_bits(k, h->c_nodes); push_bits(k, h->c_f); push_bits(k, h->c_fb); push_bits(k, h->nc);
  push_bits(k, h->cfg.smoother); push_bits(k, h->cfg.pre); push_bits(k, h->cfg.post);
  push_bits(k, h->cfg.omega); push_bits(k, h->cfg.cheb_lower); push_bits(k, h->prof_on); push_bits(k, h->vc_zdot); push_bits(k, h->vc_zdot_stride);
  push_bits(k, h->tune.fine_rows); push_bits(k, h->tune.fine_zc); push_bits(k, h->tune.bottom);
  for (int r : h->tune.rowsplit) push_bits(k, r);
  return k;
}

std::vector<uint64_t> vc_rotating(const rso_handle* h) {
  std::vector<uint64_t> k;
  for (const Level& l : h->L) { push_bits(k, l.u32); push_bits(k, l.r32); push_bits(k, l.t32); }
  return k;
}

void vc_set_rotating(rso_handle* h, const std::vector<uint64_t>& v) {
  size_t i = 0;
  for (Level& l : h->L) {
    std::memcpy(&l.u32, &v[i++], sizeof(float*));
    std::memcpy(&l.r32, &v[i++], sizeof(float*));
    std::memcpy(&l.t32, &v[i++], sizeof(float*));
  }
}

void vc_drop(VcGraph& g) {
  if (g.exec) cudaGraphExecDestroy(g.exec);
  prof_pairs_free(g.pairs);
  g.exec = nullptr;
  g.pairs = nullptr;
}
}  // namespace

void vcycle_graphs_harvest(rso_handle* h) {
  VcCache* c = (VcCache*)h->vcg;
  if (!c) return;
  for (auto& g : c->graphs)
    if (g.unread) {
      prof_harvest(h, g.pairs);
      g.unread = false;
    }
}

void vcycle_graphs_free(rso_handle* h) {
  VcCache* c = (VcCache*)h->vcg;
  if (!c) return;
  for (auto& g : c->graphs) vc_drop(g);
  delete c;
  h->vcg = nullptr;
}

rso_status vcycle_mixed(rso_handle* h) {
  if (!h->vc_graphs || h->stream == nullptr) return vcycle_mixed_launches(h);
  if (!h->vcg) h->vcg = new VcCache();
  VcCache* c = (VcCache*)h->vcg;
  if (c->broken) return vcycle_mixed_launches(h);
  const std::vector<uint64_t> key = vc_key(h);
  for (auto& g : c->graphs)
    if (g.key == key) {
      if (g.unread) {  // its events still hold the previous replay's times
        RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
        vcycle_graphs_harvest(h);
      }
      RSO_CHECK_CUDA(h, cudaGraphLaunch(g.exec, h->stream));
      note_launches(g.kernels);
      vc_set_rotating(h, g.after);
      g.unread = prof_pairs_used(g.pairs);
      return launch_check(h, "vcycle graph");
    }
  bool seen = false;
  for (const auto& k : c->seen) seen = seen || k == key;
  if (!seen) {
    if (c->seen.size() >= kMaxSeen) c->seen.erase(c->seen.begin());
    c->seen.push_back(key);
    return vcycle_mixed_launches(h);
  }
  // capture: the launches are recorded, not run; the graph then runs once
  const std::vector<uint64_t> before = vc_rotating(h);
  VcGraph g;
  g.key = key;
  if (h->prof_on) g.pairs = prof_pairs_new(128);
  h->cap_prof = g.pairs;
  cudaGraph_t graph = nullptr;
  rso_status st = RSO_OK;
  if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    st = RSO_ERR_CUDA;
  } else {
    st = vcycle_mixed_launches(h);
    if (cudaStreamEndCapture(h->stream, &graph) != cudaSuccess) st = RSO_ERR_CUDA;
  }
  h->cap_prof = nullptr;
  cudaGetLastError();  // a failed capture leaves its error here; the plain V-cycle below reports its own
  if (st == RSO_OK && graph && cudaGraphInstantiate(&g.exec, graph, 0) != cudaSuccess) {
    g.exec = nullptr;
    st = RSO_ERR_CUDA;
  }
  if (st == RSO_OK) {
    size_t n = 0;
    cudaGraphGetNodes(graph, nullptr, &n);
    std::vector<cudaGraphNode_t> nodes(n);
    if (n) cudaGraphGetNodes(graph, nodes.data(), &n);
    for (auto nd : nodes) {
      cudaGraphNodeType t;
      if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) g.kernels++;
    }
  }
  if (graph) cudaGraphDestroy(graph);
  if (st != RSO_OK) {
    // run this V-cycle (and every later one) as plain launches from the state it started in
    vc_drop(g);
    c->broken = true;
    cudaGetLastError();
    vc_set_rotating(h, before);
    return vcycle_mixed_launches(h);
  }
  g.after = vc_rotating(h);
  // the captured launches were counted when they were recorded
  RSO_CHECK_CUDA(h, cudaGraphLaunch(g.exec, h->stream));
  g.unread = prof_pairs_used(g.pairs);
  if (c->graphs.size() >= kMaxGraphs) {
    if (c->graphs.front().unread) {
      RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
      vcycle_graphs_harvest(h);
    }
    vc_drop(c->graphs.front());
    c->graphs.erase(c->graphs.begin());
  }
  c->graphs.push_back(std::move(g));
  return launch_check(h, "vcycle graph");
}

// reliable-update PCG: x (FP64) += alpha p (FP32), and p = z + beta p in FP32
// (DIR_ONLY: the direction update alone, x having taken the step already)
template <bool DIR_ONLY>
__global__ void k_cg32_step_dir(long long n4, const double* __restrict__ alpha, const double* __restrict__ beta,
                                const float4* __restrict__ z, float4* __restrict__ p, double2* __restrict__ x) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n4) return;
  const float4 pi = p[i], zi = z[i];
  if (!DIR_ONLY) {
    const double a = *alpha;
    double2 x0 = x[2 * i], x1 = x[2 * i + 1];
    x0.x += a * pi.x;
    x0.y += a * pi.y;
    x1.x += a * pi.z;
    x1.y += a * pi.w;
    x[2 * i] = x0;
    x[2 * i + 1] = x1;
  }
  const float b = (float)*beta;
  p[i] = make_float4(zi.x + b * pi.x, zi.y + b * pi.y, zi.z + b * pi.z, zi.w + b * pi.w);
}
__global__ void k_cg32_step(long long n4, const double* __restrict__ alpha, const float4* __restrict__ p,
                            double2* __restrict__ x) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n4) return;
  const float4 pi = p[i];
  const double a = *alpha;
  double2 x0 = x[2 * i], x1 = x[2 * i + 1];
  x0.x += a * pi.x;
  x0.y += a * pi.y;
  x1.x += a * pi.z;
  x1.y += a * pi.w;
  x[2 * i] = x0;
  x[2 * i + 1] = x1;
}

// Deferred FP64 steps: x += alpha_j p_j for the k directions waiting in the
// ring, in their order (the step k_cg32_step_dir takes every iteration, taken
// later with the same operations in the same order, so x is bit-identical at
// every point where it is read)
constexpr int kStepRing = 4;
struct StepRing {
  const float4* p[kStepRing];
};
__global__ void k_cg32_flush(long long n4, const double* __restrict__ alpha, const StepRing R, int k,
                             double2* __restrict__ x) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n4) return;
  double2 x0 = x[2 * i], x1 = x[2 * i + 1];
#pragma unroll
  for (int j = 0; j < kStepRing; j++) {
    if (j >= k) break;
    const float4 pi = R.p[j][i];
    const double a = alpha[j];
    x0.x += a * pi.x;
    x0.y += a * pi.y;
    x1.x += a * pi.z;
    x1.y += a * pi.w;
  }
  x[2 * i] = x0;
  x[2 * i + 1] = x1;
}
// p_out = z + beta p_in in FP32 (the direction update of k_cg32_step_dir);
// p_out may be p_in
__global__ void k_cg32_dir(long long n4, const double* __restrict__ beta, const float4* __restrict__ z,
                           const float4* p_in, float4* p_out) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n4) return;
  const float4 pi = p_in[i], zi = z[i];
  const float b = (float)*beta;
  p_out[i] = make_float4(zi.x + b * pi.x, zi.y + b * pi.y, zi.z + b * pi.z, zi.w + b * pi.w);
}
// alpha = rz / pq, also kept for the deferred step
__global__ void k_cg_alpha_keep(double* s, double* keep) {
  s[2] = s[0] / s[1];
  *keep = s[2];
}

// Mixed-precision PCG with the Krylov recurrence in FP32 (no counterpart in
// the reference, whose CG is FP64): p, q = K p, r and z are FP32 and the
// iterate x accumulates alpha p in FP64.  The recursive FP32 residual drifts
// from the true one by the FP32 operator's rounding, so whenever it has
// dropped by h->krylov32 since the last replacement, and before stopping, the
// true residual f - K x is formed in FP64 and replaces it (residual
// replacement, the search direction kept).  The reported residual is always a
// true FP64 one.
// A cycle (iterations between replacements) ends after at most kCycleMax
// iterations.  A replacement whose true residual is not below
// max(0.5, sqrt(factor), sqrt(claimed)) times the previous one, claimed being
// the reduction the recursive residual showed over the cycle, means the FP32
// recurrence stalls (an operator too ill-conditioned for it): the solve then
// continues from the current iterate with the FP64 recurrence (*stalled,
// *used = the iterations spent here).  The claimed term keeps a short last
// cycle, ended by the tolerance after a small reduction, from counting as a
// stall.  h->krylov32_cycles > 0 hands over after that many cycles as well.
constexpr int kCycleMax = 30;
double stall_ratio(double factor, double claimed) {
  return std::max(std::max(0.5, std::sqrt(factor)), std::sqrt(std::max(claimed, 0.0)));
}
// ---------------------------------------------------------------- device-controlled solve
// The loop of solve_pcg_k32 below as one CUDA graph of kSolveUnroll
// iterations, each three conditional IF nodes: the first holds q = K p with
// p.q, alpha, the recursive residual update and a one-thread control kernel
// (k_pcg_ctl_a); the second the FP64 residual replacement and its control
// kernel (k_pcg_ctl_b); the third the V-cycle, r.z, beta and the direction
// update.  The control kernels take the host loop's decisions on the same
// device scalars with the same double arithmetic, so the graph reproduces the
// host loop's iterations; when the solve stops they switch off every later
// iteration of the graph.  The graph is straight-line (no WHILE node), so a
// launch ends after at most kSolveUnroll iterations whatever the control
// kernels decide; the host launches it again while the solve goes on.
constexpr int kSolveUnroll = 16;
struct PcgCtl {
  double fn, tol, krylov32, rbase, rel, rnorm;
  int max_iter, cycles_max, it, since, cycles, replace, status, done, n_rep, n_cont;
};
enum { PCG_RUNNING = 0, PCG_STALLED = 1, PCG_NONFINITE = 2 };
struct PcgGo {
  cudaGraphConditionalHandle go[kSolveUnroll];  // one per unrolled iteration
};

__device__ __forceinline__ void pcg_stop(PcgCtl* c, const PcgGo& g, int i) {
  c->done = 1;
  for (int j = i + 1; j < kSolveUnroll; j++) cudaGraphSetConditional(g.go[j], 0);
}

// after the recursive residual update: s[5] = r.r
__global__ void k_pcg_ctl_a(PcgCtl* c, const double* s, PcgGo g, int i, cudaGraphConditionalHandle hr,
                            cudaGraphConditionalHandle hc) {
  const double rnorm = sqrt(s[5]);
  c->it++;
  c->since++;
  c->rnorm = rnorm;
  if (!isfinite(rnorm)) {
    c->status = PCG_NONFINITE;
    c->replace = 0;
    cudaGraphSetConditional(hr, 0);
    cudaGraphSetConditional(hc, 0);
    pcg_stop(c, g, i);
    return;
  }
  const bool rep = rnorm < c->krylov32 * c->rbase || rnorm < c->tol * c->fn || c->it >= c->max_iter ||
                   c->since >= kCycleMax;
  c->replace = rep;
  if (rep) {
    c->n_rep++;
  } else {
    c->rel = rnorm / c->fn;
    c->n_cont++;
  }
  cudaGraphSetConditional(hr, rep ? 1u : 0u);
  cudaGraphSetConditional(hc, rep ? 0u : 1u);
}

__device__ __forceinline__ double stall_ratio_dev(double factor, double claimed) {
  return fmax(fmax(0.5, sqrt(factor)), sqrt(fmax(claimed, 0.0)));
}

// after the replacement: s[8] = true r.r
__global__ void k_pcg_ctl_b(PcgCtl* c, const double* s, PcgGo g, int i, cudaGraphConditionalHandle hc) {
  const double rtrue = sqrt(s[8]);
  c->rel = rtrue / c->fn;
  if (!isfinite(c->rel)) {
    c->status = PCG_NONFINITE;
    pcg_stop(c, g, i);
    return;
  }
  if (c->rel < c->tol || c->it >= c->max_iter) {
    pcg_stop(c, g, i);
    return;
  }
  c->cycles++;
  if (rtrue > stall_ratio_dev(c->krylov32, c->rnorm / c->rbase) * c->rbase ||
      (c->cycles_max > 0 && c->cycles >= c->cycles_max)) {
    c->status = PCG_STALLED;  // the true residual of x is in r
    pcg_stop(c, g, i);
    return;
  }
  c->rbase = rtrue;
  c->since = 0;
  c->n_cont++;
  cudaGraphSetConditional(hc, 1);
}

// the direction update of k_cg32_step_dir with the step taken or not as the
// control block says (after a replacement x has taken it already)
__global__ void k_cg32_step_dir_ctl(long long n4, const double* __restrict__ alpha, const double* __restrict__ beta,
                                    const float4* __restrict__ z, float4* __restrict__ p, double2* __restrict__ x,
                                    const PcgCtl* __restrict__ c) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n4) return;
  const float4 pi = p[i], zi = z[i];
  if (!c->replace) {
    const double a = *alpha;
    double2 x0 = x[2 * i], x1 = x[2 * i + 1];
    x0.x += a * pi.x;
    x0.y += a * pi.y;
    x1.x += a * pi.z;
    x1.y += a * pi.w;
    x[2 * i] = x0;
    x[2 * i + 1] = x1;
  }
  const float b = (float)*beta;
  p[i] = make_float4(zi.x + b * pi.x, zi.y + b * pi.y, zi.z + b * pi.z, zi.w + b * pi.w);
}

namespace {
struct SolveGraph {
  std::vector<uint64_t> key;
  cudaGraphExec_t exec = nullptr;
  long long k_iter = 0, k_rep = 0, k_cont = 0;  // kernels per iteration / replacement / continuation
};
struct SolveGraphs {
  std::vector<SolveGraph> graphs;
  PcgCtl* ctl = nullptr;
  PcgCtl* h_ctl = nullptr;
  cudaStream_t cs = nullptr;
  bool broken = false;
};
constexpr size_t kMaxSolveGraphs = 4;

// the launches a captured body records go to the capture stream
struct StreamSwap {
  rso_handle* h;
  cudaStream_t saved;
  StreamSwap(rso_handle* hh, cudaStream_t s) : h(hh), saved(hh->stream) { h->stream = s; }
  ~StreamSwap() { h->stream = saved; }
};

long long count_kernels(cudaGraph_t g) {
  size_t n = 0;
  cudaGraphGetNodes(g, nullptr, &n);
  std::vector<cudaGraphNode_t> nodes(n);
  if (n) cudaGraphGetNodes(g, nodes.data(), &n);
  long long k = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) k++;
  }
  return k;
}

// adds to G an IF node on handle hc after `dep` (none if null) whose body
// records the launches of `body`, captured on stream cs
template <class F>
rso_status add_if(rso_handle* h, cudaGraph_t G, cudaGraphNode_t* dep, cudaGraphConditionalHandle hc,
                  cudaStream_t cs, F body, cudaGraphNode_t* node, long long* kernels) {
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = hc;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 1;
  if (cudaGraphAddNode(node, G, dep, dep ? 1 : 0, &cp) != cudaSuccess) return RSO_ERR_CUDA;
  cudaGraph_t bg = cp.conditional.phGraph_out[0];
  if (cudaStreamBeginCaptureToGraph(cs, bg, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) != cudaSuccess)
    return RSO_ERR_CUDA;
  rso_status r;
  {
    StreamSwap sw(h, cs);
    r = body();
  }
  cudaGraph_t out = nullptr;
  if (cudaStreamEndCapture(cs, &out) != cudaSuccess) r = RSO_ERR_CUDA;
  *kernels = count_kernels(bg);
  return r;
}
}  // namespace

void solve_graphs_free(rso_handle* h) {
  SolveGraphs* c = (SolveGraphs*)h->sgc;
  if (!c) return;
  for (auto& g : c->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  cudaFree(c->ctl);
  if (c->h_ctl) cudaFreeHost(c->h_ctl);
  if (c->cs) cudaStreamDestroy(c->cs);
  delete c;
  h->sgc = nullptr;
}

// Builds the unrolled graph of the loop for iterate x and right-hand side f
// (FP64, padded); the V-cycle's rotating level vectors are left as they were.
static rso_status build_solve_graph(rso_handle* h, SolveGraphs* c, const double* f, double* x, SolveGraph* g) {
  Level& l0 = h->L[0];
  const long long n3 = 3 * l0.NP, n4 = n3 / 4;
  double* s = h->scal;
  float* r32 = l0.f32;
  float* p32 = reinterpret_cast<float*>(h->z);
  float* q32 = reinterpret_cast<float*>(h->q);
  PcgCtl* ctl = c->ctl;
  const std::vector<uint64_t> rot = vc_rotating(h);
  cudaGraph_t G = nullptr;
  rso_status st = RSO_OK;
  do {
    if (cudaGraphCreate(&G, 0) != cudaSuccess) { st = RSO_ERR_CUDA; break; }
    PcgGo go;
    cudaGraphConditionalHandle hr[kSolveUnroll], hc[kSolveUnroll];
    for (int i = 0; i < kSolveUnroll && st == RSO_OK; i++)
      if (cudaGraphConditionalHandleCreate(&go.go[i], G, 1, cudaGraphCondAssignDefault) != cudaSuccess ||
          cudaGraphConditionalHandleCreate(&hr[i], G, 0, cudaGraphCondAssignDefault) != cudaSuccess ||
          cudaGraphConditionalHandleCreate(&hc[i], G, 0, cudaGraphCondAssignDefault) != cudaSuccess)
        st = RSO_ERR_CUDA;
    if (st != RSO_OK) break;
    cudaGraphNode_t prev = nullptr, node = nullptr;
    for (int i = 0; i < kSolveUnroll && st == RSO_OK; i++) {
      long long k1 = 0, kr = 0, kc = 0;
      st = add_if(h, G, prev ? &prev : nullptr, go.go[i], c->cs, [&]() -> rso_status {
        RSO_TRY(fine_applyK_dot32(h, p32, q32, s + 1));
        k_cg_alpha<<<1, 1, 0, h->stream>>>(s);
        RSO_TRY(cg32_resid_rr(h, n3, s + 2, q32, r32, s + 5));
        k_pcg_ctl_a<<<1, 1, 0, h->stream>>>(ctl, s, go, i, hr[i], hc[i]);
        return launch_check(h, "pcg graph");
      }, &node, &k1);
      if (st != RSO_OK) break;
      prev = node;
      // the FP64 residual replacement
      st = add_if(h, G, &prev, hr[i], c->cs, [&]() -> rso_status {
        k_cg32_step<<<cdiv(n4, 256), 256, 0, h->stream>>>(n4, s + 2, reinterpret_cast<const float4*>(p32),
                                                          reinterpret_cast<double2*>(x));
        RSO_TRY(fine_residual64_rr(h, x, f, h->r, r32, s + 8));  // r, its FP32 copy and r . r
        k_pcg_ctl_b<<<1, 1, 0, h->stream>>>(ctl, s, go, i, hc[i]);
        return launch_check(h, "pcg graph");
      }, &node, &kr);
      if (st != RSO_OK) break;
      prev = node;
      // the V-cycle and the direction update
      st = add_if(h, G, &prev, hc[i], c->cs, [&]() -> rso_status {
        RSO_TRY(vcycle_mixed_launches(h));  // r . z into s[3] from its last fine step when h->vc_zdot says so
        const float* z32 = l0.u32;
        if (h->vc_zdot != s + 3) RSO_TRY(dot_ff(h, r32, z32, n3, s + 3));
        k_cg_beta<<<1, 1, 0, h->stream>>>(s);
        k_cg32_step_dir_ctl<<<cdiv(n4, 256), 256, 0, h->stream>>>(
            n4, s + 2, s + 4, reinterpret_cast<const float4*>(z32), reinterpret_cast<float4*>(p32),
            reinterpret_cast<double2*>(x), ctl);
        return launch_check(h, "pcg graph");
      }, &node, &kc);
      if (st != RSO_OK) break;
      prev = node;
      vc_set_rotating(h, rot);  // every unrolled V-cycle starts from the same vectors
      g->k_iter = k1; g->k_rep = kr; g->k_cont = kc;
    }
    if (st != RSO_OK) break;
    if (cudaGraphInstantiate(&g->exec, G, 0) != cudaSuccess) { g->exec = nullptr; st = RSO_ERR_CUDA; }
  } while (false);
  if (G) cudaGraphDestroy(G);
  vc_set_rotating(h, rot);
  cudaGetLastError();  // a failed capture leaves its error here
  return st;
}

// Runs the loop from the state solve_pcg_k32 prepared (p, r32, q, s[0] = r.z)
// on the device.  Returns RSO_ERR_UNSUPPORTED when no graph could be made
// (nothing has run then; the host loop takes over).
static rso_status pcg32_graph(rso_handle* h, const double* f, double* x, double tol, int max_iter, double fn,
                              double rbase, int* it, double* rel, bool* stalled) {
  if (!h->sgc) h->sgc = new SolveGraphs();
  SolveGraphs* c = (SolveGraphs*)h->sgc;
  if (c->broken) return RSO_ERR_UNSUPPORTED;
  if (!c->ctl) {
    if (cudaMalloc((void**)&c->ctl, sizeof(PcgCtl)) != cudaSuccess ||
        cudaMallocHost((void**)&c->h_ctl, sizeof(PcgCtl)) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->cs, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      c->broken = true;
      return RSO_ERR_UNSUPPORTED;
    }
  }
  // what vc_key holds without the rotating level vectors (the graph does not
  // depend on which of them a V-cycle starts from), and the loop's own vectors
  std::vector<uint64_t> key = vc_key(h, false);
  push_bits(key, f); push_bits(key, x); push_bits(key, h->z); push_bits(key, h->q); push_bits(key, h->r);
  push_bits(key, h->rp64); push_bits(key, h->scal);
  SolveGraph* g = nullptr;
  for (auto& e : c->graphs)
    if (e.key == key) g = &e;
  if (!g) {
    SolveGraph ng;
    ng.key = key;
    if (build_solve_graph(h, c, f, x, &ng) != RSO_OK) {
      if (ng.exec) cudaGraphExecDestroy(ng.exec);
      c->broken = true;
      return RSO_ERR_UNSUPPORTED;
    }
    if (c->graphs.size() >= kMaxSolveGraphs) {
      cudaGraphExecDestroy(c->graphs.front().exec);
      c->graphs.erase(c->graphs.begin());
    }
    c->graphs.push_back(ng);
    g = &c->graphs.back();
  }
  PcgCtl& hc = *c->h_ctl;
  hc = PcgCtl{};
  hc.fn = fn; hc.tol = tol; hc.krylov32 = h->krylov32; hc.rbase = rbase;
  hc.max_iter = max_iter; hc.cycles_max = h->krylov32_cycles;
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(c->ctl, c->h_ctl, sizeof(PcgCtl), cudaMemcpyHostToDevice, h->stream));
  // each launch runs at most kSolveUnroll iterations; the control block says
  // when the solve has stopped
  const int max_launches = max_iter / kSolveUnroll + 2;
  for (int launch = 0;; launch++) {
    RSO_CHECK_CUDA(h, cudaGraphLaunch(g->exec, h->stream));
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(c->h_ctl, c->ctl, sizeof(PcgCtl), cudaMemcpyDeviceToHost, h->stream));
    RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
    if (hc.done) break;
    if (launch + 1 >= max_launches) { h->err = "device-controlled PCG did not stop"; return RSO_ERR_STATE; }
  }
  note_launches(g->k_iter * hc.it + g->k_rep * hc.n_rep + g->k_cont * hc.n_cont);
  *it = hc.it;
  *rel = hc.rel;
  if (hc.status == PCG_NONFINITE) { h->err = "non-finite residual in PCG"; return RSO_ERR_NONFINITE; }
  *stalled = hc.status == PCG_STALLED;
  return RSO_OK;
}

static rso_status solve_pcg_k32(rso_handle* h, const double* f, double* x, double tol, int max_iter,
                                rso_solve_info* info, bool* stalled, int* used, bool x_zero) {
  Level& l0 = h->L[0];
  const long long n3 = 3 * l0.NP, n4 = n3 / 4;
  double* s = h->scal;  // s[0]=rz, s[1]=pq, s[2]=alpha, s[3]=rz_new, s[4]=beta, s[5]=rr
  float* r32 = l0.f32;  // the V-cycle's right-hand side (not rotated by the smoothers)
  // the V-cycle's result is L[0].u32, a pointer the Chebyshev and Jacobi
  // smoothers rotate: read it after every V-cycle
  float* p32 = reinterpret_cast<float*>(h->z);  // FP64 buffers unused by the mixed recurrence
  float* q32 = reinterpret_cast<float*>(h->q);
  if ((n3 & 3) || (reinterpret_cast<uintptr_t>(x) & 15)) {
    h->err = "reliable-update PCG: x must be 16-byte aligned";
    return RSO_ERR_INVALID_ARG;
  }
  auto true_residual = [&](double* rn2) -> rso_status {
    RSO_TRY(fine_residual<double>(h, x, f, h->r, h->rp64));
    return dot_host(h, h->r, h->r, n3, rn2);
  };
  // in a replacement: the true residual with its FP32 copy (the recurrence's
  // new r) and r . r from one pass; the padding of r32 keeps the zeros the
  // first copy gave it
  auto true_residual_rr = [&](double* rn2) -> rso_status {
    RSO_TRY(fine_residual64_rr(h, x, f, h->r, r32, h->scal + 15));
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(h->h_scal + 15, h->scal + 15, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
    *rn2 = h->h_scal[15];
    return RSO_OK;
  };
  double fn2 = 0, rn2 = 0;
  RSO_TRY(dot_host(h, f, f, n3, &fn2));
  // from a zero iterate the residual is f (the operator pass would give f
  // exactly: K 0 = 0 at every node); h->r is first needed at a replacement
  if (x_zero) rn2 = fn2;
  else RSO_TRY(true_residual(&rn2));
  const double fn = std::sqrt(fn2);
  int it = 0;
  double rel = fn > 0 ? std::sqrt(rn2) / fn : 0.0;
  if (fn == 0) {
    RSO_CHECK_CUDA(h, cudaMemsetAsync(x, 0, sizeof(double) * n3, h->stream));
    rel = 0;
  }
  *stalled = false;
  if (rel >= tol && fn > 0) {
    double rbase = std::sqrt(rn2);  // residual norm at the last replacement
    int since = 0;                  // iterations since then
    int cycles = 0;                 // replacements so far
    // the operator writes interior nodes only: the padding of q (an FP64
    // buffer seen as FP32, so old doubles split across its entries) must be zero
    RSO_CHECK_CUDA(h, cudaMemsetAsync(q32, 0, sizeof(float) * n3, h->stream));
    k_d2f<<<cdiv(n3, 256), 256, 0, h->stream>>>(x_zero ? f : h->r, r32, n3); rso::note_launch();
    // r . z comes out of the V-cycle's last fine step when it is a Jacobi or
    // Chebyshev step (after a post-smoothing), else from its own pass
    const bool fuse = h->cfg.smoother != RSO_SMOOTH_GS && h->cfg.post >= 1;
    struct ZdotReset {
      rso_handle* h;
      ~ZdotReset() { h->vc_zdot = nullptr; }
    } zreset{h};
    h->vc_zdot = fuse ? s + 0 : nullptr;
    RSO_TRY(vcycle_mixed(h));
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(p32, l0.u32, sizeof(float) * n3, cudaMemcpyDeviceToDevice, h->stream));
    if (!fuse) RSO_TRY(dot_ff(h, r32, l0.u32, n3, s + 0));
    h->vc_zdot = fuse ? s + 3 : nullptr;
    rso_status gs = RSO_ERR_UNSUPPORTED;
    if (h->solve_graphs && h->vc_graphs && !h->prof_on && h->stream && max_iter > 0)
      gs = pcg32_graph(h, f, x, tol, max_iter, fn, rbase, &it, &rel, stalled);
    if (gs != RSO_ERR_UNSUPPORTED) {
      RSO_TRY(gs);
      max_iter = 0;  // the loop below has run on the device
    }
    // one system: the FP64 steps wait in a ring of four FP32 directions (the
    // two halves of the FP64 buffers z and p) and enter x at the next
    // replacement or when the ring is full, so a step reads each direction
    // once more instead of x's 16 bytes per entry every iteration
    const bool defer = l0.nb == 1;
    float* ring[kStepRing] = {p32, p32 + n3, reinterpret_cast<float*>(h->p), reinterpret_cast<float*>(h->p) + n3};
    double* ring_alpha = h->scal + 40;
    int pend = 0;     // steps waiting: directions ring[0 .. pend), step sizes ring_alpha[0 .. pend)
    float* pc = p32;  // the current direction, ring[pend] until its step size is known
    auto flush = [&]() -> rso_status {
      if (pend == 0) return RSO_OK;
      StepRing R;
      for (int j = 0; j < kStepRing; j++) R.p[j] = reinterpret_cast<const float4*>(ring[j < pend ? j : 0]);
      k_cg32_flush<<<cdiv(n4, 256), 256, 0, h->stream>>>(n4, ring_alpha, R, pend, reinterpret_cast<double2*>(x));
      rso::note_launch();
      pend = 0;
      return launch_check(h, "pcg32 deferred steps");
    };
    while (it < max_iter) {
      RSO_TRY(fine_applyK_dot32(h, pc, q32, s + 1));
      if (defer) {
        k_cg_alpha_keep<<<1, 1, 0, h->stream>>>(s, ring_alpha + pend); rso::note_launch();
        pend++;
      } else {
        k_cg_alpha<<<1, 1, 0, h->stream>>>(s); rso::note_launch();
      }
      RSO_TRY(cg32_resid_rr(h, n3, s + 2, q32, r32, s + 5));
      RSO_CHECK_CUDA(h, cudaMemcpyAsync(h->h_scal + 5, s + 5, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
      RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
      vcycle_graphs_harvest(h);
      it++;
      since++;
      const double rnorm = std::sqrt(h->h_scal[5]);
      if (!std::isfinite(rnorm)) { h->err = "non-finite residual in PCG"; return RSO_ERR_NONFINITE; }
      const bool replace =
          rnorm < h->krylov32 * rbase || rnorm < tol * fn || it >= max_iter || since >= kCycleMax;
      if (replace) {
        if (defer) {
          RSO_TRY(flush());
        } else {
          k_cg32_step<<<cdiv(n4, 256), 256, 0, h->stream>>>(n4, s + 2, reinterpret_cast<const float4*>(pc),
                                                            reinterpret_cast<double2*>(x));
          rso::note_launch();
        }
        RSO_TRY(true_residual_rr(&rn2));
        const double rtrue = std::sqrt(rn2);
        rel = rtrue / fn;
        if (!std::isfinite(rel)) { h->err = "non-finite residual in PCG"; return RSO_ERR_NONFINITE; }
        if (rel < tol || it >= max_iter) break;
        cycles++;
        if (rtrue > stall_ratio(h->krylov32, rnorm / rbase) * rbase ||
            (h->krylov32_cycles > 0 && cycles >= h->krylov32_cycles)) {  // h->r holds the true residual of x
          *stalled = true;
          break;
        }
        rbase = rtrue;
        since = 0;
      } else {
        rel = rnorm / fn;
      }
      RSO_TRY(vcycle_mixed(h));
      const float* z32 = l0.u32;
      if (!fuse) RSO_TRY(dot_ff(h, r32, z32, n3, s + 3));
      k_cg_beta<<<1, 1, 0, h->stream>>>(s); rso::note_launch();
      if (defer) {
        if (pend == kStepRing) RSO_TRY(flush());
        float* pn = ring[pend];  // pc itself right after a flush of one step
        k_cg32_dir<<<cdiv(n4, 256), 256, 0, h->stream>>>(n4, s + 4, reinterpret_cast<const float4*>(z32),
                                                         reinterpret_cast<const float4*>(pc),
                                                         reinterpret_cast<float4*>(pn));
        pc = pn;
      } else if (replace) {
        k_cg32_step_dir<true><<<cdiv(n4, 256), 256, 0, h->stream>>>(
            n4, s + 2, s + 4, reinterpret_cast<const float4*>(z32), reinterpret_cast<float4*>(pc),
            reinterpret_cast<double2*>(x));
      } else {
        k_cg32_step_dir<false><<<cdiv(n4, 256), 256, 0, h->stream>>>(
            n4, s + 2, s + 4, reinterpret_cast<const float4*>(z32), reinterpret_cast<float4*>(pc),
            reinterpret_cast<double2*>(x));
      }
      rso::note_launch();
      RSO_TRY(launch_check(h, "pcg32"));
    }
  }
  *used = it;
  if (*stalled) return RSO_OK;
  RSO_TRY(displacement_project(h, x));  // support-free problems: no rigid motion in the solution
  RSO_TRY(fine_stage_check(h));
  if (info) { info->iterations = it; info->rel_res = rel; }
  if (rel >= tol && fn > 0) { h->err = "PCG did not reach the tolerance within max_iter"; return RSO_ERR_BUDGET_EXCEEDED; }
  return RSO_OK;
}

// CG preconditioned by one V-cycle.  In mixed precision the preconditioned
// residual z stays FP32 (it only enters r.z and the direction update), the
// FP32 copy of r is written by the fused residual update, and the norm of r
// comes out of the same pass.
rso_status solve_pcg(rso_handle* h, const double* f, double* x, double tol, int max_iter, rso_solve_info* info,
                     bool x_zero) {
  Level& l0 = h->L[0];
  const long long n3 = 3 * l0.NP;
  const bool mixed = h->cfg.precision == RSO_MIXED;
  int used = 0;  // iterations of an FP32 recurrence that stalled
  if (mixed && h->krylov32 > 0 && l0.nb == 1) {
    bool stalled = false;
    const rso_status st = solve_pcg_k32(h, f, x, tol, max_iter, info, &stalled, &used, x_zero);
    if (st != RSO_OK || !stalled) return st;
    max_iter -= used;  // the FP64 recurrence from the current iterate for the rest
  }
  // q may hold FP32 words of an earlier FP32 recurrence, and the operator
  // writes interior nodes only while the residual update reads every entry
  if (mixed) RSO_CHECK_CUDA(h, cudaMemsetAsync(h->q, 0, sizeof(double) * n3, h->stream));
  double* s = h->scal;
  RSO_TRY(fine_residual<double>(h, x, f, h->r, h->rp64));
  double fn2 = 0, rn2 = 0;
  RSO_TRY(dot_host(h, f, f, n3, &fn2));
  RSO_TRY(dot_host(h, h->r, h->r, n3, &rn2));
  const double fn = std::sqrt(fn2);
  int it = 0;
  double rel = fn > 0 ? std::sqrt(rn2) / fn : 0.0;
  if (fn == 0) {
    RSO_CHECK_CUDA(h, cudaMemsetAsync(x, 0, sizeof(double) * n3, h->stream));
    rel = 0;
  }
  if (rel >= tol && fn > 0) {
    if (mixed) {
      k_d2f<<<cdiv(n3, 256), 256, 0, h->stream>>>(h->r, h->L[0].f32, n3); rso::note_launch();
      RSO_TRY(vcycle_mixed(h));
      k_f2d<<<cdiv(n3, 256), 256, 0, h->stream>>>(h->L[0].u32, h->p, n3); rso::note_launch();
      RSO_TRY(dot_df(h, h->r, h->L[0].u32, n3, s + 0));
    } else {
      RSO_TRY(precondition(h, h->r, h->z));
      RSO_CHECK_CUDA(h, cudaMemcpyAsync(h->p, h->z, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->stream));
      RSO_TRY(dot(h, h->r, h->z, n3, s + 0));
    }
    while (it < max_iter) {
      RSO_TRY(fine_applyK_dot(h, h->p, h->q, h->rp64, s + 1));
      k_cg_alpha<<<1, 1, 0, h->stream>>>(s); rso::note_launch();
      RSO_TRY(cg_resid_rr(h, n3, s + 2, h->q, h->r, mixed ? h->L[0].f32 : nullptr, s + 5));
      RSO_CHECK_CUDA(h, cudaMemcpyAsync(h->h_scal + 5, s + 5, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
      RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
      vcycle_graphs_harvest(h);
      rn2 = h->h_scal[5];
      it++;
      rel = std::sqrt(rn2) / fn;
      if (!std::isfinite(rel)) { h->err = "non-finite residual in PCG"; return RSO_ERR_NONFINITE; }
      if (rel < tol || it >= max_iter) {
        k_cg_step<<<cdiv(n3, 256), 256, 0, h->stream>>>(n3, s + 2, h->p, x); rso::note_launch();
        break;
      }
      if (mixed) {
        RSO_TRY(vcycle_mixed(h));
        RSO_TRY(dot_df(h, h->r, h->L[0].u32, n3, s + 3));
        k_cg_beta<<<1, 1, 0, h->stream>>>(s); rso::note_launch();
        k_cg_step_dir<float><<<cdiv(n3, 256), 256, 0, h->stream>>>(n3, s + 2, s + 4, h->L[0].u32, h->p, x); rso::note_launch();
      } else {
        RSO_TRY(precondition(h, h->r, h->z));
        RSO_TRY(dot(h, h->r, h->z, n3, s + 3));
        k_cg_beta<<<1, 1, 0, h->stream>>>(s); rso::note_launch();
        k_cg_step_dir<double><<<cdiv(n3, 256), 256, 0, h->stream>>>(n3, s + 2, s + 4, h->z, h->p, x); rso::note_launch();
      }
      RSO_TRY(launch_check(h, "pcg"));
    }
  }
  RSO_TRY(displacement_project(h, x));
  RSO_TRY(fine_stage_check(h));
  if (info) { info->iterations = it + used; info->rel_res = rel; }
  if (rel >= tol && fn > 0) { h->err = "PCG did not reach the tolerance within max_iter"; return RSO_ERR_BUDGET_EXCEEDED; }
  return RSO_OK;
}

// x <- x + M (f - K x) repeated (defect correction; plain V-cycles in FP64 mode)
rso_status solve_vcycles(rso_handle* h, const double* f, double* x, double tol, int max_iter, rso_solve_info* info) {
  Level& l0 = h->L[0];
  const long long n3 = 3 * l0.NP;
  double fn2 = 0, rn2 = 0;
  RSO_TRY(dot_host(h, f, f, n3, &fn2));
  const double fn = std::sqrt(fn2);
  int it = 0;
  double rel = 0;
  RSO_TRY(fine_residual<double>(h, x, f, h->r, h->rp64));
  RSO_TRY(dot_host(h, h->r, h->r, n3, &rn2));
  rel = fn > 0 ? std::sqrt(rn2) / fn : 0;
  while (rel >= tol && it < max_iter && fn > 0) {
    RSO_TRY(precondition(h, h->r, h->z));
    RSO_TRY(axpby(h, n3, 1.0, h->z, 1.0, x));
    RSO_TRY(fine_residual<double>(h, x, f, h->r, h->rp64));
    RSO_TRY(dot_host(h, h->r, h->r, n3, &rn2));
    rel = std::sqrt(rn2) / fn;
    it++;
    if (!std::isfinite(rel) || rel > 1e4) { h->err = "defect correction diverged"; return RSO_ERR_DIVERGED; }
  }
  RSO_TRY(displacement_project(h, x));
  RSO_TRY(fine_stage_check(h));
  if (info) { info->iterations = it; info->rel_res = rel; }
  if (rel >= tol && fn > 0) { h->err = "V-cycle iteration did not reach the tolerance"; return RSO_ERR_BUDGET_EXCEEDED; }
  return RSO_OK;
}

// reference-sequenced FP64 V-cycle on a caller iterate (padded vectors)
rso_status vcycle_fp64(rso_handle* h, double* u, const double* f, int pre, int post, int symmetric, double* rel) {
  Level& l0 = h->L[0];
  const long long n3 = 3 * l0.NP;
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(l0.u64, u, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->stream));
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(l0.f64, f, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->stream));
  RSO_TRY(vcycle_levels<double>(h, pre, post, symmetric, false));
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(u, h->L[0].u64, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->stream));
  RSO_TRY(fine_residual<double>(h, u, f, h->r, h->rp64));
  double rn2 = 0, fn2 = 0;
  RSO_TRY(dot_host(h, h->r, h->r, n3, &rn2));
  RSO_TRY(dot_host(h, f, f, n3, &fn2));
  if (rel) *rel = fn2 > 0 ? std::sqrt(rn2 / fn2) : std::sqrt(rn2);
  return RSO_OK;
}

}  // namespace rso
