// Surface-point self-support (deal_surface_points,
// optimization/optimization.cpp:1185-1221): the iso-surface rho = 0.5 of the
// spline design sampled on a background grid, and the overhang constraint
// with its coefficient gradient evaluated at the samples.
//
// Sampling (generate_spline_surface_nodes, grid/Grid.cpp:4067-4112):
//   1. k_mc_values: the spline minus 0.5 at the (mc + 2)^3 cell centres of
//      the model box enlarged by one cell, 0 - 0.5 outside the box
//      (Grid::compute_background_mcPoints_value, grid/Grid.cu:4066-4175);
//   2. the grid edges whose end values straddle 0 (a corner counts as inside
//      at <= 0, marchingcube/MarchingCube.cpp:104-107) compacted in edge order
//      (grid point x fastest, then y, z; then the axis);
//   3. the reference's thinning (Grid::compute_surface_nodes_in_model,
//      grid/Grid.cpp:3861-4060): an equal-distance pick of 3 n edges when there
//      are more than 2 n per requested point, their crossings (linear
//      interpolation from the lower corner, MarchingCube.cpp:23-31) kept when
//      they lie inside an active element, then a final equal-distance pick of
//      n, padded with the first point when fewer remain, or n points at the
//      origin when none remain (generateEquidistantIntegers, :3831-3847,
//      picks clamped to the list).
//   Each step is an order-preserving compaction: per-CTA counts, one scan of
//   the counts, and a second pass that writes each kept entry at its rank.
//
// Constraint (grid/Grid.cu:5709-6505, grid/Grid.cpp:4263-4280):
//   k_surf_eval   normal = spline gradient at the point, orientation probe
//                 1e-3 along it (void there: +1, else -1);
//   k_surf_value  normals flipped when the probes sum below 0; overhang flags
//                 at the default and the optimisation angle; per-point penalty
//                 of the mode (p-norm 8, h-function 10, sigmoid 0.09,
//                 grid/Grid.h:371-375) and the per-point weights of its
//                 derivative with respect to the normal;
//   k_surf_grad   the chain to the 4x4x4 (order^3) coefficients around each
//                 point, accumulated with FP64 atomics and divided by the
//                 count (points with n_z < 0 in the even modes, all points in
//                 the odd ones).
//   The reference's gradient kernel adds into the coefficient array without
//   atomics from every point at once; here the additions are atomic.  A point
//   whose normal is zero (outside the knot support) contributes nothing.
//
// The spline arithmetic runs in FP64 with explicitly rounded operations, so
// the background values and crossing coordinates follow the CPU oracle's
// operation order exactly.
#include "rso_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace rso {

namespace {

constexpr int SC_THREADS = 256;                 // compaction CTA; each thread takes PT consecutive entries
constexpr int SP_THREADS = 256;                 // per-point kernels

struct SplineP {
  int order, nb[3];
  float bmin[3], step[3];
  const float* kn[3];
};

struct MCGrid {
  int n;            // points per axis (mc + 2)
  float lo[3], hi[3], eh[3];
};

// spline basis values (and first derivatives) at coordinate u of axis a
// (Cox-de Boor, Piegl-Tiller A2.2/A2.3: the recursion of SplineBasisDeriX,
// grid/Grid.cu:514-610); the span index in float as the reference forms it
__device__ bool basis_vd(const SplineP& S, int a, double u, int* I, double* N, double* dN) {
  const int o = S.order, p = o - 1;
  const float pf = __double2float_rn(u);
  const int i = (int)__fdiv_rn(__fsub_rn(pf, S.bmin[a]), S.step[a]) + o;
  *I = i;
  if (i < o || i > S.nb[a]) return false;
  const int span = i - 1;
  const float* K = S.kn[a];
  double ndu[5][5], left[5], right[5];
  ndu[0][0] = 1.0;
  for (int j = 1; j <= p; j++) {
    left[j] = __dsub_rn(u, (double)K[span + 1 - j]);
    right[j] = __dsub_rn((double)K[span + j], u);
    double saved = 0.0;
    for (int r = 0; r < j; r++) {
      ndu[j][r] = __dadd_rn(right[r + 1], left[j - r]);
      const double temp = __ddiv_rn(ndu[r][j - 1], ndu[j][r]);
      ndu[r][j] = __dadd_rn(saved, __dmul_rn(right[r + 1], temp));
      saved = __dmul_rn(left[j - r], temp);
    }
    ndu[j][j] = saved;
  }
  for (int j = 0; j <= p; j++) N[j] = ndu[j][p];
  if (dN)
    for (int r = 0; r <= p; r++) {
      double d = 0;
      if (p >= 1) {
        if (r >= 1) d = __ddiv_rn(ndu[r - 1][p - 1], ndu[p][r - 1]);
        if (r <= p - 1) d = __dsub_rn(d, __ddiv_rn(ndu[r][p - 1], ndu[p][r]));
        d = __dmul_rn(d, (double)p);
      }
      dN[r] = d;
    }
  return true;
}

__device__ __forceinline__ long long cidx(const SplineP& S, int a, int b, int q) {
  return a + (long long)b * S.nb[0] + (long long)q * S.nb[0] * S.nb[1];
}

// spline value (and gradient when g != nullptr) at a point; false outside the support
__device__ bool spline_at(const SplineP& S, const double* __restrict__ c, const double pt[3], double* v, double* g) {
  const int o = S.order;
  int I[3];
  double N[3][5], D[3][5];
  for (int a = 0; a < 3; a++)
    if (!basis_vd(S, a, pt[a], &I[a], N[a], g ? D[a] : nullptr)) return false;
  double s = 0, g0 = 0, g1 = 0, g2 = 0;
  for (int q = 0; q < o; q++)
    for (int b = 0; b < o; b++)
      for (int a = 0; a < o; a++) {
        const double cc = c[cidx(S, I[0] - o + a, I[1] - o + b, I[2] - o + q)];
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(__dmul_rn(cc, N[0][a]), N[1][b]), N[2][q]));
        if (g) {
          g0 = __dadd_rn(g0, __dmul_rn(__dmul_rn(__dmul_rn(cc, D[0][a]), N[1][b]), N[2][q]));
          g1 = __dadd_rn(g1, __dmul_rn(__dmul_rn(__dmul_rn(cc, N[0][a]), D[1][b]), N[2][q]));
          g2 = __dadd_rn(g2, __dmul_rn(__dmul_rn(__dmul_rn(cc, N[0][a]), N[1][b]), D[2][q]));
        }
      }
  *v = s;
  if (g) { g[0] = g0; g[1] = g1; g[2] = g2; }
  return true;
}

// cell centre x of one axis: boxOrispan + x * eh + 0.5 * eh (float, then the
// half step in double, as grid/Grid.cu:4114 writes it)
__device__ __forceinline__ float mc_coord(float lo, float eh, int x) {
  const float t = __fadd_rn(__fsub_rn(lo, eh), __fmul_rn((float)x, eh));
  return __double2float_rn(__dadd_rn((double)t, 0.5 * (double)eh));
}

__global__ void __launch_bounds__(SP_THREADS) k_mc_values(SplineP S, const double* __restrict__ c, MCGrid G,
                                                          float* __restrict__ val) {
  const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n3 = (long long)G.n * G.n * G.n;
  if (id >= n3) return;
  const int ix[3] = {(int)(id % G.n), (int)(id / G.n % G.n), (int)(id / ((long long)G.n * G.n))};
  double pt[3];
  bool outside_box = false;
  for (int a = 0; a < 3; a++) {
    const float p = mc_coord(G.lo[a], G.eh[a], ix[a]);
    outside_box |= p < G.lo[a] || p > G.hi[a];
    pt[a] = (double)p;
  }
  double v;
  float vf = spline_at(S, c, pt, &v, nullptr) ? __double2float_rn(v) : -0.2f;
  if (outside_box) vf = 0.f;
  val[id] = __double2float_rn(__dsub_rn((double)vf, 0.5));
}

// ---------------------------------------------------------------- compaction
__device__ __forceinline__ unsigned block_excl_scan(unsigned v, unsigned* total) {
  __shared__ unsigned wsum[SC_THREADS / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    unsigned s = lane < SC_THREADS / 32 ? wsum[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < SC_THREADS / 32) wsum[lane] = s;
  }
  __syncthreads();
  const unsigned before = (w > 0 ? wsum[w - 1] : 0u) + x - v;
  if (total) *total = wsum[SC_THREADS / 32 - 1];
  __syncthreads();
  return before;
}

template <class P, int PT>
__global__ void __launch_bounds__(SC_THREADS) k_sc_count(P pred, long long n, unsigned* __restrict__ cnt) {
  const long long base = blockIdx.x * (long long)(SC_THREADS * PT) + (long long)threadIdx.x * PT;
  unsigned k = 0;
  for (int i = 0; i < PT; i++)
    if (base + i < n && pred(base + i)) k++;
  unsigned total;
  block_excl_scan(k, &total);
  if (threadIdx.x == 0) cnt[blockIdx.x] = total;
}

// exclusive scan of nb CTA counts in place; the total lands in cnt[nb]
__global__ void __launch_bounds__(SC_THREADS) k_sc_scan(unsigned* __restrict__ cnt, int nb) {
  const int per = (nb + SC_THREADS - 1) / SC_THREADS;
  const int b0 = threadIdx.x * per;
  unsigned s = 0;
  for (int i = 0; i < per; i++)
    if (b0 + i < nb) s += cnt[b0 + i];
  unsigned total;
  unsigned run = block_excl_scan(s, &total);
  for (int i = 0; i < per; i++)
    if (b0 + i < nb) {
      const unsigned c = cnt[b0 + i];
      cnt[b0 + i] = run;
      run += c;
    }
  if (threadIdx.x == 0) cnt[nb] = total;
}

template <class P, class E, int PT>
__global__ void __launch_bounds__(SC_THREADS) k_sc_emit(P pred, E emit, long long n, const unsigned* __restrict__ off) {
  static_assert(PT <= 32, "one flag bit per entry");
  const long long base = blockIdx.x * (long long)(SC_THREADS * PT) + (long long)threadIdx.x * PT;
  unsigned flags = 0, k = 0;
  for (int i = 0; i < PT; i++)
    if (base + i < n && pred(base + i)) { flags |= 1u << i; k++; }
  unsigned pos = off[blockIdx.x] + block_excl_scan(k, nullptr);
  for (int i = 0; i < PT; i++)
    if (flags >> i & 1u) emit(pos++, base + i);
}

// crossing of the edge e = 3 g + axis between grid point g and g + e_axis
struct EdgePred {
  const float* val;
  int n;
  __device__ bool operator()(long long e) const {
    const long long g = e / 3;
    const int a = (int)(e - 3 * g);
    const int ix[3] = {(int)(g % n), (int)(g / n % n), (int)(g / ((long long)n * n))};
    if (ix[a] + 1 >= n) return false;
    const long long st = a == 0 ? 1 : (a == 1 ? n : (long long)n * n);
    return (val[g] <= 0.f) != (val[g + st] <= 0.f);
  }
};

struct EdgeEmit {
  unsigned* out;
  __device__ void operator()(unsigned pos, long long e) const { out[pos] = (unsigned)e; }
};

__device__ __forceinline__ void crossing(const MCGrid& G, const float* __restrict__ val, unsigned e, float p[3]) {
  const long long g = e / 3;
  const int a = (int)(e - 3 * g);
  const int ix[3] = {(int)(g % G.n), (int)(g / G.n % G.n), (int)(g / ((long long)G.n * G.n))};
  for (int b = 0; b < 3; b++) p[b] = mc_coord(G.lo[b], G.eh[b], ix[b]);
  const long long st = a == 0 ? 1 : (a == 1 ? G.n : (long long)G.n * G.n);
  const float v1 = val[g], v2 = val[g + st];
  if (fabsf(__fsub_rn(v1, v2)) > 0.00001f) {
    const float p2 = mc_coord(G.lo[a], G.eh[a], ix[a] + 1);
    const float t = __fdiv_rn(__fsub_rn(p2, p[a]), __fsub_rn(v2, v1));
    p[a] = __fadd_rn(p[a], __fmul_rn(t, __fsub_rn(0.f, v1)));
  }
}

__device__ __forceinline__ bool in_model(const Level& L, const float p[3]) {
  const int dims[3] = {L.ex, L.ey, L.ez};
  int e[3];
  for (int b = 0; b < 3; b++) {
    const float f = floorf(p[b]);
    if (!(f >= 0.f && f < (float)dims[b])) return false;
    e[b] = (int)f;
  }
  return L.emask[L.eidx(e[0], e[1], e[2])] != 0;
}

// j-th of m equal-distance picks from a list of `range` (clamped; m >= range: j)
__device__ __forceinline__ long long equi(long long j, long long range, long long m) {
  if (m >= range) return j;
  const double step = m > 1 ? (double)range / (double)(m - 1) : 0.0;
  const long long k = (long long)__dmul_rn((double)j, step);
  return k < range - 1 ? k : range - 1;
}

// candidate j of the first pick (all edges when the list is not thinned)
struct PickPred {
  Level L;
  MCGrid G;
  const float* val;
  const unsigned* edges;
  long long num, m1;
  __device__ bool operator()(long long j) const {
    float p[3];
    crossing(G, val, edges[equi(j, num, m1)], p);
    return in_model(L, p);
  }
};

struct PickEmit {
  MCGrid G;
  const float* val;
  const unsigned* edges;
  long long num, m1;
  float* out;        // SoA x, y, z with stride cap
  long long cap;
  __device__ void operator()(unsigned pos, long long j) const {
    float p[3];
    crossing(G, val, edges[equi(j, num, m1)], p);
    out[pos] = p[0];
    out[cap + pos] = p[1];
    out[2 * cap + pos] = p[2];
  }
};

__global__ void k_final_pick(const float* __restrict__ kept, long long cap, long long nk, int npts,
                             float* __restrict__ xyz) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= npts) return;
  float p[3] = {0.f, 0.f, 0.f};
  if (nk > 0) {
    const long long s = nk >= npts ? equi(j, nk, npts) : (j < nk ? j : 0);
    for (int b = 0; b < 3; b++) p[b] = kept[b * cap + s];
  }
  for (int b = 0; b < 3; b++) xyz[(long long)b * npts + j] = p[b];
}

// ---------------------------------------------------------------- constraint
__device__ __forceinline__ double heav(double s, double beta) {
  const double eta = 0.5;
  return (tanh(beta * eta) + tanh(beta * (s - eta))) / (tanh(beta * eta) + tanh(beta * (1 - eta)));
}

__global__ void __launch_bounds__(SP_THREADS) k_surf_eval(SplineP S, const double* __restrict__ c,
                                                          const float* __restrict__ xyz, int n, double beta,
                                                          double* __restrict__ nrm, uint8_t* __restrict__ ins,
                                                          float* __restrict__ dir) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double pt[3] = {(double)xyz[k], (double)xyz[n + k], (double)xyz[2 * n + k]};
  double v, g[3] = {0, 0, 0};
  const bool in = spline_at(S, c, pt, &v, g);
  if (!in) g[0] = g[1] = g[2] = 0;
  for (int a = 0; a < 3; a++) nrm[(long long)a * n + k] = g[a];
  ins[k] = in;
  // orientation probe 1e-3 along the unnormalised gradient (grid/Grid.cu:5810-5870)
  const double pd[3] = {__dadd_rn(pt[0], __dmul_rn(1e-3, g[0])), __dadd_rn(pt[1], __dmul_rn(1e-3, g[1])),
                        __dadd_rn(pt[2], __dmul_rn(1e-3, g[2]))};
  double vd;
  if (!spline_at(S, c, pd, &vd, nullptr)) vd = -0.1;
  dir[k] = heav(vd, beta) < 0.5 ? 1.f : -1.f;
}

struct SurfPar {
  int mode;
  double cosang, cosdef;
};

__device__ __forceinline__ void surf_pen(int m, double inner, double* f, double* df) {
  if (m <= 1) {
    *f = pow(inner, 8.0);
    *df = 8.0 * pow(inner, 7.0);
  } else if (m <= 3) {
    *f = inner >= 1 ? 10.0 * (inner - 1) * (inner - 1) : 0;
    *df = inner >= 1 ? 20.0 * (inner - 1) : 0;
  } else {
    const double cc = 0.09, e = exp(-(inner - 1.5) / cc);
    *f = 1 / (1 + e);
    *df = 1 / (1 + e) / (1 + e) / cc * e;
  }
}

// dirsum: the probe sum on the device (flip when < 0, derivative sign +1 when > 0)
__global__ void __launch_bounds__(SP_THREADS) k_surf_value(int n, double* __restrict__ nrm,
                                                           const uint8_t* __restrict__ ins,
                                                           const double* __restrict__ dirsum, SurfPar P,
                                                           double* __restrict__ per, float* __restrict__ per_f,
                                                           uint8_t* __restrict__ flags, float* __restrict__ down,
                                                           double* __restrict__ w) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double ds = *dirsum;
  const double flip = ds < 0 ? -1.0 : 1.0, direction = ds > 0 ? 1.0 : -1.0;
  double q[3];
  for (int a = 0; a < 3; a++) {
    q[a] = flip * nrm[(long long)a * n + k];
    nrm[(long long)a * n + k] = q[a];
  }
  const double nn = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(q[0], q[0]), __dmul_rn(q[1], q[1])), __dmul_rn(q[2], q[2])));
  const bool dn = q[2] < 0;
  const bool on = nn > 0 && (P.mode % 2 == 1 || dn);
  double f = 0, df = 0;
  if (on) surf_pen(P.mode, q[2] / nn / P.cosang, &f, &df);
  per[k] = f;
  if (per_f) per_f[k] = (float)f;
  down[k] = dn ? 1.f : 0.f;
  flags[k] = (dn && nn > 0 && q[2] / nn / P.cosdef > 1) ? 1 : 0;
  flags[n + k] = (dn && nn > 0 && q[2] / nn / P.cosang > 1) ? 1 : 0;
  // d inner / d normal = (nn e_z - q_z q / nn) / (nn^2 cos)
  double wv[3] = {0, 0, 0};
  if (on && ins[k]) {
    const double s = direction * df / (nn * nn * P.cosang);
    for (int a = 0; a < 3; a++) wv[a] = s * ((a == 2 ? nn : 0.0) - q[2] * q[a] / nn);
  }
  for (int a = 0; a < 3; a++) w[(long long)a * n + k] = wv[a];
}

__global__ void __launch_bounds__(SP_THREADS) k_sumd_partial(const double* __restrict__ a, long long n,
                                                             double* __restrict__ part) {
  __shared__ double ws[SP_THREADS / 32];
  double s = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s += a[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int i = 0; i < SP_THREADS / 32; i++) t += ws[i];
    part[blockIdx.x] = t;
  }
}

// dc += w . (dN N N, N dN N, N N dN) / count over the order^3 coefficients of each point
// dc += w . (dN N N, N dN N, N N dN) / count over the order^3 coefficients of
// each point.  A warp whose points all fall in the same knot cell (a run of
// nearby samples, or the copies of the first point that pad a short list)
// sums its contributions with shuffles and adds each once; other warps add
// per point.
__global__ void __launch_bounds__(SP_THREADS) k_surf_grad(SplineP S, const float* __restrict__ xyz, int n,
                                                          const double* __restrict__ w,
                                                          const double* __restrict__ down_sum, int mode,
                                                          double* __restrict__ dc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  bool has = k < n;
  double w0 = 0, w1 = 0, w2 = 0;
  if (has) {
    w0 = w[k]; w1 = w[n + k]; w2 = w[2 * (long long)n + k];
    has = !(w0 == 0 && w1 == 0 && w2 == 0);
  }
  const int o = S.order;
  int I[3] = {0, 0, 0};
  double N[3][5] = {}, D[3][5] = {};
  if (has) {
    const double pt[3] = {(double)xyz[k], (double)xyz[n + k], (double)xyz[2 * n + k]};
    for (int a = 0; a < 3 && has; a++) has = basis_vd(S, a, pt[a], &I[a], N[a], D[a]);
  }
  const double cnt = mode % 2 == 0 ? *down_sum : (double)n;
  const double scale = cnt == 0 ? 0.0 : 1.0 / cnt;
  const long long key = has ? cidx(S, I[0], I[1], I[2]) : -1;
  const long long key0 = __shfl_sync(0xffffffffu, key, 0);
  const bool uniform = __all_sync(0xffffffffu, key == key0) && key0 >= 0;
  for (int q = 0; q < o; q++)
    for (int b = 0; b < o; b++) {
      const double nyz = N[1][b] * N[2][q];
      const double t1 = w1 * D[1][b] * N[2][q] + w2 * N[1][b] * D[2][q];
      for (int a = 0; a < o; a++) {
        double v = has ? scale * (w0 * D[0][a] * nyz + N[0][a] * t1) : 0.0;
        const long long ci = cidx(S, I[0] - o + a, I[1] - o + b, I[2] - o + q);
        if (uniform) {
#pragma unroll
          for (int sh = 16; sh > 0; sh >>= 1) v += __shfl_xor_sync(0xffffffffu, v, sh);
          if (lane == 0) atomicAdd(&dc[ci], v);
        } else if (has) {
          atomicAdd(&dc[ci], v);
        }
      }
    }
}

__global__ void k_f2d_c(const float* __restrict__ a, double* __restrict__ b, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (double)a[i];
}
__global__ void k_d2f_c(const double* __restrict__ a, float* __restrict__ b, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

}  // namespace

// state kept on the handle between calls; buffers grow, never shrink
struct SurfState {
  int n = 0, cap = 0;                 // points, capacity
  float* xyz = nullptr;               // SoA, stride n
  double* nrm = nullptr;              // outward normals, SoA stride n
  double* w = nullptr;                // derivative weights, SoA stride n
  double* per = nullptr;
  float* dir = nullptr;
  float* down = nullptr;
  uint8_t* ins = nullptr;
  uint8_t* flags = nullptr;           // actual (n), virtual (n)
  long long mc_cap = 0, edge_cap = 0, kept_cap = 0, cnt_cap = 0;
  float* mcval = nullptr;
  unsigned* edges = nullptr;
  float* kept = nullptr;              // SoA stride kept_cap
  unsigned* cnt = nullptr;            // CTA counts + total
  double* scal = nullptr;             // probe sum, penalty sum, down count
  double* h_scal = nullptr;           // pinned mirror
  unsigned* h_cnt = nullptr;
  bool have_box = false;              // bounding box of the active elements
  float box[6];
};

static SurfState* surf(rso_handle* h) {
  if (!h->surf) h->surf = new SurfState();
  return (SurfState*)h->surf;
}

void surface_free(rso_handle* h) {
  SurfState* s = (SurfState*)h->surf;
  if (!s) return;
  cudaFree(s->xyz); cudaFree(s->nrm); cudaFree(s->w); cudaFree(s->per); cudaFree(s->dir); cudaFree(s->down);
  cudaFree(s->ins); cudaFree(s->flags); cudaFree(s->mcval); cudaFree(s->edges); cudaFree(s->kept);
  cudaFree(s->cnt); cudaFree(s->scal);
  if (s->h_scal) cudaFreeHost(s->h_scal);
  if (s->h_cnt) cudaFreeHost(s->h_cnt);
  delete s;
  h->surf = nullptr;
}

template <class T>
static rso_status grow(rso_handle* h, T** p, long long* cap, long long need, long long per_entry = 1) {
  if (need <= *cap) return RSO_OK;
  cudaFree(*p);
  *p = nullptr;
  RSO_CHECK_CUDA(h, cudaMalloc((void**)p, sizeof(T) * (size_t)(need * per_entry)));
  *cap = need;
  return RSO_OK;
}

static rso_status points_reserve(rso_handle* h, int n) {
  SurfState* s = surf(h);
  if (!s->scal) {
    RSO_CHECK_CUDA(h, cudaMalloc((void**)&s->scal, 8 * sizeof(double)));
    RSO_CHECK_CUDA(h, cudaMallocHost((void**)&s->h_scal, 8 * sizeof(double)));
    RSO_CHECK_CUDA(h, cudaMallocHost((void**)&s->h_cnt, 4 * sizeof(unsigned)));
  }
  if (n <= s->cap) return RSO_OK;
  cudaFree(s->xyz); cudaFree(s->nrm); cudaFree(s->w); cudaFree(s->per); cudaFree(s->dir); cudaFree(s->down);
  cudaFree(s->ins); cudaFree(s->flags);
  s->xyz = nullptr; s->nrm = nullptr; s->w = nullptr; s->per = nullptr; s->dir = nullptr; s->down = nullptr;
  s->ins = nullptr; s->flags = nullptr;
  s->cap = 0;
  RSO_CHECK_CUDA(h, cudaMalloc((void**)&s->xyz, sizeof(float) * 3 * (size_t)n));
  RSO_CHECK_CUDA(h, cudaMalloc((void**)&s->nrm, sizeof(double) * 3 * (size_t)n));
  RSO_CHECK_CUDA(h, cudaMalloc((void**)&s->w, sizeof(double) * 3 * (size_t)n));
  RSO_CHECK_CUDA(h, cudaMalloc((void**)&s->per, sizeof(double) * (size_t)n));
  RSO_CHECK_CUDA(h, cudaMalloc((void**)&s->dir, sizeof(float) * (size_t)n));
  RSO_CHECK_CUDA(h, cudaMalloc((void**)&s->down, sizeof(float) * (size_t)n));
  RSO_CHECK_CUDA(h, cudaMalloc((void**)&s->ins, (size_t)n));
  RSO_CHECK_CUDA(h, cudaMalloc((void**)&s->flags, 2 * (size_t)n));
  s->cap = n;
  return RSO_OK;
}

static SplineP spline_p(const rso_handle* h) {
  const Spline& sp = h->sp;
  SplineP S;
  S.order = sp.order;
  size_t off = 0;
  for (int a = 0; a < 3; a++) {
    S.nb[a] = sp.nb[a];
    S.bmin[a] = sp.bmin[a];
    S.step[a] = sp.step[a];
    S.kn[a] = sp.knots_dev + off;
    off += sp.knots[a].size();
  }
  return S;
}

// order-preserving compaction of [0, n) under pred, PT entries per thread;
// returns the kept count
template <int PT, class P, class E>
static rso_status compact(rso_handle* h, P pred, E emit, long long n, long long* kept) {
  SurfState* s = surf(h);
  const long long nb = (n + SC_THREADS * PT - 1) / (SC_THREADS * PT);
  *kept = 0;
  if (nb == 0) return RSO_OK;
  RSO_TRY(grow(h, &s->cnt, &s->cnt_cap, nb + 1));
  k_sc_count<P, PT><<<(int)nb, SC_THREADS, 0, h->stream>>>(pred, n, s->cnt); note_launch();
  k_sc_scan<<<1, SC_THREADS, 0, h->stream>>>(s->cnt, (int)nb); note_launch();
  k_sc_emit<P, E, PT><<<(int)nb, SC_THREADS, 0, h->stream>>>(pred, emit, n, s->cnt); note_launch();
  RSO_TRY(launch_check(h, "surface compaction"));
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(s->h_cnt, s->cnt + nb, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  *kept = s->h_cnt[0];
  return RSO_OK;
}

// computed once per handle (the element mask does not change after rso_create)
void active_box(rso_handle* h, float box[6]) {
  SurfState* s = surf(h);
  if (!s->have_box) {
    const Level& l = h->L[0];
    int lo[3] = {l.ex, l.ey, l.ez}, hi[3] = {-1, -1, -1};
    const int dims[3] = {l.ex, l.ey, l.ez};
    const uint8_t* m = h->h_emask[0].data();
    for (int z = 0; z < l.ez; z++)
      for (int y = 0; y < l.ey; y++, m += l.ex) {
        int x0 = 0, x1 = l.ex - 1;
        while (x0 < l.ex && !m[x0]) x0++;
        if (x0 == l.ex) continue;
        while (!m[x1]) x1--;
        lo[0] = std::min(lo[0], x0); hi[0] = std::max(hi[0], x1);
        lo[1] = std::min(lo[1], y); hi[1] = std::max(hi[1], y);
        lo[2] = std::min(lo[2], z); hi[2] = std::max(hi[2], z);
      }
    for (int a = 0; a < 3; a++) {
      if (hi[a] < 0) { lo[a] = 0; hi[a] = dims[a] - 1; }
      s->box[a] = (float)lo[a];
      s->box[3 + a] = (float)(hi[a] + 1);
    }
    s->have_box = true;
  }
  std::memcpy(box, s->box, sizeof(float) * 6);
}

rso_status surface_points(rso_handle* h, const double* c, int mc, int npts, const float* box,
                          rso_surface_info* info) {
  SurfState* s = surf(h);
  const Level& l = h->L[0];
  MCGrid G;
  G.n = mc + 2;
  for (int a = 0; a < 3; a++) {
    G.lo[a] = box[a];
    G.hi[a] = box[3 + a];
    G.eh[a] = (box[3 + a] - box[a]) / (float)mc;
  }
  const long long n3 = (long long)G.n * G.n * G.n;
  if (3 * n3 >= (1ll << 32)) { h->err = "background grid too large"; return RSO_ERR_INVALID_ARG; }
  RSO_TRY(points_reserve(h, npts));
  RSO_TRY(grow(h, &s->mcval, &s->mc_cap, n3));
  const SplineP S = spline_p(h);
  k_mc_values<<<cdiv(n3, SP_THREADS), SP_THREADS, 0, h->stream>>>(S, c, G, s->mcval); note_launch();
  RSO_TRY(launch_check(h, "mc_values"));
  // crossing edges, in edge order
  RSO_TRY(grow(h, &s->edges, &s->edge_cap, 3 * n3));
  long long num = 0;
  // 16 edges per thread (cheap tests), 2 candidates per thread in the pick (a crossing each)
  RSO_TRY(compact<16>(h, EdgePred{s->mcval, G.n}, EdgeEmit{s->edges}, 3 * n3, &num));
  // first pick (3 npts of them when there are more than 2 npts per point), inside the model
  const bool thin = npts > 0 && num / npts > 2;
  const long long m1 = thin ? std::min<long long>(3ll * npts, num) : num;
  RSO_TRY(grow(h, &s->kept, &s->kept_cap, std::max<long long>(m1, 1), 3));
  long long nk = 0;
  if (m1 > 0) {
    PickPred pp{l, G, s->mcval, s->edges, num, thin ? 3ll * npts : num};
    PickEmit pe{G, s->mcval, s->edges, num, thin ? 3ll * npts : num, s->kept, s->kept_cap};
    RSO_TRY(compact<2>(h, pp, pe, m1, &nk));
  }
  if (npts > 0) {
    k_final_pick<<<cdiv(npts, SP_THREADS), SP_THREADS, 0, h->stream>>>(s->kept, s->kept_cap, nk, npts, s->xyz);
    note_launch();
    RSO_TRY(launch_check(h, "surface final pick"));
  }
  s->n = std::max(npts, 0);
  if (info) {
    info->n_crossings = num;
    info->n_first_pick = m1;
    info->n_in_model = nk;
    info->n_points = s->n;
    info->reserved = 0;
  }
  return RSO_OK;
}

rso_status surface_selfsupport(rso_handle* h, const double* c, double beta, int mode, double opt_angle,
                               double default_angle, float* per_out, double* dc, double* value, double* count,
                               double* dirsum) {
  SurfState* s = surf(h);
  const int n = s->n;
  if (n <= 0) { h->err = "no surface points"; return RSO_ERR_STATE; }
  const SplineP S = spline_p(h);
  const int nblk = cdiv(n, SP_THREADS);
  k_surf_eval<<<nblk, SP_THREADS, 0, h->stream>>>(S, c, s->xyz, n, beta, s->nrm, s->ins, s->dir); note_launch();
  RSO_TRY(launch_check(h, "surf_eval"));
  RSO_TRY(sum_float(h, s->dir, n, s->scal + 0));
  SurfPar P{mode, std::cos(opt_angle), std::cos(default_angle)};
  k_surf_value<<<nblk, SP_THREADS, 0, h->stream>>>(n, s->nrm, s->ins, s->scal + 0, P, s->per, per_out, s->flags,
                                                   s->down, s->w); note_launch();
  RSO_TRY(launch_check(h, "surf_value"));
  const int nred = std::min(nblk, 512);
  k_sumd_partial<<<nred, SP_THREADS, 0, h->stream>>>(s->per, n, h->red); note_launch();
  RSO_TRY(reduce_partials(h, h->red, nred, s->scal + 1));
  RSO_TRY(sum_float(h, s->down, n, s->scal + 2));
  if (dc) {
    RSO_CHECK_CUDA(h, cudaMemsetAsync(dc, 0, sizeof(double) * h->sp.n_coeff, h->stream));
    k_surf_grad<<<nblk, SP_THREADS, 0, h->stream>>>(S, s->xyz, n, s->w, s->scal + 2, mode, dc); note_launch();
    RSO_TRY(launch_check(h, "surf_grad"));
  }
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(s->h_scal, s->scal, 3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  const double ds = s->h_scal[0], sum = s->h_scal[1];
  const double cnt = mode % 2 == 0 ? s->h_scal[2] : (double)n;
  if (dirsum) *dirsum = ds;
  if (count) *count = cnt;
  double v = 0;
  if (cnt != 0) v = mode <= 1 ? std::pow(sum / cnt, 1 / 8.0) - 1 : sum / cnt;
  if (value) *value = v;
  return RSO_OK;
}

}  // namespace rso

using namespace rso;

static rso_status coeff_in(rso_handle* h, const float* coeff) {
  k_f2d_c<<<cdiv(h->sp.n_coeff, 256), 256, 0, h->stream>>>(coeff, h->coef_a, h->sp.n_coeff); note_launch();
  return launch_check(h, "surface coefficients");
}

extern "C" rso_status rso_surface_points(rso_handle* h, const float* coeff, int mc_res, int n_points,
                                         const float* model_box, rso_surface_info* info) {
  if (!h || !coeff || mc_res < 1 || mc_res > 1022 || n_points < 0) return RSO_ERR_INVALID_ARG;
  if (!h->sp.order) { h->err = "spline not set up"; return RSO_ERR_STATE; }
  float box[6];
  if (model_box) {
    std::memcpy(box, model_box, sizeof(box));
    for (int a = 0; a < 3; a++)
      if (!(box[3 + a] > box[a])) { h->err = "empty model box"; return RSO_ERR_INVALID_ARG; }
  } else {
    active_box(h, box);
  }
  RSO_TRY(coeff_in(h, coeff));
  RSO_TRY(surface_points(h, h->coef_a, mc_res, n_points, box, info));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_set_surface_points(rso_handle* h, const float* xyz, int n_points) {
  if (!h || (!xyz && n_points > 0) || n_points < 0) return RSO_ERR_INVALID_ARG;
  RSO_TRY(points_reserve(h, n_points));
  SurfState* s = surf(h);
  if (n_points > 0)
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(s->xyz, xyz, sizeof(float) * 3 * (size_t)n_points, cudaMemcpyDefault,
                                      h->stream));
  s->n = n_points;
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_get_surface_points(rso_handle* h, float* xyz, int capacity, int* n_points) {
  if (!h) return RSO_ERR_INVALID_ARG;
  const int n = h->surf ? ((SurfState*)h->surf)->n : 0;
  if (n_points) *n_points = n;
  if (!xyz) return RSO_OK;
  if (capacity < n) { h->err = "capacity below the number of surface points"; return RSO_ERR_INVALID_ARG; }
  if (n > 0)
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(xyz, ((SurfState*)h->surf)->xyz, sizeof(float) * 3 * (size_t)n,
                                      cudaMemcpyDefault, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_surface_selfsupport(rso_handle* h, const float* coeff, double beta, int mode,
                                              double opt_angle, double default_angle, float* per_point, float* dc,
                                              double* value, double* count, double* direction_sum) {
  if (!h || !coeff || mode < 0 || mode > 5) return RSO_ERR_INVALID_ARG;
  if (!h->sp.order) { h->err = "spline not set up"; return RSO_ERR_STATE; }
  RSO_TRY(coeff_in(h, coeff));
  RSO_TRY(surface_selfsupport(h, h->coef_a, beta, mode, opt_angle, default_angle, per_point, dc ? h->coef_b : nullptr,
                              value, count, direction_sum));
  if (dc) {
    k_d2f_c<<<cdiv(h->sp.n_coeff, 256), 256, 0, h->stream>>>(h->coef_b, dc, h->sp.n_coeff); note_launch();
    RSO_TRY(launch_check(h, "surface gradient"));
  }
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_get_surface_normals(rso_handle* h, double* normals, uint8_t* flags) {
  if (!h) return RSO_ERR_INVALID_ARG;
  SurfState* s = (SurfState*)h->surf;
  const int n = s ? s->n : 0;
  if (n > 0 && normals)
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(normals, s->nrm, sizeof(double) * 3 * (size_t)n, cudaMemcpyDefault, h->stream));
  if (n > 0 && flags)
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(flags, s->flags, 2 * (size_t)n, cudaMemcpyDefault, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}
