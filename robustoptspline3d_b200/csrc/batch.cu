// Batched solves: k systems K u_i = f_i on one operator (the load cases of a
// worst-case or multi-load study).  Every level vector becomes a slab of k
// consecutive vectors and the levels carry nb = k, so each V-cycle kernel
// launch works on all k systems (the fine operator, transfers and row-split
// stencil kernels over a system index in the grid, the large-level stencil
// kernel reading each stencil entry once for up to four systems, the cluster
// kernel of the small levels over system x node pairs).  CG runs one
// recurrence per system with per-system scalars; a converged system keeps
// alpha = beta = 0 while the others continue.  In mixed precision the
// recurrence is FP32 with FP64 residual replacement, as for single solves,
// each system replacing on its own rule.
#include "rso_internal.cuh"
#include <algorithm>
#include <chrono>
#include <cmath>
#include <utility>

namespace rso {

constexpr int BR_BLOCKS = 296, BR_THREADS = 512, KS = 8;  // KS doubles of scalars per system

__device__ __forceinline__ double b_block_sum(double v) {
  __shared__ double ws[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) ws[w] = v;
  __syncthreads();
  v = (threadIdx.x < blockDim.x / 32) ? ws[lane] : 0.0;
  if (w == 0)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  return v;
}

// partial sums of a_b . b_b for every system b = blockIdx.y
template <typename B>
__global__ void __launch_bounds__(BR_THREADS) k_bdot(long long n, const double* __restrict__ a,
                                                     const B* __restrict__ b, double* __restrict__ part) {
  const long long o = (long long)blockIdx.y * n;
  double s = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s += a[o + i] * (double)b[o + i];
  s = b_block_sum(s);
  if (threadIdx.x == 0) part[blockIdx.y * BR_BLOCKS + blockIdx.x] = s;
}

// r -= alpha_b q, FP32 copy of r, partial sums of r.r per system
__global__ void __launch_bounds__(BR_THREADS) k_bresid(long long n, const double* __restrict__ s,
                                                       const double* __restrict__ q, double* __restrict__ r,
                                                       float* __restrict__ r32, double* __restrict__ part) {
  const long long o = (long long)blockIdx.y * n;
  const double a = s[blockIdx.y * KS + 2];
  double acc = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double ri = r[o + i] - a * q[o + i];
    r[o + i] = ri;
    if (r32) r32[o + i] = (float)ri;
    acc += ri * ri;
  }
  acc = b_block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.y * BR_BLOCKS + blockIdx.x] = acc;
}

__global__ void k_bsum(const double* __restrict__ part, double* __restrict__ s, int slot) {
  double v = 0;
  for (int i = threadIdx.x; i < BR_BLOCKS; i += blockDim.x) v += part[blockIdx.x * BR_BLOCKS + i];
  v = b_block_sum(v);
  if (threadIdx.x == 0) s[blockIdx.x * KS + slot] = v;
}

// s: 0 rz, 1 pq, 2 alpha, 3 rz_new, 4 beta, 5 rr, 6 ff
__global__ void k_balpha(int k, double* s, const int* __restrict__ done) {
  const int b = threadIdx.x;
  if (b >= k) return;
  const double pq = s[b * KS + 1];
  s[b * KS + 2] = (done[b] || pq == 0.0) ? 0.0 : s[b * KS + 0] / pq;
}
__global__ void k_bbeta(int k, double* s, const int* __restrict__ done) {
  const int b = threadIdx.x;
  if (b >= k) return;
  const double rz = s[b * KS + 0];
  s[b * KS + 4] = (done[b] || rz == 0.0) ? 0.0 : s[b * KS + 3] / rz;
  s[b * KS + 0] = s[b * KS + 3];
}

// x += alpha_b p; p = z + beta_b p
template <typename Z>
__global__ void k_bstep_dir(long long n, long long total, const double* __restrict__ s, const Z* __restrict__ z,
                            double* __restrict__ p, double* __restrict__ x) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= total) return;
  const long long b = i / n;
  const double pi = p[i];
  x[i] += s[b * KS + 2] * pi;
  p[i] = (double)z[i] + s[b * KS + 4] * pi;
}
__global__ void k_bstep(long long n, long long total, const double* __restrict__ s, const double* __restrict__ p,
                        double* __restrict__ x) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= total) return;
  x[i] += s[(i / n) * KS + 2] * p[i];
}
__global__ void k_bd2f(long long total, const double* __restrict__ a, float* __restrict__ b) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < total) b[i] = (float)a[i];
}
__global__ void k_bf2d(long long total, const float* __restrict__ a, double* __restrict__ b) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < total) b[i] = (double)a[i];
}

// FP32 Krylov recurrence of the batch (reliable-update PCG, as solve_pcg_k32):
// r -= alpha_b q in FP32 with per-system sums of r.r, per-system a.b of FP32
// vectors; the steps x (FP64) += alpha_b p (FP32) and p = z + beta_b p below
__global__ void __launch_bounds__(BR_THREADS) k_bresid32(long long n, const double* __restrict__ s,
                                                         const float* __restrict__ q, float* __restrict__ r,
                                                         double* __restrict__ part) {
  const long long o = (long long)blockIdx.y * n;
  const float a = (float)s[blockIdx.y * KS + 2];
  double acc = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float ri = r[o + i] - a * q[o + i];
    r[o + i] = ri;
    acc += (double)ri * ri;
  }
  acc = b_block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.y * BR_BLOCKS + blockIdx.x] = acc;
}
__global__ void __launch_bounds__(BR_THREADS) k_bdot32(long long n, const float* __restrict__ a,
                                                       const float* __restrict__ b, double* __restrict__ part) {
  const long long o = (long long)blockIdx.y * n;
  double acc = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    acc += (double)a[o + i] * b[o + i];
  acc = b_block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.y * BR_BLOCKS + blockIdx.x] = acc;
}
// Deferred steps of the batch (as in solve_pcg_k32): each new direction goes
// to the next slot of a ring of three FP32 slabs (the two halves of p's
// memory and the half of q's the FP32 q leaves free), each system's step
// size beside it, and x takes the waiting steps in their order at a
// replacement or when the ring is full: the FP64 operations of the
// per-iteration step in the same order, so x is bit-identical.
constexpr int kBRing = 3;
struct BRing {
  const float* p[kBRing];
};
__global__ void k_balpha_keep(int k, double* s, const int* __restrict__ done, double* __restrict__ keep) {
  const int b = threadIdx.x;
  if (b >= k) return;
  const double pq = s[b * KS + 1];
  const double a = (done[b] || pq == 0.0) ? 0.0 : s[b * KS + 0] / pq;
  s[b * KS + 2] = a;
  keep[b] = a;
}
__global__ void k_bflush(long long n, long long total, int k, const double* __restrict__ alpha, const BRing R, int cnt,
                         double* __restrict__ x) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= total) return;
  const long long b = i / n;
  double xi = x[i];
#pragma unroll
  for (int j = 0; j < kBRing; j++) {
    if (j >= cnt) break;
    xi += alpha[j * k + b] * R.p[j][i];
  }
  x[i] = xi;
}
// p_out = z + beta_b p_in (p_out may be p_in)
__global__ void k_bdir32(long long n, long long total, const double* __restrict__ s, const float* __restrict__ z,
                         const float* p_in, float* p_out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= total) return;
  const long long b = i / n;
  p_out[i] = z[i] + (float)s[b * KS + 4] * p_in[i];
}

// r32 = r for the systems whose bit is set in mask (k <= 64)
__global__ void k_bd2f_sel(long long n, long long total, const double* __restrict__ r, float* __restrict__ r32,
                           unsigned long long mask) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= total || !((mask >> (i / n)) & 1ULL)) return;
  r32[i] = (float)r[i];
}

static void batch_free(rso_handle* h) {
  auto& B = h->batch;
  for (auto* v : {&B.u32, &B.f32, &B.r32, &B.t32})
    for (float* p : *v) cudaFree(p);
  for (auto* v : {&B.u64, &B.f64, &B.r64, &B.t64})
    for (double* p : *v) cudaFree(p);
  B.u32.clear(); B.f32.clear(); B.r32.clear(); B.t32.clear();
  B.u64.clear(); B.f64.clear(); B.r64.clear(); B.t64.clear();
  for (double* p : {B.x, B.r, B.p, B.q, B.z, B.cf, B.red, B.fpart, B.xfer, B.scal, B.ralpha}) cudaFree(p);
  if (B.h_scal) cudaFreeHost(B.h_scal);
  cudaFree(B.done);
  B = rso_handle::Batch();  // c_fb aliases B.cf, freed above
  h->c_fb = nullptr;
}

void batch_release(rso_handle* h) { batch_free(h); }

static rso_status batch_alloc(rso_handle* h, int k) {
  auto& B = h->batch;
  if (B.cap >= k) return RSO_OK;
  batch_free(h);
  const bool mixed = h->cfg.precision == RSO_MIXED;
  const size_t nl = h->L.size();
#define BALLOC(ptr, bytes)                                                   \
  do {                                                                       \
    if (cudaMalloc((void**)&(ptr), (bytes)) != cudaSuccess) {                \
      cudaGetLastError();                                                    \
      batch_free(h);                                                         \
      h->err = "out of device memory for the batch of systems";              \
      return RSO_ERR_OOM;                                                    \
    }                                                                        \
  } while (0)
  for (size_t li = 0; li < nl; li++) {
    const size_t n = (size_t)k * 3 * h->L[li].NP;
    if (mixed) {
      float *a, *b, *c, *d;
      BALLOC(a, 4 * n); B.u32.push_back(a);
      BALLOC(b, 4 * n); B.f32.push_back(b);
      BALLOC(c, 4 * n); B.r32.push_back(c);
      BALLOC(d, 4 * n); B.t32.push_back(d);
    } else {
      double *a, *b, *c, *d;
      BALLOC(a, 8 * n); B.u64.push_back(a);
      BALLOC(b, 8 * n); B.f64.push_back(b);
      BALLOC(c, 8 * n); B.r64.push_back(c);
      BALLOC(d, 8 * n); B.t64.push_back(d);
    }
  }
  const size_t n0 = (size_t)k * 3 * h->L[0].NP;
  BALLOC(B.x, 8 * n0); BALLOC(B.r, 8 * n0); BALLOC(B.p, 8 * n0); BALLOC(B.q, 8 * n0);
  BALLOC(B.z, 8 * n0);  // FP64 z, or the padded right-hand sides of the FP32 recurrence
  BALLOC(B.cf, sizeof(double) * std::max(1, 3 * h->nc) * k);
  BALLOC(B.red, sizeof(double) * BR_BLOCKS * k);
  BALLOC(B.fpart, sizeof(double) * h->fpart_n * k);
  BALLOC(B.xfer, sizeof(double) * h->xfer_n * k);
  BALLOC(B.scal, sizeof(double) * KS * k);
  BALLOC(B.ralpha, sizeof(double) * kBRing * k);
  BALLOC(B.done, sizeof(int) * k);
#undef BALLOC
  if (cudaMallocHost((void**)&B.h_scal, sizeof(double) * KS * k) != cudaSuccess) {
    cudaGetLastError();
    batch_free(h);
    h->err = "out of pinned host memory for the batch";
    return RSO_ERR_OOM;
  }
  h->c_fb = B.cf;
  B.cap = k;
  return RSO_OK;
}

// swaps the batch slabs into the levels (nb = k) for the lifetime of the guard
struct BatchScope {
  rso_handle* h;
  std::vector<Level> saved;
  double* xfer;
  size_t xfer_n;
  double* fpart;
  long long fpart_n;
  BatchScope(rso_handle* hh, int k) : h(hh), saved(hh->L), xfer(hh->xfer), xfer_n(hh->xfer_n), fpart(hh->fpart),
                                      fpart_n(hh->fpart_n) {
    auto& B = h->batch;
    const bool mixed = h->cfg.precision == RSO_MIXED;
    for (size_t li = 0; li < h->L.size(); li++) {
      Level& l = h->L[li];
      l.nb = k;
      if (mixed) { l.u32 = B.u32[li]; l.f32 = B.f32[li]; l.r32 = B.r32[li]; l.t32 = B.t32[li]; }
      else { l.u64 = B.u64[li]; l.f64 = B.f64[li]; l.r64 = B.r64[li]; l.t64 = B.t64[li]; }
    }
    h->xfer = B.xfer;
    h->xfer_n = xfer_n * k;
    h->fpart = B.fpart;
    h->fpart_n = fpart_n * k;
  }
  ~BatchScope() {
    h->L = saved;
    h->xfer = xfer;
    h->xfer_n = xfer_n;
    h->fpart = fpart;
    h->fpart_n = fpart_n;
  }
};

static double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

rso_status solve_pcg_batch(rso_handle* h, int k, const double* F, double* U, double tol, int max_iter,
                           rso_solve_info* infos) {
  if (h->cfg.smoother == RSO_SMOOTH_GS) {
    h->err = "batched solves need the damped Jacobi or Chebyshev smoother";
    return RSO_ERR_UNSUPPORTED;
  }
  RSO_TRY(batch_alloc(h, k));
  auto& B = h->batch;
  const double t0 = now_ms();
  const long long n3 = 3 * h->L[0].NP, tot = (long long)k * n3, nn3 = 3 * h->L[0].nn;
  const bool mixed = h->cfg.precision == RSO_MIXED;
  const bool k32 = mixed && h->krylov32 > 0;
  // dense -> padded slabs: x holds the initial guesses; the right-hand sides
  // go to q for now (FP64 recurrence) or to z, kept for the residual
  // replacements (FP32 recurrence, whose p and q are FP32 in p's and q's memory)
  double* fpad = k32 ? B.z : B.q;
  for (int b = 0; b < k; b++) {
    RSO_TRY(pad_nodes(h, 0, U + b * nn3, B.x + b * n3));
    RSO_TRY(pad_nodes(h, 0, F + b * nn3, fpad + b * n3));
    RSO_TRY(zero_support(h, B.x + b * n3));
    RSO_TRY(zero_support(h, fpad + b * n3));
    RSO_TRY(displacement_project(h, fpad + b * n3));  // support-free problems, as rso_solve
  }
  std::vector<int> it(k, 0), done(k, 0);
  std::vector<double> fn(k, 0), rel(k, 0);
  rso_status status = RSO_OK;
  {
    BatchScope scope(h, k);
    Level& l0 = h->L[0];
    const dim3 rg(BR_BLOCKS, k);
    double* s = B.scal;
    // r = f - K x; |f|^2 and |r|^2 per system
    RSO_TRY(fine_residual<double>(h, B.x, fpad, B.r, h->rp64));
    k_bdot<double><<<rg, BR_THREADS, 0, h->stream>>>(n3, fpad, fpad, B.red); rso::note_launch();
    k_bsum<<<k, BR_THREADS, 0, h->stream>>>(B.red, s, 6); rso::note_launch();
    k_bdot<double><<<rg, BR_THREADS, 0, h->stream>>>(n3, B.r, B.r, B.red); rso::note_launch();
    k_bsum<<<k, BR_THREADS, 0, h->stream>>>(B.red, s, 5); rso::note_launch();
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(B.h_scal, s, sizeof(double) * KS * k, cudaMemcpyDeviceToHost, h->stream));
    RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
    int left = 0;
    for (int b = 0; b < k; b++) {
      fn[b] = std::sqrt(B.h_scal[b * KS + 6]);
      rel[b] = fn[b] > 0 ? std::sqrt(B.h_scal[b * KS + 5]) / fn[b] : 0.0;
      done[b] = rel[b] < tol ? 1 : 0;
      left += !done[b];
    }
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(B.done, done.data(), sizeof(int) * k, cudaMemcpyHostToDevice, h->stream));
    auto precondition_z = [&]() -> rso_status {
      if (mixed) {
        k_bd2f<<<cdiv(tot, 256), 256, 0, h->stream>>>(tot, B.r, l0.f32); rso::note_launch();
        return vcycle_mixed(h);
      }
      RSO_CHECK_CUDA(h, cudaMemcpyAsync(l0.f64, B.r, sizeof(double) * tot, cudaMemcpyDeviceToDevice, h->stream));
      RSO_TRY(vcycle_levels<double>(h, h->cfg.pre, h->cfg.post, 1, true));
      RSO_CHECK_CUDA(h, cudaMemcpyAsync(B.z, h->L[0].u64, sizeof(double) * tot, cudaMemcpyDeviceToDevice, h->stream));
      return RSO_OK;
    };
    // an FP32 recurrence that stalls hands over to the FP64 one (as for single
    // solves: a cycle ends after at most kCycleMax iterations, and a true
    // residual not below max(0.5, sqrt(factor)) of the previous one stalls)
    bool stalled = false;
    int used = 0;
    if (left > 0 && k32) {
      constexpr int kCycleMax = 30;
      std::vector<int> since(k, 0), cycles(k, 0);
      std::vector<double> rrec(k, 0.0);  // recursive residual norms at the last iteration
      float* p32 = reinterpret_cast<float*>(B.p);
      float* q32 = reinterpret_cast<float*>(B.q);
      float* r32 = l0.f32;  // the batched V-cycle's right-hand sides (the smoothers rotate u, not f)
      std::vector<double> rbase(k);
      for (int b = 0; b < k; b++) rbase[b] = rel[b] * fn[b];
      // the operator writes interior nodes only: q's padding must be zero
      RSO_CHECK_CUDA(h, cudaMemsetAsync(q32, 0, sizeof(float) * tot, h->stream));
      k_bd2f<<<cdiv(tot, 256), 256, 0, h->stream>>>(tot, B.r, r32); rso::note_launch();
      // r . z of every system from the V-cycle's last fine step (a post-smoothing
      // Jacobi or Chebyshev step), as in single solves
      const bool fuse = h->cfg.post >= 1;
      struct ZdotReset {
        rso_handle* h;
        ~ZdotReset() {
          h->vc_zdot = nullptr;
          h->vc_zdot_stride = 1;
        }
      } zreset{h};
      h->vc_zdot = fuse ? s + 0 : nullptr;
      h->vc_zdot_stride = KS;
      RSO_TRY(vcycle_mixed(h));
      RSO_CHECK_CUDA(h, cudaMemcpyAsync(p32, l0.u32, sizeof(float) * tot, cudaMemcpyDeviceToDevice, h->stream));
      if (!fuse) {
        k_bdot32<<<rg, BR_THREADS, 0, h->stream>>>(n3, r32, l0.u32, B.red); rso::note_launch();
        k_bsum<<<k, BR_THREADS, 0, h->stream>>>(B.red, s, 0); rso::note_launch();
      }
      h->vc_zdot = fuse ? s + 3 : nullptr;
      // the deferred steps' ring (see k_bflush)
      float* ring[kBRing] = {p32, p32 + tot, q32 + tot};
      int pend = 0;     // steps waiting: directions ring[0 .. pend), step sizes B.ralpha[0 .. pend)
      float* pc = p32;  // the current direction, ring[pend] until its step sizes are known
      auto flush = [&]() -> rso_status {
        if (pend == 0) return RSO_OK;
        BRing R;
        for (int j = 0; j < kBRing; j++) R.p[j] = ring[j < pend ? j : 0];
        k_bflush<<<cdiv(tot, 256), 256, 0, h->stream>>>(n3, tot, k, B.ralpha, R, pend, B.x); rso::note_launch();
        pend = 0;
        return launch_check(h, "batched pcg32 deferred steps");
      };
      int iter = 0;
      while (true) {
        RSO_TRY(fine_applyK_dot32(h, pc, q32, s + 1, KS));
        k_balpha_keep<<<1, 64, 0, h->stream>>>(k, s, B.done, B.ralpha + (long long)pend * k); rso::note_launch();
        pend++;
        k_bresid32<<<rg, BR_THREADS, 0, h->stream>>>(n3, s, q32, r32, B.red); rso::note_launch();
        k_bsum<<<k, BR_THREADS, 0, h->stream>>>(B.red, s, 5); rso::note_launch();
        RSO_CHECK_CUDA(h, cudaMemcpyAsync(B.h_scal, s, sizeof(double) * KS * k, cudaMemcpyDeviceToHost, h->stream));
        RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
        vcycle_graphs_harvest(h);
        iter++;
        // systems asking for a replacement: their recursive residual dropped
        // by the factor since their last one, or below the tolerance; all at
        // the iteration limit
        unsigned long long ask = 0;
        for (int b = 0; b < k; b++) {
          if (done[b]) continue;
          it[b] = iter;
          since[b]++;
          const double rn = std::sqrt(B.h_scal[b * KS + 5]);
          if (!std::isfinite(rn)) { h->err = "non-finite residual in batched PCG"; return RSO_ERR_NONFINITE; }
          rel[b] = rn / fn[b];
          rrec[b] = rn;
          if (rn < tol * fn[b] || rn < h->krylov32 * rbase[b] || iter >= max_iter || since[b] >= kCycleMax)
            ask |= 1ULL << b;
        }
        const bool replace = ask != 0;
        if (replace) {
          // every system takes its step now (frozen ones have alpha 0; the
          // direction update below then leaves x alone); the true FP64
          // residuals replace the recursive ones of the asking systems only,
          // so each system follows the sequence of its own single solve
          RSO_TRY(flush());
          RSO_TRY(fine_residual<double>(h, B.x, fpad, B.r, h->rp64));
          k_bdot<double><<<rg, BR_THREADS, 0, h->stream>>>(n3, B.r, B.r, B.red); rso::note_launch();
          k_bsum<<<k, BR_THREADS, 0, h->stream>>>(B.red, s, 5); rso::note_launch();
          RSO_CHECK_CUDA(h, cudaMemcpyAsync(B.h_scal, s, sizeof(double) * KS * k, cudaMemcpyDeviceToHost, h->stream));
          RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
          left = 0;
          unsigned long long take = 0;
          for (int b = 0; b < k; b++) {
            if (done[b]) continue;
            if (!((ask >> b) & 1ULL)) { left++; continue; }
            const double rtrue = std::sqrt(B.h_scal[b * KS + 5]);
            rel[b] = rtrue / fn[b];
            if (!std::isfinite(rel[b])) { h->err = "non-finite residual in batched PCG"; return RSO_ERR_NONFINITE; }
            if (rel[b] < tol) { done[b] = 1; continue; }
            cycles[b]++;
            if (rtrue > stall_ratio(h->krylov32, rrec[b] / rbase[b]) * rbase[b] ||
                (h->krylov32_cycles > 0 && cycles[b] >= h->krylov32_cycles))
              stalled = true;
            rbase[b] = rtrue;
            since[b] = 0;
            left++;
            take |= 1ULL << b;
          }
          if (left == 0 || iter >= max_iter) { stalled = false; break; }
          if (stalled) {  // B.r holds every system's true residual of B.x
            used = iter;
            RSO_CHECK_CUDA(h, cudaMemcpyAsync(B.done, done.data(), sizeof(int) * k, cudaMemcpyHostToDevice, h->stream));
            break;
          }
          if (take) { k_bd2f_sel<<<cdiv(tot, 256), 256, 0, h->stream>>>(n3, tot, B.r, r32, take); rso::note_launch(); }
          RSO_CHECK_CUDA(h, cudaMemcpyAsync(B.done, done.data(), sizeof(int) * k, cudaMemcpyHostToDevice, h->stream));
        }
        RSO_TRY(vcycle_mixed(h));
        if (!fuse) {
          k_bdot32<<<rg, BR_THREADS, 0, h->stream>>>(n3, r32, l0.u32, B.red); rso::note_launch();
          k_bsum<<<k, BR_THREADS, 0, h->stream>>>(B.red, s, 3); rso::note_launch();
        }
        k_bbeta<<<1, 64, 0, h->stream>>>(k, s, B.done); rso::note_launch();
        if (pend == kBRing) RSO_TRY(flush());
        float* pn = ring[pend];  // pc itself right after a flush of one step
        k_bdir32<<<cdiv(tot, 256), 256, 0, h->stream>>>(n3, tot, s, l0.u32, pc, pn); rso::note_launch();
        pc = pn;
        RSO_TRY(launch_check(h, "batched pcg32"));
      }
    }
    if (left > 0 && (!k32 || stalled)) {
      // q held the FP32 recurrence's q (or nothing yet), and the operator
      // writes interior nodes only while the residual update reads every entry
      if (stalled) RSO_CHECK_CUDA(h, cudaMemsetAsync(B.q, 0, sizeof(double) * tot, h->stream));
      RSO_TRY(precondition_z());
      if (mixed) {
        k_bf2d<<<cdiv(tot, 256), 256, 0, h->stream>>>(tot, h->L[0].u32, B.p); rso::note_launch();
        k_bdot<float><<<rg, BR_THREADS, 0, h->stream>>>(n3, B.r, h->L[0].u32, B.red); rso::note_launch();
      } else {
        RSO_CHECK_CUDA(h, cudaMemcpyAsync(B.p, B.z, sizeof(double) * tot, cudaMemcpyDeviceToDevice, h->stream));
        k_bdot<double><<<rg, BR_THREADS, 0, h->stream>>>(n3, B.r, B.z, B.red); rso::note_launch();
      }
      k_bsum<<<k, BR_THREADS, 0, h->stream>>>(B.red, s, 0); rso::note_launch();
      int iter = 0;
      while (true) {
        RSO_TRY(fine_applyK_dot(h, B.p, B.q, h->rp64, s + 1, KS));
        k_balpha<<<1, 64, 0, h->stream>>>(k, s, B.done); rso::note_launch();
        k_bresid<<<rg, BR_THREADS, 0, h->stream>>>(n3, s, B.q, B.r, mixed ? h->L[0].f32 : nullptr, B.red); rso::note_launch();
        k_bsum<<<k, BR_THREADS, 0, h->stream>>>(B.red, s, 5); rso::note_launch();
        RSO_CHECK_CUDA(h, cudaMemcpyAsync(B.h_scal, s, sizeof(double) * KS * k, cudaMemcpyDeviceToHost, h->stream));
        RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
        vcycle_graphs_harvest(h);
        iter++;
        left = 0;
        for (int b = 0; b < k; b++) {
          if (done[b]) continue;
          it[b] = used + iter;
          rel[b] = std::sqrt(B.h_scal[b * KS + 5]) / fn[b];
          if (!std::isfinite(rel[b])) { h->err = "non-finite residual in batched PCG"; return RSO_ERR_NONFINITE; }
          if (rel[b] < tol) done[b] = 2;  // converged in this iteration: x still takes this step
          else left++;
        }
        if (left == 0 || used + iter >= max_iter) {
          k_bstep<<<cdiv(tot, 256), 256, 0, h->stream>>>(n3, tot, s, B.p, B.x); rso::note_launch();
          break;
        }
        // systems that converged now take their last step with the direction update, then freeze
        RSO_TRY(precondition_z());
        if (mixed) { k_bdot<float><<<rg, BR_THREADS, 0, h->stream>>>(n3, B.r, h->L[0].u32, B.red); rso::note_launch(); }
        else { k_bdot<double><<<rg, BR_THREADS, 0, h->stream>>>(n3, B.r, B.z, B.red); rso::note_launch(); }
        k_bsum<<<k, BR_THREADS, 0, h->stream>>>(B.red, s, 3); rso::note_launch();
        k_bbeta<<<1, 64, 0, h->stream>>>(k, s, B.done); rso::note_launch();
        if (mixed) { k_bstep_dir<float><<<cdiv(tot, 256), 256, 0, h->stream>>>(n3, tot, s, h->L[0].u32, B.p, B.x); }
        else { k_bstep_dir<double><<<cdiv(tot, 256), 256, 0, h->stream>>>(n3, tot, s, B.z, B.p, B.x); }
        rso::note_launch();
        for (int b = 0; b < k; b++)
          if (done[b] == 2) done[b] = 1;
        RSO_CHECK_CUDA(h, cudaMemcpyAsync(B.done, done.data(), sizeof(int) * k, cudaMemcpyHostToDevice, h->stream));
        RSO_TRY(launch_check(h, "batched pcg"));
      }
    }
  }
  for (int b = 0; b < k; b++) {
    RSO_TRY(displacement_project(h, B.x + b * n3));  // support-free problems
    RSO_TRY(unpad_nodes(h, 0, B.x + b * n3, U + b * nn3));
    if (rel[b] >= tol && fn[b] > 0) status = RSO_ERR_BUDGET_EXCEEDED;
  }
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  RSO_TRY(fine_stage_check(h));
  const double ms = now_ms() - t0;
  if (infos)
    for (int b = 0; b < k; b++) { infos[b].iterations = it[b]; infos[b].rel_res = rel[b]; infos[b].ms = ms; }
  if (status != RSO_OK) h->err = "batched PCG: a system did not reach the tolerance within max_iter";
  return status;
}

}  // namespace rso

using namespace rso;

extern "C" rso_status rso_solve_batch(rso_handle* h, int k, const double* F, double* U, double tol, int max_iter,
                                      rso_solve_info* infos) {
  if (!h || !F || !U || k < 1 || k > 64 || !(tol > 0) || max_iter < 0) return RSO_ERR_INVALID_ARG;
  if (!h->operators_ready) { h->err = "call rso_update_operators after rso_set_density"; return RSO_ERR_STATE; }
  return solve_pcg_batch(h, k, F, U, tol, max_iter, infos);
}
