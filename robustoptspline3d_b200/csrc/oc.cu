// Optimality-criteria (OC) updaters: the reference's alternative to MMA.
//
// updateDensities / updateDensities2 (optimization/optimization.cu:394-598)
// and updateCoeff (:600-706) search, by bisection on a sensitivity threshold
// g in [0, max |sens|], the multiplicative update
//   x' = clamp(clamp(x (|min(s, 0)| / g)^damp, x - step, x + step), lo, hi)
// (trySensMultiplier_kernel :366-392, tryCSensMultiplier_kernel :560-598)
// whose volume fraction meets the goal; shell elements are held at 1.  The
// search runs on the device (one trial kernel with its volume partials per
// bisection step); the threshold, the volume and the bracket are FP32 host
// scalars as in the reference.
#include "rso_internal.cuh"
#include <cmath>

namespace rso {
namespace {

constexpr int OC_BLOCKS = 592, OC_THREADS = 256;

// one trial over n entries: out = trial(src); volume partials over the
// entries that count (active elements in dense order when L is given,
// everything otherwise); inactive entries keep src
__global__ void __launch_bounds__(OC_THREADS) k_oc_try(long long n, const Level L, int dense_elems,
                                                       const float* __restrict__ src, const float* __restrict__ sens,
                                                       float g, float step, float damp, float lo, float hi,
                                                       const uint8_t* __restrict__ shell, float* __restrict__ out,
                                                       double* __restrict__ part) {
  double s = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (dense_elems) {
      const int x = (int)(i % L.ex), y = (int)((i / L.ex) % L.ey), z = (int)(i / ((long long)L.ex * L.ey));
      if (!L.emask[L.eidx(x, y, z)]) {
        out[i] = src[i];
        continue;
      }
    }
    float gi = sens[i];
    if (gi > 0) gi = 0;
    gi = fabsf(gi);
    const float old = src[i];
    float v = old * powf(gi / g, damp);
    v = fminf(fmaxf(v, old - step), old + step);
    v = fminf(fmaxf(v, lo), hi);
    if (shell && shell[i]) v = 1.f;
    out[i] = v;
    s += v;
  }
  __shared__ double ws[OC_THREADS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
#pragma unroll
    for (int w = 0; w < OC_THREADS / 32; w++) t += ws[w];
    part[blockIdx.x] = t;
  }
}

// max |a| over n entries (active elements only when dense_elems)
__global__ void __launch_bounds__(OC_THREADS) k_oc_maxabs(long long n, const Level L, int dense_elems,
                                                          const float* __restrict__ a, double* __restrict__ part) {
  double m = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (dense_elems) {
      const int x = (int)(i % L.ex), y = (int)((i / L.ex) % L.ey), z = (int)(i / ((long long)L.ex * L.ey));
      if (!L.emask[L.eidx(x, y, z)]) continue;
    }
    m = fmax(m, (double)fabsf(a[i]));
  }
  __shared__ double ws[OC_THREADS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
#pragma unroll
    for (int w = 0; w < OC_THREADS / 32; w++) t = fmax(t, ws[w]);
    part[blockIdx.x] = t;
  }
}

__global__ void k_oc_maxfinal(const double* __restrict__ part, int n, double* __restrict__ out) {
  double m = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, part[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  __shared__ double ws[32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x / 32); w++) t = fmax(t, ws[w]);
    *out = t;
  }
}

__global__ void k_oc_change(long long n, const float* __restrict__ a, const float* __restrict__ b,
                            double* __restrict__ part_max, double* __restrict__ part_sum) {
  double m = 0, s = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double d = fabs((double)a[i] - (double)b[i]);
    m = fmax(m, d);
    s += d;
  }
  __shared__ double wm[OC_THREADS / 32], wsum[OC_THREADS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    s += __shfl_down_sync(0xffffffffu, s, o);
  }
  if ((threadIdx.x & 31) == 0) { wm[threadIdx.x >> 5] = m; wsum[threadIdx.x >> 5] = s; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tm = 0, ts = 0;
    for (int w = 0; w < OC_THREADS / 32; w++) { tm = fmax(tm, wm[w]); ts += wsum[w]; }
    part_max[blockIdx.x] = tm;
    part_sum[blockIdx.x] = ts;
  }
}

// host copy of a device double
rso_status read_d(rso_handle* h, const double* dev, double* out) {
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(out, dev, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

rso_status maxabs(rso_handle* h, long long n, int dense, const float* a, float* out) {
  k_oc_maxabs<<<OC_BLOCKS, OC_THREADS, 0, h->stream>>>(n, h->L[0], dense, a, h->red); note_launch();
  k_oc_maxfinal<<<1, 512, 0, h->stream>>>(h->red, OC_BLOCKS, h->scal + 14); note_launch();
  RSO_TRY(launch_check(h, "oc maxabs"));
  double m = 0;
  RSO_TRY(read_d(h, h->scal + 14, &m));
  *out = (float)m;
  return RSO_OK;
}

// one trial; returns the volume fraction (FP32, as the reference's Vratio)
rso_status trial(rso_handle* h, long long n, int dense, const float* src, const float* sens, float g, float step,
                 float damp, float lo, float hi, const uint8_t* shell, float* out, double denom, float* vratio) {
  k_oc_try<<<OC_BLOCKS, OC_THREADS, 0, h->stream>>>(n, h->L[0], dense, src, sens, g, step, damp, lo, hi, shell, out,
                                                    h->red);
  note_launch();
  RSO_TRY(launch_check(h, "oc trial"));
  RSO_TRY(reduce_partials(h, h->red, OC_BLOCKS, h->scal + 14));
  double s = 0;
  RSO_TRY(read_d(h, h->scal + 14, &s));
  *vratio = (float)(s / denom);
  return RSO_OK;
}

}  // namespace
}  // namespace rso

using namespace rso;

extern "C" rso_status rso_oc_update_density(rso_handle* h, int variant, const float* rho_src_dev,
                                            const float* sens_dev, const uint8_t* shell_dev, double vgoal,
                                            double step, double damp, float* rho_out_dev, double* info_host) {
  if (!h || !rho_src_dev || !sens_dev || !rho_out_dev || (variant != 0 && variant != 1)) return RSO_ERR_INVALID_ARG;
  const Level& l = h->L[0];
  const long long n = l.ne;
  const double denom = (double)l.n_active_e;
  if (denom <= 0) { h->err = "no active elements"; return RSO_ERR_STATE; }
  float gmax = 0;
  RSO_TRY(maxabs(h, n, 1, sens_dev, &gmax));
  const float goal = (float)vgoal, st = (float)step, dp = (float)damp, rmin = (float)h->cfg.rho_min;
  float lo = 0.f, hi = gmax, g = (lo + hi) / 2, V = 2.f;
  float* tmp = h->e_c;  // trial densities (dense order; the buffer holds NQ >= ne floats)
  int itn = 0, trials = 0;
  do {
    g = (lo + hi) / 2;
    RSO_TRY(trial(h, n, 1, rho_src_dev, sens_dev, g, st, dp, rmin, 1.f, shell_dev, tmp, denom, &V));
    trials++;
    if (V > goal) lo = g;
    else if (V < goal) hi = g;
  } while (variant == 0 ? (std::fabs(V - goal) > 1e-4f && itn++ < 30)
                        : (std::fabs(V - goal) > 1e-4f && (hi - lo) / (lo + hi) > 1e-3f && itn++ < 50));
  float Vf = 0;
  RSO_TRY(trial(h, n, 1, rho_src_dev, sens_dev, g, st, dp, rmin, 1.f, shell_dev, rho_out_dev, denom, &Vf));
  if (info_host) {
    info_host[0] = g;
    info_host[1] = Vf;
    info_host[2] = trials;
    // largest and mean |change| over all elements
    k_oc_change<<<OC_BLOCKS, OC_THREADS, 0, h->stream>>>(n, rho_out_dev, rho_src_dev, h->red, h->red + OC_BLOCKS);
    note_launch();
    RSO_TRY(launch_check(h, "oc change"));
    k_oc_maxfinal<<<1, 512, 0, h->stream>>>(h->red, OC_BLOCKS, h->scal + 14); note_launch();
    RSO_TRY(reduce_partials(h, h->red + OC_BLOCKS, OC_BLOCKS, h->scal + 13));
    double m = 0, s = 0;
    RSO_TRY(read_d(h, h->scal + 14, &m));
    RSO_TRY(read_d(h, h->scal + 13, &s));
    info_host[3] = m;
    info_host[4] = s / (double)n;
  }
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_oc_update_coeff(rso_handle* h, float* coeff_dev, const float* csens_dev, double vgoal,
                                          double step, double damp, double cmin, double cmax, float* rho_out_dev,
                                          double* info_host) {
  if (!h || !coeff_dev || !csens_dev) return RSO_ERR_INVALID_ARG;
  if (!h->sp.order) { h->err = "spline not set up"; return RSO_ERR_STATE; }
  const Level& l = h->L[0];
  const long long nc = h->sp.n_coeff;
  const double denom = (double)l.n_active_e;
  float gmax = 0;
  RSO_TRY(maxabs(h, nc, 0, csens_dev, &gmax));
  // the search varies the coefficients from a copy of the incoming ones
  float* copy = h->e_c;  // holds NQ >= n_coeff floats
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(copy, coeff_dev, sizeof(float) * nc, cudaMemcpyDeviceToDevice, h->stream));
  const float goal = (float)vgoal, st = (float)step, dp = (float)damp, lo_c = (float)cmin, hi_c = (float)cmax;
  float lo = 0.f, hi = gmax, g = (lo + hi) / 2, V = 2.f;
  int itn = 0, trials = 0;
  auto volume_of = [&](const float* c, float* vr) -> rso_status {
    // coeff -> density (the reference's coeff2density), volume over the active elements
    RSO_TRY(to_f64(h, c, h->coef_a, nc));
    RSO_TRY(coeff2density(h, h->coef_a, nullptr, h->e_a));
    RSO_TRY(sum_float(h, h->e_a, l.NQ, h->scal + 14));
    double s = 0;
    RSO_TRY(read_d(h, h->scal + 14, &s));
    *vr = (float)(s / denom);
    return RSO_OK;
  };
  do {
    g = (lo + hi) / 2;
    float unused = 0;
    RSO_TRY(trial(h, nc, 0, copy, csens_dev, g, st, dp, lo_c, hi_c, nullptr, coeff_dev, 1.0, &unused));
    RSO_TRY(volume_of(coeff_dev, &V));
    trials++;
    if (V > goal) lo = g;
    else if (V < goal) hi = g;
  } while (std::fabs(V - goal) > 1e-4f && itn++ < 30);
  // the reference applies the final threshold to the last trial's
  // coefficients (not to the incoming ones) and maps them to densities
  float unused = 0;
  RSO_TRY(trial(h, nc, 0, coeff_dev, csens_dev, g, st, dp, lo_c, hi_c, nullptr, coeff_dev, 1.0, &unused));
  float Vf = 0;
  RSO_TRY(volume_of(coeff_dev, &Vf));
  if (rho_out_dev) RSO_TRY(unpad_elems_f(h, h->e_a, rho_out_dev));
  if (info_host) {
    info_host[0] = g;
    info_host[1] = Vf;
    info_host[2] = trials;
  }
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}
