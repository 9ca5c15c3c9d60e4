// FP64 reductions (warp-shuffle trees, deterministic two-pass), layout
// conversions between the public dense layout and the padded device layout,
// and small elementwise helpers.
#include "rso_internal.cuh"

namespace rso {

constexpr int RED_BLOCKS = 592;  // 4 x 148 SMs
constexpr int RED_THREADS = 512;

rso_status launch_check(rso_handle* h, const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    h->err = std::string(what) + ": " + cudaGetErrorString(e);
    return RSO_ERR_CUDA;
  }
  return RSO_OK;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double ws[32];
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) ws[w] = v;
  __syncthreads();
  v = (threadIdx.x < blockDim.x / 32) ? ws[lane] : 0.0;
  if (w == 0) v = warp_sum(v);
  __syncthreads();
  return v;
}

__global__ void __launch_bounds__(RED_THREADS) k_dot_partial(const double* __restrict__ a, const double* __restrict__ b,
                                                             long long n, double* __restrict__ part) {
  double s = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s += a[i] * b[i];
  s = block_sum(s);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void __launch_bounds__(RED_THREADS) k_sumf_partial(const float* __restrict__ a, long long n,
                                                              double* __restrict__ part) {
  double s = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s += (double)a[i];
  s = block_sum(s);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void __launch_bounds__(RED_THREADS) k_final(const double* __restrict__ part, int np, double* out) {
  double s = 0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) s += part[i];
  s = block_sum(s);
  if (threadIdx.x == 0) *out = s;
}

rso_status dot(rso_handle* h, const double* a, const double* b, long long n, double* dev_out) {
  k_dot_partial<<<RED_BLOCKS, RED_THREADS, 0, h->stream>>>(a, b, n, h->red); rso::note_launch();
  k_final<<<1, RED_THREADS, 0, h->stream>>>(h->red, RED_BLOCKS, dev_out); rso::note_launch();
  return launch_check(h, "dot");
}

// CG residual step fused with its norm: r -= a q, sum r.r, and (mixed
// precision) the FP32 copy of r that the V-cycle smooths.  The matching
// x += a p is deferred to the direction update, which reads p anyway.
__global__ void __launch_bounds__(RED_THREADS) k_cg_resid_rr(long long n, const double* __restrict__ alpha,
                                                             const double* __restrict__ q, double* __restrict__ r,
                                                             float* __restrict__ r32, double* __restrict__ part) {
  const double a = *alpha;
  double s = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double ri = r[i] - a * q[i];
    r[i] = ri;
    if (r32) r32[i] = (float)ri;
    s += ri * ri;
  }
  s = block_sum(s);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// sum a.b with b in FP32 (the mixed-precision preconditioned residual)
__global__ void __launch_bounds__(RED_THREADS) k_dot_df_partial(const double* __restrict__ a,
                                                                const float* __restrict__ b, long long n,
                                                                double* __restrict__ part) {
  double s = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s += a[i] * (double)b[i];
  s = block_sum(s);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

rso_status cg_resid_rr(rso_handle* h, long long n, const double* alpha, const double* q, double* r, float* r32,
                       double* rr_dev) {
  k_cg_resid_rr<<<RED_BLOCKS, RED_THREADS, 0, h->stream>>>(n, alpha, q, r, r32, h->red); rso::note_launch();
  k_final<<<1, RED_THREADS, 0, h->stream>>>(h->red, RED_BLOCKS, rr_dev); rso::note_launch();
  return launch_check(h, "cg_resid_rr");
}

// FP32 Krylov recurrence (reliable-update PCG): r -= a q in FP32 with the
// sum r.r in FP64, and a.b of two FP32 vectors summed in FP64; 16-byte
// vectors (3 NP is a multiple of 4 and the buffers are 256-byte aligned)
__global__ void __launch_bounds__(RED_THREADS) k_cg32_resid_rr(long long n4, const double* __restrict__ alpha,
                                                               const float4* __restrict__ q, float4* __restrict__ r,
                                                               double* __restrict__ part) {
  const float a = (float)*alpha;
  double s = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
    const float4 qi = q[i];
    float4 ri = r[i];
    ri.x -= a * qi.x;
    ri.y -= a * qi.y;
    ri.z -= a * qi.z;
    ri.w -= a * qi.w;
    r[i] = ri;
    s += (double)ri.x * ri.x + (double)ri.y * ri.y + (double)ri.z * ri.z + (double)ri.w * ri.w;
  }
  s = block_sum(s);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void __launch_bounds__(RED_THREADS) k_dot_ff_partial(const float4* __restrict__ a,
                                                                const float4* __restrict__ b, long long n4,
                                                                double* __restrict__ part) {
  double s = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
    const float4 x = a[i], y = b[i];
    s += (double)x.x * y.x + (double)x.y * y.y + (double)x.z * y.z + (double)x.w * y.w;
  }
  s = block_sum(s);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

rso_status cg32_resid_rr(rso_handle* h, long long n, const double* alpha, const float* q, float* r, double* rr_dev) {
  if ((n & 3) || ((reinterpret_cast<uintptr_t>(q) | reinterpret_cast<uintptr_t>(r)) & 15)) {
    h->err = "cg32_resid_rr: vectors must be 16-byte aligned multiples of 4 entries";
    return RSO_ERR_STATE;
  }
  k_cg32_resid_rr<<<RED_BLOCKS, RED_THREADS, 0, h->stream>>>(n / 4, alpha, reinterpret_cast<const float4*>(q),
                                                              reinterpret_cast<float4*>(r), h->red);
  rso::note_launch();
  k_final<<<1, RED_THREADS, 0, h->stream>>>(h->red, RED_BLOCKS, rr_dev); rso::note_launch();
  return launch_check(h, "cg32_resid_rr");
}

rso_status dot_ff(rso_handle* h, const float* a, const float* b, long long n, double* dev_out) {
  if ((n & 3) || ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15)) {
    h->err = "dot_ff: vectors must be 16-byte aligned multiples of 4 entries";
    return RSO_ERR_STATE;
  }
  k_dot_ff_partial<<<RED_BLOCKS, RED_THREADS, 0, h->stream>>>(reinterpret_cast<const float4*>(a),
                                                               reinterpret_cast<const float4*>(b), n / 4, h->red);
  rso::note_launch();
  k_final<<<1, RED_THREADS, 0, h->stream>>>(h->red, RED_BLOCKS, dev_out); rso::note_launch();
  return launch_check(h, "dot_ff");
}

// one sum per system: out[b * stride] = sum of part[b * nper .. (b + 1) * nper)
__global__ void __launch_bounds__(RED_THREADS) k_final_batch(const double* __restrict__ part, int nper,
                                                             double* __restrict__ out, int stride) {
  const double* p = part + (long long)blockIdx.x * nper;
  double s = 0;
  for (int i = threadIdx.x; i < nper; i += blockDim.x) s += p[i];
  s = block_sum(s);
  if (threadIdx.x == 0) out[(long long)blockIdx.x * stride] = s;
}

rso_status reduce_partials_batch(rso_handle* h, const double* part, int nper, int nb, double* dev_out, int stride) {
  k_final_batch<<<nb, RED_THREADS, 0, h->stream>>>(part, nper, dev_out, stride); rso::note_launch();
  return launch_check(h, "reduce_partials_batch");
}

rso_status reduce_partials(rso_handle* h, const double* part, int n, double* dev_out) {
  k_final<<<1, RED_THREADS, 0, h->stream>>>(part, n, dev_out); rso::note_launch();
  return launch_check(h, "reduce_partials");
}

// power-iteration step in FP32: r = u - t (t = u - D^-1 K u), with the sums
// u.u and r.r accumulated in FP64 and returned to the host
__global__ void __launch_bounds__(RED_THREADS) k_pow_step(long long n, const float* __restrict__ u,
                                                          const float* __restrict__ t, float* __restrict__ r,
                                                          double* __restrict__ part) {
  double su = 0, sr = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float ui = u[i], ri = ui - t[i];
    r[i] = ri;
    su += (double)ui * ui;
    sr += (double)ri * ri;
  }
  su = block_sum(su);
  sr = block_sum(sr);
  if (threadIdx.x == 0) { part[blockIdx.x] = su; part[RED_BLOCKS + blockIdx.x] = sr; }
}

rso_status pow_step(rso_handle* h, long long n, const float* u, const float* t, float* r, double* uu, double* rr) {
  k_pow_step<<<RED_BLOCKS, RED_THREADS, 0, h->stream>>>(n, u, t, r, h->red); rso::note_launch();
  k_final<<<1, RED_THREADS, 0, h->stream>>>(h->red, RED_BLOCKS, h->scal + 6); rso::note_launch();
  k_final<<<1, RED_THREADS, 0, h->stream>>>(h->red + RED_BLOCKS, RED_BLOCKS, h->scal + 7); rso::note_launch();
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(h->h_scal + 6, h->scal + 6, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  *uu = h->h_scal[6];
  *rr = h->h_scal[7];
  return RSO_OK;
}

rso_status dot_df(rso_handle* h, const double* a, const float* b, long long n, double* dev_out) {
  k_dot_df_partial<<<RED_BLOCKS, RED_THREADS, 0, h->stream>>>(a, b, n, h->red); rso::note_launch();
  k_final<<<1, RED_THREADS, 0, h->stream>>>(h->red, RED_BLOCKS, dev_out); rso::note_launch();
  return launch_check(h, "dot_df");
}

rso_status dot_host(rso_handle* h, const double* a, const double* b, long long n, double* out) {
  RSO_TRY(dot(h, a, b, n, h->scal + 15));
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(h->h_scal + 15, h->scal + 15, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  *out = h->h_scal[15];
  return RSO_OK;
}

rso_status sum_float(rso_handle* h, const float* a, long long n, double* dev_out) {
  k_sumf_partial<<<RED_BLOCKS, RED_THREADS, 0, h->stream>>>(a, n, h->red); rso::note_launch();
  k_final<<<1, RED_THREADS, 0, h->stream>>>(h->red, RED_BLOCKS, dev_out); rso::note_launch();
  return launch_check(h, "sum_float");
}

// ---------------------------------------------------------------- layouts
__global__ void k_pad_nodes(Level L, const double* __restrict__ dense, double* __restrict__ pad, int to_pad) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= L.nn) return;
  int x = i % L.nx, y = (i / L.nx) % L.ny, z = i / ((long long)L.nx * L.ny);
  long long j = L.nidx(x, y, z);
  for (int c = 0; c < 3; c++) {
    if (to_pad) pad[j + c * L.NP] = dense[i + c * L.nn];
    else pad[i + c * L.nn] = dense[j + c * L.NP];  // 'dense' is the padded source here
  }
}

rso_status pad_nodes(rso_handle* h, int level, const double* dense, double* padded) {
  const Level& l = h->L[level];
  RSO_CHECK_CUDA(h, cudaMemsetAsync(padded, 0, sizeof(double) * 3 * l.NP, h->stream));
  k_pad_nodes<<<cdiv(l.nn, 256), 256, 0, h->stream>>>(l, dense, padded, 1); rso::note_launch();
  return launch_check(h, "pad_nodes");
}

rso_status unpad_nodes(rso_handle* h, int level, const double* padded, double* dense) {
  const Level& l = h->L[level];
  k_pad_nodes<<<cdiv(l.nn, 256), 256, 0, h->stream>>>(l, padded, dense, 0); rso::note_launch();
  return launch_check(h, "unpad_nodes");
}

__global__ void k_pad_elems(Level L, const float* __restrict__ src, float* __restrict__ dst, int to_pad) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= L.ne) return;
  int x = i % L.ex, y = (i / L.ex) % L.ey, z = i / ((long long)L.ex * L.ey);
  long long j = L.eidx(x, y, z);
  if (to_pad) dst[j] = L.emask[j] ? src[i] : 0.f;
  else dst[i] = L.emask[j] ? src[j] : 0.f;
}

rso_status pad_elems_f(rso_handle* h, const float* dense, float* padded) {
  const Level& l = h->L[0];
  RSO_CHECK_CUDA(h, cudaMemsetAsync(padded, 0, sizeof(float) * l.NQ, h->stream));
  k_pad_elems<<<cdiv(l.ne, 256), 256, 0, h->stream>>>(l, dense, padded, 1); rso::note_launch();
  return launch_check(h, "pad_elems");
}

rso_status unpad_elems_f(rso_handle* h, const float* padded, float* dense) {
  const Level& l = h->L[0];
  k_pad_elems<<<cdiv(l.ne, 256), 256, 0, h->stream>>>(l, padded, dense, 0); rso::note_launch();
  return launch_check(h, "unpad_elems");
}

// zero the support DOFs (and inactive nodes) of a padded fine vector
__global__ void k_zero_support(Level L, double* v) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= L.NP) return;
  uint8_t c = L.vclass[i];
  if (!(c & NC_ACTIVE) || (c & NC_SUPPORT)) { v[i] = 0; v[i + L.NP] = 0; v[i + 2 * L.NP] = 0; }
}

rso_status zero_support(rso_handle* h, double* padded) {
  const Level& l = h->L[0];
  k_zero_support<<<cdiv(l.NP, 256), 256, 0, h->stream>>>(l, padded); rso::note_launch();
  return launch_check(h, "zero_support");
}

// ---------------------------------------------------------------- elementwise
__global__ void k_axpby(long long n, double a, const double* __restrict__ x, double b, double* __restrict__ y) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) y[i] = a * x[i] + b * y[i];
}
rso_status axpby(rso_handle* h, long long n, double a, const double* x, double b, double* y) {
  k_axpby<<<cdiv(n, 256), 256, 0, h->stream>>>(n, a, x, b, y); rso::note_launch();
  return launch_check(h, "axpby");
}

__global__ void k_fill_d(double* p, long long n, double v) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}
__global__ void k_fill_f(float* p, long long n, float v) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}
rso_status fill_d(rso_handle* h, double* p, long long n, double v) {
  k_fill_d<<<cdiv(n, 256), 256, 0, h->stream>>>(p, n, v); rso::note_launch();
  return launch_check(h, "fill_d");
}
rso_status fill_f(rso_handle* h, float* p, long long n, float v) {
  k_fill_f<<<cdiv(n, 256), 256, 0, h->stream>>>(p, n, v); rso::note_launch();
  return launch_check(h, "fill_f");
}

}  // namespace rso
