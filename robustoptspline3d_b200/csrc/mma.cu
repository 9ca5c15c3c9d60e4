// Svanberg MMA (the reference's mma_t: optimization/mma_t.h:159-266,
// mma_t.cpp:18-118, mma_t.cu:15-909) in FP64 on the device.  The n-sized
// work (asymptotes, p/q, the reduced-system sums, the step bounds and the
// KKT residual of every line-search trial) runs in fused kernels with
// deterministic two-pass reductions; the (m+1)^2 dual system and the
// m-sized bookkeeping run on the host, as the reference does with Eigen.
#include "rso_internal.cuh"
#include <cmath>
#include <vector>
#include <algorithm>

constexpr int MMA_MAXM = 8;
constexpr int MMA_RED = 40;   // max reductions in one pass
constexpr int MMA_BLOCKS = 256;
constexpr int MMA_THREADS = 256;

struct rso_mma {
  int n = 0, m = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  double *x = nullptr, *xmin = nullptr, *xmax = nullptr, *L = nullptr, *U = nullptr, *alpha = nullptr,
         *beta = nullptr, *lastdx = nullptr, *xi = nullptr, *eta = nullptr, *curx = nullptr;
  double *P = nullptr, *Q = nullptr, *Dx = nullptr, *hdx = nullptr, *G = nullptr, *dx = nullptr, *dxi = nullptr,
         *deta = nullptr;
  double *part = nullptr, *res = nullptr, *h_res = nullptr;
  std::vector<double> y, lambda, mu, s, a, c, d, b, lam_pq;
  double z = 1, zeta = 1, a0 = 1, eps = 1;
  int stop_counter = 0;
};

namespace {

struct MPar {
  int n, m;
  double eps;
  double lam[MMA_MAXM];
  double dl[MMA_MAXM];
  double step;
};

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double wmax(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// reduce R values per thread over the block; op 0 sum, 1 max; partial[r * gridDim.x + block]
template <int R>
__device__ void block_reduce(double (&v)[R], const int* ops, int nr, double* part) {
  __shared__ double sh[MMA_RED][MMA_THREADS / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int r = 0; r < nr; r++) {
    const double t = ops[r] ? wmax(v[r]) : wsum(v[r]);
    if (lane == 0) sh[r][w] = t;
  }
  __syncthreads();
  if (threadIdx.x < nr) {
    const int r = threadIdx.x;
    double acc = ops[r] ? -1e300 : 0.0;
    for (int k = 0; k < MMA_THREADS / 32; k++) acc = ops[r] ? fmax(acc, sh[r][k]) : acc + sh[r][k];
    part[(long long)r * gridDim.x + blockIdx.x] = acc;
  }
}

__global__ void k_final(const double* part, int nblocks, int nr, const int* ops_dummy, int opmask_lo,
                        int opmask_hi, double* out) {
  const int r = threadIdx.x;
  if (r >= nr) return;
  const bool mx = r < 32 ? ((opmask_lo >> r) & 1) : ((opmask_hi >> (r - 32)) & 1);
  double acc = mx ? -1e300 : 0.0;
  for (int b = 0; b < nblocks; b++) acc = mx ? fmax(acc, part[(long long)r * nblocks + b]) : acc + part[(long long)r * nblocks + b];
  out[r] = acc;
}

__global__ void k_pq(int n, int m, const double* __restrict__ df, const double* __restrict__ dg,
                     const double* __restrict__ x, const double* __restrict__ L, const double* __restrict__ U,
                     const double* __restrict__ xmin, const double* __restrict__ xmax, double* __restrict__ P,
                     double* __restrict__ Q) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double ux = U[i] - x[i], xl = x[i] - L[i], raa = 1e-5 / (xmax[i] - xmin[i]);
    for (int j = 0; j <= m; j++) {
      const double d = j == 0 ? df[i] : dg[(long long)(j - 1) * n + i];
      const double pos = fmax(d, 0.0), neg = fmax(-d, 0.0);
      P[(long long)j * n + i] = ux * ux * (1.001 * pos + 0.001 * neg + raa);
      Q[(long long)j * n + i] = xl * xl * (0.001 * pos + 1.001 * neg + raa);
    }
  }
}

// gproxy_j = sum p_{j+1}/(U-x) + q_{j+1}/(x-L)
__global__ void __launch_bounds__(MMA_THREADS) k_gp(MPar p, const double* __restrict__ x, const double* __restrict__ L,
                                                    const double* __restrict__ U, const double* __restrict__ P,
                                                    const double* __restrict__ Q, double* part) {
  double v[MMA_MAXM] = {0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < p.n; i += (long long)gridDim.x * blockDim.x) {
    const double ux = U[i] - x[i], xl = x[i] - L[i];
    for (int j = 0; j < p.m; j++) v[j] += P[(long long)(j + 1) * p.n + i] / ux + Q[(long long)(j + 1) * p.n + i] / xl;
  }
  int ops[MMA_MAXM] = {0};
  block_reduce<MMA_MAXM>(v, ops, p.m, part);
}

__global__ void k_reset(int n, double* x, const double* alpha, const double* beta, double* xi, double* eta) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double xv = 0.5 * (alpha[i] + beta[i]);
    x[i] = xv;
    xi[i] = fmax(1.0 / (xv - alpha[i]), 1.0);
    eta[i] = fmax(1.0 / (beta[i] - xv), 1.0);
  }
}

// Newton system sums: A11[j][k] = sum G_j G_k / Dx, s_j = sum G_j hdx/Dx, gp_j
__global__ void __launch_bounds__(MMA_THREADS) k_prep(MPar p, const double* __restrict__ x, const double* __restrict__ L,
                                                      const double* __restrict__ U, const double* __restrict__ alpha,
                                                      const double* __restrict__ beta, const double* __restrict__ xi,
                                                      const double* __restrict__ eta, const double* __restrict__ P,
                                                      const double* __restrict__ Q, double* __restrict__ Dx,
                                                      double* __restrict__ hdx, double* __restrict__ G, double* part) {
  double v[MMA_RED];
  for (int r = 0; r < MMA_RED; r++) v[r] = 0;
  const int m = p.m, n = p.n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double ux = U[i] - x[i], xl = x[i] - L[i];
    double pl = P[i], ql = Q[i];
    for (int j = 0; j < m; j++) { pl += p.lam[j] * P[(long long)(j + 1) * n + i]; ql += p.lam[j] * Q[(long long)(j + 1) * n + i]; }
    const double psi = 2 * pl / (ux * ux * ux) + 2 * ql / (xl * xl * xl);
    const double dxv = psi + xi[i] / (x[i] - alpha[i]) + eta[i] / (beta[i] - x[i]);
    const double varphi = pl / (ux * ux) - ql / (xl * xl);
    const double h = -(p.eps / (x[i] - alpha[i]) - p.eps / (beta[i] - x[i]) - varphi);
    Dx[i] = dxv;
    hdx[i] = h;
    double g[MMA_MAXM];
    for (int j = 0; j < m; j++) {
      g[j] = P[(long long)(j + 1) * n + i] / (ux * ux) - Q[(long long)(j + 1) * n + i] / (xl * xl);
      G[(long long)j * n + i] = g[j];
    }
    int r = 0;
    for (int j = 0; j < m; j++)
      for (int k = 0; k < m; k++) v[r++] += g[j] * (g[k] / dxv);
    for (int j = 0; j < m; j++) v[r++] += g[j] * (h / dxv);
    for (int j = 0; j < m; j++) v[r++] += P[(long long)(j + 1) * n + i] / ux + Q[(long long)(j + 1) * n + i] / xl;
  }
  int ops[MMA_RED] = {0};
  block_reduce<MMA_RED>(v, ops, m * m + 2 * m, part);
}

// search direction in x and the bound multipliers, with the step bounds
__global__ void __launch_bounds__(MMA_THREADS) k_dir(MPar p, const double* __restrict__ x,
                                                     const double* __restrict__ alpha, const double* __restrict__ beta,
                                                     const double* __restrict__ xi, const double* __restrict__ eta,
                                                     const double* __restrict__ Dx, const double* __restrict__ hdx,
                                                     const double* __restrict__ G, double* __restrict__ dx,
                                                     double* __restrict__ dxi, double* __restrict__ deta, double* part) {
  double v[4] = {-1e300, -1e300, -1e300, -1e300};
  const double cf = 0.99;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < p.n; i += (long long)gridDim.x * blockDim.x) {
    double t = -hdx[i] / Dx[i];
    for (int j = 0; j < p.m; j++) t -= p.dl[j] * G[(long long)j * p.n + i] / Dx[i];
    const double xa = x[i] - alpha[i], bx = beta[i] - x[i];
    const double di = p.eps / xa - t / xa * xi[i] - xi[i];
    const double de = p.eps / bx + eta[i] / bx * t - eta[i];
    dx[i] = t; dxi[i] = di; deta[i] = de;
    v[0] = fmax(v[0], (-1 / cf) * (t / xa));
    v[1] = fmax(v[1], (1 / cf) * (t / bx));
    v[2] = fmax(v[2], (-1 / cf) * di / xi[i]);
    v[3] = fmax(v[3], (-1 / cf) * de / eta[i]);
  }
  int ops[4] = {1, 1, 1, 1};
  block_reduce<4>(v, ops, 4, part);
}

// KKT residual pieces at x + step dx (step = 0: current point)
__global__ void __launch_bounds__(MMA_THREADS) k_kkt(MPar p, const double* __restrict__ x, const double* __restrict__ L,
                                                     const double* __restrict__ U, const double* __restrict__ alpha,
                                                     const double* __restrict__ beta, const double* __restrict__ xi,
                                                     const double* __restrict__ eta, const double* __restrict__ dx,
                                                     const double* __restrict__ dxi, const double* __restrict__ deta,
                                                     const double* __restrict__ P, const double* __restrict__ Q,
                                                     double* part) {
  // 0: sum rex^2, 1: sum rexsi^2, 2: sum reeta^2, 3..3+m-1: g_j; 3+m..5+m: max |.|
  double v[3 + MMA_MAXM + 3];
  for (int r = 0; r < 3 + MMA_MAXM + 3; r++) v[r] = 0;
  const int m = p.m, n = p.n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double xt = x[i] + p.step * dx[i];
    const double xit = xi[i] + p.step * dxi[i];
    const double et = eta[i] + p.step * deta[i];
    const double ux = U[i] - xt, xl = xt - L[i];
    double pl = P[i], ql = Q[i];
    for (int j = 0; j < m; j++) { pl += p.lam[j] * P[(long long)(j + 1) * n + i]; ql += p.lam[j] * Q[(long long)(j + 1) * n + i]; }
    const double rex = pl / (ux * ux) - ql / (xl * xl) - xit + et;
    const double rxs = xit * (xt - alpha[i]) - p.eps;
    const double ret = et * (beta[i] - xt) - p.eps;
    v[0] += rex * rex; v[1] += rxs * rxs; v[2] += ret * ret;
    for (int j = 0; j < m; j++) v[3 + j] += P[(long long)(j + 1) * n + i] / ux + Q[(long long)(j + 1) * n + i] / xl;
    v[3 + m] = fmax(v[3 + m], fabs(rex));
    v[4 + m] = fmax(v[4 + m], fabs(rxs));
    v[5 + m] = fmax(v[5 + m], fabs(ret));
  }
  int ops[3 + MMA_MAXM + 3];
  for (int r = 0; r < 3 + MMA_MAXM + 3; r++) ops[r] = r >= 3 + m ? 1 : 0;
  block_reduce<3 + MMA_MAXM + 3>(v, ops, 6 + m, part);
}

__global__ void k_accept(int n, double step, double* x, double* xi, double* eta, const double* dx, const double* dxi,
                         const double* deta) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    x[i] += step * dx[i]; xi[i] += step * dxi[i]; eta[i] += step * deta[i];
  }
}

// adjust_asym (mma_t.cu:164-226) and |dx|^2
__global__ void __launch_bounds__(MMA_THREADS) k_asym(int n, const double* __restrict__ x, const double* __restrict__ curx,
                                                      double* __restrict__ lastdx, double* __restrict__ L,
                                                      double* __restrict__ U, double* __restrict__ alpha,
                                                      double* __restrict__ beta, const double* __restrict__ xmin,
                                                      const double* __restrict__ xmax, double* part) {
  double v[1] = {0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double d1 = x[i] - curx[i], d2 = lastdx[i];
    double gamma = 1;
    if (d1 * d2 > 0) gamma = 1.2;
    if (d1 * d2 < 0) gamma = 0.7;
    const double xv = x[i], st = xmax[i] - xmin[i];
    double nl = xv - gamma * (xv - d1 - L[i]);
    double nu = xv + gamma * (U[i] - xv + d1);
    nl = fmin(fmax(nl, xv - 10 * st), xv - 0.01 * st);
    nu = fmin(fmax(nu, xv + 0.01 * st), xv + 10 * st);
    L[i] = nl; U[i] = nu;
    double na = xmin[i];
    na = fmax(na, nl + 0.1 * (xv - nl));
    na = fmax(na, xv - 0.5 * st);
    double nb = xmax[i];
    nb = fmin(nb, nu - 0.1 * (nu - xv));
    nb = fmin(nb, xv + 0.5 * st);
    alpha[i] = na; beta[i] = nb;
    lastdx[i] = d1;
    v[0] += d1 * d1;
  }
  int ops[1] = {0};
  block_reduce<1>(v, ops, 1, part);
}

// clamp_asymptotes (mma_t.cu:747-761)
__global__ void k_clamp_asym(int n, const double* x, double* L, double* U, double* alpha, double* beta,
                             const double* xmin, const double* xmax) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double st = xmax[i] - xmin[i], xv = x[i];
    L[i] = fmin(fmax(L[i], xv - 10 * st), xv - 0.01 * st);
    U[i] = fmin(fmax(U[i], xv + 0.01 * st), xv + 10 * st);
    alpha[i] = fmax(xmin[i], fmax(L[i] + 0.1 * (xv - L[i]), xv - 0.5 * st));
    beta[i] = fmin(xmax[i], fmin(U[i] - 0.1 * (U[i] - xv), xv + 0.5 * st));
  }
}

#define MMA_CHECK(s, call)                                                         \
  do {                                                                             \
    cudaError_t _e = (call);                                                       \
    if (_e != cudaSuccess) { (s)->err = cudaGetErrorString(_e); return RSO_ERR_CUDA; } \
  } while (0)

// run one reduction pass's final stage and copy nr results to the host
rso_status finish_red(rso_mma* s, int nr, unsigned long long maxmask) {
  k_final<<<1, 64, 0, s->stream>>>(s->part, MMA_BLOCKS, nr, nullptr, (int)(maxmask & 0xffffffffu),
                                   (int)(maxmask >> 32), s->res); rso::note_launch();
  MMA_CHECK(s, cudaGetLastError());
  MMA_CHECK(s, cudaMemcpyAsync(s->h_res, s->res, sizeof(double) * nr, cudaMemcpyDeviceToHost, s->stream));
  MMA_CHECK(s, cudaStreamSynchronize(s->stream));
  return RSO_OK;
}

void dense_solve(int N, std::vector<double> A, std::vector<double> b, std::vector<double>& x) {
  for (int k = 0; k < N; k++) {
    int piv = k;
    for (int i = k + 1; i < N; i++) if (std::fabs(A[i * N + k]) > std::fabs(A[piv * N + k])) piv = i;
    if (piv != k) { for (int j = 0; j < N; j++) std::swap(A[k * N + j], A[piv * N + j]); std::swap(b[k], b[piv]); }
    for (int i = k + 1; i < N; i++) {
      const double f = A[i * N + k] / A[k * N + k];
      for (int j = k; j < N; j++) A[i * N + j] -= f * A[k * N + j];
      b[i] -= f * b[k];
    }
  }
  x.assign(N, 0.0);
  for (int i = N - 1; i >= 0; i--) {
    double t = b[i];
    for (int j = i + 1; j < N; j++) t -= A[i * N + j] * x[j];
    x[i] = t / A[i * N + i];
  }
}

MPar mpar(rso_mma* s, const std::vector<double>& lam) {
  MPar p;
  p.n = s->n; p.m = s->m; p.eps = s->eps; p.step = 0;
  for (int j = 0; j < MMA_MAXM; j++) { p.lam[j] = j < s->m ? lam[j] : 0; p.dl[j] = 0; }
  return p;
}

}  // namespace

extern "C" rso_status rso_mma_create(int n, int m, const double* xmin, const double* xmax, rso_mma** out) {
  if (!out || n <= 0 || m < 1 || m > MMA_MAXM || !xmin || !xmax) return RSO_ERR_INVALID_ARG;
  if (m * m + 2 * m > MMA_RED) return RSO_ERR_INVALID_ARG;
  rso_mma* s = new rso_mma();
  s->n = n; s->m = m;
  auto fail = [&](rso_status st) { rso_mma_destroy(s); return st; };
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(RSO_ERR_CUDA);
  double** vecs[] = {&s->x, &s->xmin, &s->xmax, &s->L, &s->U, &s->alpha, &s->beta, &s->lastdx, &s->xi, &s->eta,
                     &s->curx, &s->Dx, &s->hdx, &s->dx, &s->dxi, &s->deta};
  for (double** v : vecs)
    if (cudaMalloc(v, sizeof(double) * n) != cudaSuccess) return fail(RSO_ERR_OOM);
  if (cudaMalloc(&s->P, sizeof(double) * n * (m + 1)) != cudaSuccess) return fail(RSO_ERR_OOM);
  if (cudaMalloc(&s->Q, sizeof(double) * n * (m + 1)) != cudaSuccess) return fail(RSO_ERR_OOM);
  if (cudaMalloc(&s->G, sizeof(double) * n * m) != cudaSuccess) return fail(RSO_ERR_OOM);
  if (cudaMalloc(&s->part, sizeof(double) * MMA_RED * MMA_BLOCKS) != cudaSuccess) return fail(RSO_ERR_OOM);
  if (cudaMalloc(&s->res, sizeof(double) * 64) != cudaSuccess) return fail(RSO_ERR_OOM);
  if (cudaMallocHost(&s->h_res, sizeof(double) * 64) != cudaSuccess) return fail(RSO_ERR_OOM);
  cudaMemcpy(s->xmin, xmin, sizeof(double) * n, cudaMemcpyHostToDevice);
  cudaMemcpy(s->xmax, xmax, sizeof(double) * n, cudaMemcpyHostToDevice);
  // set_bound (mma_t.cu:809-819) and init_subproblem_variable (:797-807)
  cudaMemcpy(s->alpha, xmin, sizeof(double) * n, cudaMemcpyHostToDevice);
  cudaMemcpy(s->beta, xmax, sizeof(double) * n, cudaMemcpyHostToDevice);
  cudaMemcpy(s->L, xmin, sizeof(double) * n, cudaMemcpyHostToDevice);
  cudaMemcpy(s->U, xmax, sizeof(double) * n, cudaMemcpyHostToDevice);
  cudaMemset(s->lastdx, 0, sizeof(double) * n);
  k_reset<<<MMA_BLOCKS, MMA_THREADS, 0, s->stream>>>(n, s->x, s->alpha, s->beta, s->xi, s->eta); rso::note_launch();
  k_clamp_asym<<<MMA_BLOCKS, MMA_THREADS, 0, s->stream>>>(n, s->x, s->L, s->U, s->alpha, s->beta, s->xmin, s->xmax); rso::note_launch();
  k_reset<<<MMA_BLOCKS, MMA_THREADS, 0, s->stream>>>(n, s->x, s->alpha, s->beta, s->xi, s->eta); rso::note_launch();
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return fail(RSO_ERR_CUDA);
  s->y.assign(m, 1.0); s->lambda.assign(m, 1.0); s->s.assign(m, 1.0); s->mu.assign(m, 0.0);
  s->a.assign(m, 0.0); s->c.assign(m, 10.0); s->d.assign(m, 1.0); s->b.assign(m, 0.0);
  for (int j = 0; j < m; j++) s->mu[j] = std::max(s->c[j] / 2, 1.0);
  s->lam_pq = s->lambda;
  *out = s;
  return RSO_OK;
}

extern "C" rso_status rso_mma_set_x_dev(rso_mma* s, const double* x) {
  if (!s || !x) return RSO_ERR_INVALID_ARG;
  MMA_CHECK(s, cudaMemcpyAsync(s->x, x, sizeof(double) * s->n, cudaMemcpyDeviceToDevice, s->stream));
  k_clamp_asym<<<MMA_BLOCKS, MMA_THREADS, 0, s->stream>>>(s->n, s->x, s->L, s->U, s->alpha, s->beta, s->xmin, s->xmax); rso::note_launch();
  MMA_CHECK(s, cudaStreamSynchronize(s->stream));
  return RSO_OK;
}

extern "C" rso_status rso_mma_set_x(rso_mma* s, const double* x) {
  if (!s || !x) return RSO_ERR_INVALID_ARG;
  MMA_CHECK(s, cudaMemcpyAsync(s->x, x, sizeof(double) * s->n, cudaMemcpyHostToDevice, s->stream));
  k_clamp_asym<<<MMA_BLOCKS, MMA_THREADS, 0, s->stream>>>(s->n, s->x, s->L, s->U, s->alpha, s->beta, s->xmin, s->xmax); rso::note_launch();
  MMA_CHECK(s, cudaStreamSynchronize(s->stream));
  return RSO_OK;
}

extern "C" rso_status rso_mma_get(rso_mma* s, double* x, double* L, double* U, double* al, double* be) {
  if (!s) return RSO_ERR_INVALID_ARG;
  const size_t b = sizeof(double) * s->n;
  if (x) MMA_CHECK(s, cudaMemcpyAsync(x, s->x, b, cudaMemcpyDeviceToHost, s->stream));
  if (L) MMA_CHECK(s, cudaMemcpyAsync(L, s->L, b, cudaMemcpyDeviceToHost, s->stream));
  if (U) MMA_CHECK(s, cudaMemcpyAsync(U, s->U, b, cudaMemcpyDeviceToHost, s->stream));
  if (al) MMA_CHECK(s, cudaMemcpyAsync(al, s->alpha, b, cudaMemcpyDeviceToHost, s->stream));
  if (be) MMA_CHECK(s, cudaMemcpyAsync(be, s->beta, b, cudaMemcpyDeviceToHost, s->stream));
  MMA_CHECK(s, cudaStreamSynchronize(s->stream));
  return RSO_OK;
}

extern "C" const double* rso_mma_x_dev(rso_mma* s) { return s ? s->x : nullptr; }

// checkpoint of what an update carries to the next: x, the asymptotes L and
// U, the move limits alpha and beta, the previous step, the stop counter
extern "C" rso_status rso_mma_state_size(const rso_mma* s, long long* n_doubles) {
  if (!s || !n_doubles) return RSO_ERR_INVALID_ARG;
  *n_doubles = 6LL * s->n + 1;
  return RSO_OK;
}

extern "C" rso_status rso_mma_save(rso_mma* s, double* state_host) {
  if (!s || !state_host) return RSO_ERR_INVALID_ARG;
  const size_t b = sizeof(double) * s->n;
  const double* parts[6] = {s->x, s->L, s->U, s->alpha, s->beta, s->lastdx};
  for (int k = 0; k < 6; k++)
    MMA_CHECK(s, cudaMemcpyAsync(state_host + (size_t)k * s->n, parts[k], b, cudaMemcpyDeviceToHost, s->stream));
  MMA_CHECK(s, cudaStreamSynchronize(s->stream));
  state_host[6LL * s->n] = (double)s->stop_counter;
  return RSO_OK;
}

extern "C" rso_status rso_mma_load(rso_mma* s, const double* state_host) {
  if (!s || !state_host) return RSO_ERR_INVALID_ARG;
  const size_t b = sizeof(double) * s->n;
  double* parts[6] = {s->x, s->L, s->U, s->alpha, s->beta, s->lastdx};
  for (int k = 0; k < 6; k++)
    MMA_CHECK(s, cudaMemcpyAsync(parts[k], state_host + (size_t)k * s->n, b, cudaMemcpyHostToDevice, s->stream));
  MMA_CHECK(s, cudaStreamSynchronize(s->stream));
  s->stop_counter = (int)state_host[6LL * s->n];
  return RSO_OK;
}

extern "C" rso_status rso_mma_update(rso_mma* S, const double* df, const double* dg, const double* g, int* converged,
                                     double* info) {
  if (!S || !df || (!dg && S->m > 0) || !g) return RSO_ERR_INVALID_ARG;
  const int n = S->n, m = S->m;
  cudaStream_t st = S->stream;
  MMA_CHECK(S, cudaMemcpyAsync(S->curx, S->x, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  // init (mma_t.cu:69-106): p, q and the proxy offsets b at the current design
  k_pq<<<MMA_BLOCKS, MMA_THREADS, 0, st>>>(n, m, df, dg, S->x, S->L, S->U, S->xmin, S->xmax, S->P, S->Q); rso::note_launch();
  k_gp<<<MMA_BLOCKS, MMA_THREADS, 0, st>>>(mpar(S, S->lambda), S->x, S->L, S->U, S->P, S->Q, S->part); rso::note_launch();
  RSO_TRY(finish_red(S, m, 0));
  for (int j = 0; j < m; j++) S->b[j] = S->h_res[j] - g[j];
  // reset (mma_t.cu:702-713)
  k_reset<<<MMA_BLOCKS, MMA_THREADS, 0, st>>>(n, S->x, S->alpha, S->beta, S->xi, S->eta); rso::note_launch();
  S->eps = 1; S->zeta = S->z = 1;
  for (int j = 0; j < m; j++) { S->y[j] = 1; S->lambda[j] = 1; S->s[j] = 1; S->mu[j] = std::max(S->c[j] / 2, 1.0); }
  S->lam_pq = S->lambda;

  double err = 1e30, lasterr = 0, step_used = 0;
  int nsub = 0;
  bool overflow = false;
  while (S->eps > 1e-6) {
    err = 1e30;
    double damp = 1;
    int stays = 0;
    while (err > 0.9 * S->eps) {
      // Newton system (solveLinearSystem, mma_t.cu:228-328)
      MPar p = mpar(S, S->lam_pq);
      k_prep<<<MMA_BLOCKS, MMA_THREADS, 0, st>>>(p, S->x, S->L, S->U, S->alpha, S->beta, S->xi, S->eta, S->P, S->Q,
                                                 S->Dx, S->hdx, S->G, S->part); rso::note_launch();
      RSO_TRY(finish_red(S, m * m + 2 * m, 0));
      std::vector<double> A11(m * m), sg(m), gp(m);
      for (int i = 0; i < m * m; i++) A11[i] = S->h_res[i];
      for (int j = 0; j < m; j++) { sg[j] = S->h_res[m * m + j]; gp[j] = S->h_res[m * m + m + j]; }
      std::vector<double> Dy(m), Dl(m), hdy(m), hdl(m);
      double la = 0;
      for (int j = 0; j < m; j++) {
        Dy[j] = S->d[j] + S->mu[j] / S->y[j];
        Dl[j] = S->s[j] / S->lambda[j];
        hdy[j] = -(S->lambda[j] + S->eps / S->y[j] - S->c[j] - S->d[j] * S->y[j]);
        hdl[j] = -(S->z * S->a[j] + S->y[j] + S->b[j] - S->eps / S->lambda[j] - gp[j]);
        la += S->lambda[j] * S->a[j];
      }
      const double hdz = -(la + S->eps / S->z - S->a0);
      const int N = m + 1;
      std::vector<double> A(N * N, 0.0), rhs(N, 0.0), sol;
      for (int j = 0; j < m; j++) {
        A[j * N + j] += Dl[j] + 1 / Dy[j];
        for (int k = 0; k < m; k++) A[j * N + k] += A11[j * m + k];
        rhs[j] = hdl[j] + hdy[j] / Dy[j] - sg[j];
        A[j * N + m] = S->a[j];
        A[m * N + j] = S->a[j];
      }
      A[m * N + m] = -S->zeta / S->z;
      rhs[m] = hdz;
      dense_solve(N, A, rhs, sol);
      const double dz = sol[m];
      std::vector<double> dl(m), dy(m), dmu(m), ds(m);
      for (int j = 0; j < m; j++) {
        dl[j] = sol[j];
        dy[j] = dl[j] / Dy[j] - hdy[j] / Dy[j];
        dmu[j] = S->eps / S->y[j] - dy[j] * S->mu[j] / S->y[j] - S->mu[j];
        ds[j] = S->eps / S->lambda[j] - S->s[j] / S->lambda[j] * dl[j] - S->s[j];
      }
      const double dzeta = S->eps / S->z - S->zeta - (S->zeta / S->z) * dz;
      for (int j = 0; j < m; j++) p.dl[j] = dl[j];
      k_dir<<<MMA_BLOCKS, MMA_THREADS, 0, st>>>(p, S->x, S->alpha, S->beta, S->xi, S->eta, S->Dx, S->hdx, S->G, S->dx,
                                                S->dxi, S->deta, S->part); rso::note_launch();
      RSO_TRY(finish_red(S, 4, 0xfull));
      const double cf = 0.99;
      const double t1 = S->h_res[0], t2 = S->h_res[1];
      double t3 = std::max(S->h_res[2], S->h_res[3]);
      auto art = [&](double dv, double v) { t3 = std::max(t3, (-1 / cf) * dv / v); };
      for (int j = 0; j < m; j++) art(dy[j], S->y[j]);
      art(dz, S->z);
      for (int j = 0; j < m; j++) art(dl[j], S->lambda[j]);
      for (int j = 0; j < m; j++) art(dmu[j], S->mu[j]);
      art(dzeta, S->zeta);
      for (int j = 0; j < m; j++) art(ds[j], S->s[j]);
      const double max_t = 1 / std::max(std::max(t1, t2), std::max(t3, 1.0));
      // search_step (mma_t.cu:501-571) with kkt_err (:574-678)
      auto kkt = [&](double step, const std::vector<double>& lam, const std::vector<double>& yv, double zv,
                     const std::vector<double>& muv, double zetav, const std::vector<double>& sv, double dmp,
                     double* e2, double* einf) -> rso_status {
        MPar q = mpar(S, lam);
        q.step = step;
        k_kkt<<<MMA_BLOCKS, MMA_THREADS, 0, st>>>(q, S->x, S->L, S->U, S->alpha, S->beta, S->xi, S->eta, S->dx, S->dxi,
                                                  S->deta, S->P, S->Q, S->part); rso::note_launch();
        const unsigned long long mm = 0x7ull << (3 + m);
        RSO_TRY(finish_red(S, 6 + m, mm));
        S->lam_pq = lam;  // the reference's kkt_err refreshes plambda/qlambda with the trial multipliers
        double sum = S->h_res[0] + S->h_res[1] + S->h_res[2];
        double mx = std::max(-10.0, std::max(S->h_res[3 + m], std::max(S->h_res[4 + m], S->h_res[5 + m])));
        auto acc = [&](double v) { sum += v * v; mx = std::max(mx, std::fabs(v)); };
        for (int j = 0; j < m; j++) acc(S->c[j] + S->d[j] * yv[j] - lam[j] - muv[j]);
        double l2 = 0;
        for (int j = 0; j < m; j++) l2 += lam[j] * S->a[j];
        acc(S->a0 - zetav - l2);
        for (int j = 0; j < m; j++) {
          const double r = (S->h_res[3 + j] - S->a[j] * zv - yv[j] + sv[j] - S->b[j]) / dmp;
          acc(r);
        }
        for (int j = 0; j < m; j++) acc(muv[j] * yv[j] - S->eps);
        acc(zetav * zv - S->eps);
        for (int j = 0; j < m; j++) acc(lam[j] * sv[j] - S->eps);
        *e2 = std::sqrt(sum);
        *einf = mx;
        return RSO_OK;
      };
      double old_err = 0, old_inf = 0;
      RSO_TRY(kkt(0.0, S->lambda, S->y, S->z, S->mu, S->zeta, S->s, 1.0, &old_err, &old_inf));
      double step = max_t, new_err = 1e30, new_inf = 1e30;
      while (step > 1e-12 && new_err > old_err) {
        std::vector<double> nl(m), ny(m), nmu(m), ns(m);
        for (int j = 0; j < m; j++) {
          nl[j] = S->lambda[j] + dl[j] * step; ny[j] = S->y[j] + dy[j] * step;
          nmu[j] = S->mu[j] + dmu[j] * step; ns[j] = S->s[j] + ds[j] * step;
        }
        const double nz = S->z + dz * step, nzeta = S->zeta + dzeta * step;
        RSO_TRY(kkt(step, nl, ny, nz, nmu, nzeta, ns, damp, &new_err, &new_inf));
        if (new_err < old_err) {
          k_accept<<<MMA_BLOCKS, MMA_THREADS, 0, st>>>(n, step, S->x, S->xi, S->eta, S->dx, S->dxi, S->deta); rso::note_launch();
          S->lambda = nl; S->y = ny; S->mu = nmu; S->s = ns; S->z = nz; S->zeta = nzeta;
          break;
        }
        step /= 2;
      }
      step_used = step;
      err = new_inf;
      if ((err - lasterr) / err < 1e-5) stays++;
      else stays = 0;
      lasterr = err;
      if (stays > 6) { damp *= 10; stays = 0; }
      if (nsub++ > 80) { overflow = true; break; }
    }
    if (overflow) break;
    S->eps *= 0.1;
  }
  k_asym<<<MMA_BLOCKS, MMA_THREADS, 0, st>>>(n, S->x, S->curx, S->lastdx, S->L, S->U, S->alpha, S->beta, S->xmin,
                                             S->xmax, S->part); rso::note_launch();
  RSO_TRY(finish_red(S, 1, 0));
  if (std::sqrt(S->h_res[0]) < 1e-3) S->stop_counter++;
  if (info) { info[0] = err; info[1] = step_used; info[2] = nsub; info[3] = overflow; }
  if (converged) *converged = S->stop_counter > 10 ? 1 : 0;
  return RSO_OK;
}

extern "C" void rso_mma_destroy(rso_mma* s) {
  if (!s) return;
  if (s->stream) cudaStreamSynchronize(s->stream);
  double* vecs[] = {s->x, s->xmin, s->xmax, s->L, s->U, s->alpha, s->beta, s->lastdx, s->xi, s->eta, s->curx,
                    s->Dx, s->hdx, s->dx, s->dxi, s->deta, s->P, s->Q, s->G, s->part, s->res};
  for (double* v : vecs) cudaFree(v);
  if (s->h_res) cudaFreeHost(s->h_res);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

namespace rso {
double* mma_x(rso_mma* s) { return s->x; }
int mma_n(rso_mma* s) { return s->n; }
int mma_m(rso_mma* s) { return s->m; }
}  // namespace rso
