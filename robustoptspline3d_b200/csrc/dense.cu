// Dense FP64 factorisation and inverse of the coarsest-level operator.
//
// The reference solves its coarsest system on the host with Eigen's BDCSVD
// (Grid::buildCoarsestSystem / solve_fem_host, grid/Grid.cpp:3697-3752,
// :4123-4185).  Here the matrix (N = 3 x coarsest active nodes, a few
// thousand at most) is factored on the device once per operator update,
// K = L L^T, and its inverse X = L^-T L^-1 formed explicitly, so that every
// V-cycle applies the coarsest solve as one matrix-vector product.
//
// All steps work on 64 x 64 tiles of row-major N x N matrices:
//   factor:  for each diagonal tile k, Cholesky of the tile in shared memory
//            (k_potrf_tile), the tiles below it times L_kk^-T (k_trsm_panel),
//            and the trailing lower triangle minus the panel's outer product
//            (k_syrk_tiles), each a grid of independent tiles;
//   inverse: Y = L^-1 by block forward substitution on the identity (Y lower
//            triangular; k_fwd_tiles forms the right-hand side of a tile row,
//            k_trsm_rows solves it with the diagonal tile), then X = Y^T Y
//            (k_gram_tiles, lower tiles mirrored to the upper triangle).
// A singular matrix (support-free modes: the rigid motions span the null
// space) is factored as K + a R R^T with R orthonormal, and the pseudo-inverse
// follows as X - (1/a) R R^T (dense_rank_update).
#include "rso_internal.cuh"

namespace rso {

constexpr int DT = 64;        // tile edge
constexpr int DTP = DT + 1;   // padded shared-memory row (conflict-free columns)

// lower := (lower + upper) / 2, mirrored: the assembled stencils are
// symmetric up to rounding
__global__ void k_symmetrise(double* A, int N) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)N * N) return;
  const int i = (int)(idx / N), j = (int)(idx % N);
  if (j >= i) return;
  const double v = 0.5 * (A[(long long)i * N + j] + A[(long long)j * N + i]);
  A[(long long)i * N + j] = v;
  A[(long long)j * N + i] = v;
}

// Cholesky of the diagonal tile at k0 in shared memory; flag on a pivot that
// is not positive
__global__ void __launch_bounds__(256) k_potrf_tile(double* A, int N, int k0, int* flag) {
  __shared__ double S[DT][DTP];
  const int n = min(DT, N - k0), t = threadIdx.x;
  for (int idx = t; idx < n * n; idx += blockDim.x) {
    const int i = idx / n, j = idx % n;
    S[i][j] = A[(long long)(k0 + i) * N + k0 + j];
  }
  __syncthreads();
  for (int j = 0; j < n; j++) {
    if (t == 0) {
      double d = S[j][j];
      if (!(d > 0)) {
        *flag = 1;
        d = 1e-300;
      }
      S[j][j] = sqrt(d);
    }
    __syncthreads();
    const double piv = S[j][j];
    for (int i = j + 1 + t; i < n; i += blockDim.x) S[i][j] /= piv;
    __syncthreads();
    const int m = n - j - 1;
    for (int idx = t; idx < m * m; idx += blockDim.x) {
      const int i = j + 1 + idx / m, k = j + 1 + idx % m;
      if (k <= i) S[i][k] -= S[i][j] * S[k][j];
    }
    __syncthreads();
  }
  for (int idx = t; idx < n * n; idx += blockDim.x) {
    const int i = idx / n, j = idx % n;
    if (j <= i) A[(long long)(k0 + i) * N + k0 + j] = S[i][j];
  }
}

// rows below the diagonal tile at k0: A[i][k0 .. k0+n) := A[i][..] L_kk^-T,
// a CTA of 64 threads per 64 rows, one row per thread, both tiles in shared memory
__global__ void __launch_bounds__(DT) k_trsm_panel(double* A, int N, int k0) {
  extern __shared__ double dsm[];
  double(*L)[DTP] = reinterpret_cast<double(*)[DTP]>(dsm);
  double(*P)[DTP] = reinterpret_cast<double(*)[DTP]>(dsm + DT * DTP);
  const int n = min(DT, N - k0), t = threadIdx.x;
  const int r0 = k0 + n + blockIdx.x * DT, nr = min(DT, N - r0);
  for (int idx = t; idx < n * n; idx += DT) {
    const int i = idx / n, j = idx % n;
    L[i][j] = A[(long long)(k0 + i) * N + k0 + j];
  }
  for (int idx = t; idx < nr * n; idx += DT) {
    const int i = idx / n, j = idx % n;
    P[i][j] = A[(long long)(r0 + i) * N + k0 + j];
  }
  __syncthreads();
  if (t < nr) {
    for (int j = 0; j < n; j++) {
      double s = P[t][j];
      for (int m = 0; m < j; m++) s -= P[t][m] * L[j][m];
      P[t][j] = s / L[j][j];
    }
  }
  __syncthreads();
  for (int idx = t; idx < nr * n; idx += DT) {
    const int i = idx / n, j = idx % n;
    A[(long long)(r0 + i) * N + k0 + j] = P[i][j];
  }
}

// tile (ti, tj), tj <= ti, of the lower triangle below and right of the
// panel at k0: A[I][J] -= P_I P_J^T over the panel's n columns.  256 threads,
// 4 x 4 outputs each.
__device__ __forceinline__ void tile_of(int b, int* ti, int* tj) {
  int i = (int)((sqrt(8.0 * b + 1.0) - 1.0) * 0.5);
  while ((i + 1) * (i + 2) / 2 <= b) i++;
  while (i * (i + 1) / 2 > b) i--;
  *ti = i;
  *tj = b - i * (i + 1) / 2;
}
__global__ void __launch_bounds__(256) k_syrk_tiles(double* A, int N, int k0) {
  extern __shared__ double dsm[];
  double(*PI)[DT + 2] = reinterpret_cast<double(*)[DT + 2]>(dsm);            // [m][row of I]
  double(*PJ)[DT + 2] = reinterpret_cast<double(*)[DT + 2]>(dsm + DT * (DT + 2));  // [m][row of J]
  const int n = min(DT, N - k0), base = k0 + n, t = threadIdx.x;
  int ti, tj;
  tile_of(blockIdx.x, &ti, &tj);
  const int i0 = base + ti * DT, j0 = base + tj * DT;
  const int ni = min(DT, N - i0), nj = min(DT, N - j0);
  for (int idx = t; idx < DT * DT; idx += 256) {
    const int r = idx / DT, m = idx % DT;
    PI[m][r] = (r < ni && m < n) ? A[(long long)(i0 + r) * N + k0 + m] : 0.0;
    PJ[m][r] = (r < nj && m < n) ? A[(long long)(j0 + r) * N + k0 + m] : 0.0;
  }
  __syncthreads();
  const int tr = (t >> 4) * 4, tc = (t & 15) * 4;
  double acc[4][4] = {};
#pragma unroll 4
  for (int m = 0; m < DT; m++) {
    const double2 a0 = *reinterpret_cast<const double2*>(&PI[m][tr]);
    const double2 a1 = *reinterpret_cast<const double2*>(&PI[m][tr + 2]);
    const double2 b0 = *reinterpret_cast<const double2*>(&PJ[m][tc]);
    const double2 b1 = *reinterpret_cast<const double2*>(&PJ[m][tc + 2]);
    const double a[4] = {a0.x, a0.y, a1.x, a1.y}, b[4] = {b0.x, b0.y, b1.x, b1.y};
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
      for (int c = 0; c < 4; c++) acc[r][c] = fma(a[r], b[c], acc[r][c]);
  }
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int i = tr + r, j = tc + c;
      if (i < ni && j < nj && i0 + i >= j0 + j) A[(long long)(i0 + i) * N + j0 + j] -= acc[r][c];
    }
}

// Y = L^-1, tile row rb (rows r0 ..): for every tile column cb <= rb the
// right-hand side T = I_{rb,cb} - sum_{cb <= k < rb} L[rb][k] Y[k][cb],
// written into Y's tile (rb, cb)
__global__ void __launch_bounds__(256) k_fwd_tiles(const double* __restrict__ Lm, double* Y, int N, int rb) {
  extern __shared__ double dsm[];
  double(*LT)[DT + 2] = reinterpret_cast<double(*)[DT + 2]>(dsm);            // [m][row]: L[r0 + row][k0 + m]
  double(*YT)[DT + 2] = reinterpret_cast<double(*)[DT + 2]>(dsm + DT * (DT + 2));  // [m][col]: Y[k0 + m][c0 + col]
  const int cb = blockIdx.x, t = threadIdx.x;
  const int r0 = rb * DT, c0 = cb * DT, nr = min(DT, N - r0), nc = min(DT, N - c0);
  const int tr = (t >> 4) * 4, tc = (t & 15) * 4;
  double acc[4][4] = {};
  for (int kb = cb; kb < rb; kb++) {
    const int k0 = kb * DT;
    __syncthreads();
    for (int idx = t; idx < DT * DT; idx += 256) {
      const int a = idx / DT, m = idx % DT;
      LT[m][a] = a < nr ? Lm[(long long)(r0 + a) * N + k0 + m] : 0.0;
      YT[a][m] = m < nc ? Y[(long long)(k0 + a) * N + c0 + m] : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int m = 0; m < DT; m++) {
      const double2 a0 = *reinterpret_cast<const double2*>(&LT[m][tr]);
      const double2 a1 = *reinterpret_cast<const double2*>(&LT[m][tr + 2]);
      const double2 b0 = *reinterpret_cast<const double2*>(&YT[m][tc]);
      const double2 b1 = *reinterpret_cast<const double2*>(&YT[m][tc + 2]);
      const double a[4] = {a0.x, a0.y, a1.x, a1.y}, b[4] = {b0.x, b0.y, b1.x, b1.y};
#pragma unroll
      for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[r][c] = fma(a[r], b[c], acc[r][c]);
    }
  }
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int i = tr + r, j = tc + c;
      if (i < nr && j < nc) Y[(long long)(r0 + i) * N + c0 + j] = (r0 + i == c0 + j ? 1.0 : 0.0) - acc[r][c];
    }
}

// tile row rb of Y: every column c < r0 + nr solved with the diagonal tile,
// y = L_rr^-1 t, one column per thread (the tile row is at most 64 deep)
__global__ void __launch_bounds__(128) k_trsm_rows(const double* __restrict__ Lm, double* Y, int N, int rb) {
  __shared__ double L[DT][DTP];
  const int r0 = rb * DT, nr = min(DT, N - r0), t = threadIdx.x;
  for (int idx = t; idx < nr * nr; idx += blockDim.x) {
    const int i = idx / nr, j = idx % nr;
    L[i][j] = Lm[(long long)(r0 + i) * N + r0 + j];
  }
  __syncthreads();
  const int c = blockIdx.x * blockDim.x + t;
  if (c >= r0 + nr) return;
  double y[DT];
#pragma unroll
  for (int i = 0; i < DT; i++) {
    if (i < nr) {
      double s = Y[(long long)(r0 + i) * N + c];
#pragma unroll
      for (int m = 0; m < i; m++) s -= L[i][m] * y[m];
      y[i] = s / L[i][i];
      Y[(long long)(r0 + i) * N + c] = y[i];
    }
  }
}

// X = Y^T Y on the lower tiles (ti >= tj), mirrored: X[I][J] = sum over tile
// rows k >= ti of Y[k][I]^T Y[k][J] (Y is lower triangular)
__global__ void __launch_bounds__(256) k_gram_tiles(const double* __restrict__ Y, double* X, int N, int nt) {
  extern __shared__ double dsm[];
  double(*YI)[DT + 2] = reinterpret_cast<double(*)[DT + 2]>(dsm);
  double(*YJ)[DT + 2] = reinterpret_cast<double(*)[DT + 2]>(dsm + DT * (DT + 2));
  int ti, tj;
  tile_of(blockIdx.x, &ti, &tj);
  const int i0 = ti * DT, j0 = tj * DT, ni = min(DT, N - i0), nj = min(DT, N - j0), t = threadIdx.x;
  const int tr = (t >> 4) * 4, tc = (t & 15) * 4;
  double acc[4][4] = {};
  for (int kb = ti; kb < nt; kb++) {
    const int k0 = kb * DT, nk = min(DT, N - k0);
    __syncthreads();
    for (int idx = t; idx < DT * DT; idx += 256) {
      const int m = idx / DT, a = idx % DT;
      YI[m][a] = (m < nk && a < ni) ? Y[(long long)(k0 + m) * N + i0 + a] : 0.0;
      YJ[m][a] = (m < nk && a < nj) ? Y[(long long)(k0 + m) * N + j0 + a] : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int m = 0; m < DT; m++) {
      const double2 a0 = *reinterpret_cast<const double2*>(&YI[m][tr]);
      const double2 a1 = *reinterpret_cast<const double2*>(&YI[m][tr + 2]);
      const double2 b0 = *reinterpret_cast<const double2*>(&YJ[m][tc]);
      const double2 b1 = *reinterpret_cast<const double2*>(&YJ[m][tc + 2]);
      const double a[4] = {a0.x, a0.y, a1.x, a1.y}, b[4] = {b0.x, b0.y, b1.x, b1.y};
#pragma unroll
      for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[r][c] = fma(a[r], b[c], acc[r][c]);
    }
  }
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int i = tr + r, j = tc + c;
      if (i < ni && j < nj) {
        X[(long long)(i0 + i) * N + j0 + j] = acc[r][c];
        X[(long long)(j0 + j) * N + i0 + i] = acc[r][c];
      }
    }
}

// A += a R R^T (add) or A -= (1/a) R R^T, R: N x nr row-major (nr <= 6)
__global__ void k_rank_update(double* A, int N, const double* __restrict__ R, int nr, double a) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)N * N) return;
  const int i = (int)(idx / N), j = (int)(idx % N);
  double s = 0;
  for (int k = 0; k < nr; k++) s += R[(long long)i * nr + k] * R[(long long)j * nr + k];
  A[idx] += a * s;
}

static int ntiles(int N) { return (N + DT - 1) / DT; }

// K (N x N in A, overwritten by its Cholesky factor in the lower triangle),
// X = K^-1, Y scratch (N x N); flag set on a pivot that is not positive
rso_status dense_spd_inverse(rso_handle* h, double* A, double* X, double* Y, int N, int* flag) {
  // shared-memory opt-in, per device (a host call per kernel and operator update)
  const int sm2 = 2 * DT * (DT + 2) * (int)sizeof(double);  // 67,584 bytes
  const int smp = 2 * DT * DTP * (int)sizeof(double);       // 66,560 bytes
  RSO_CHECK_CUDA(h, cudaFuncSetAttribute(k_syrk_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, sm2));
  RSO_CHECK_CUDA(h, cudaFuncSetAttribute(k_fwd_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, sm2));
  RSO_CHECK_CUDA(h, cudaFuncSetAttribute(k_gram_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, sm2));
  RSO_CHECK_CUDA(h, cudaFuncSetAttribute(k_trsm_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, smp));
  const int nt = ntiles(N);
  const long long NN = (long long)N * N;
  k_symmetrise<<<(unsigned)cdiv(NN, 256), 256, 0, h->stream>>>(A, N); rso::note_launch();
  for (int kb = 0; kb < nt; kb++) {
    const int k0 = kb * DT;
    k_potrf_tile<<<1, 256, 0, h->stream>>>(A, N, k0, flag); rso::note_launch();
    const int rest = N - k0 - min(DT, N - k0);
    if (rest > 0) {
      const int rt = ntiles(rest);
      k_trsm_panel<<<rt, DT, smp, h->stream>>>(A, N, k0); rso::note_launch();
      k_syrk_tiles<<<rt * (rt + 1) / 2, 256, sm2, h->stream>>>(A, N, k0); rso::note_launch();
    }
  }
  for (int rb = 0; rb < nt; rb++) {
    k_fwd_tiles<<<rb + 1, 256, sm2, h->stream>>>(A, Y, N, rb); rso::note_launch();
    const int cols = min(N, (rb + 1) * DT);
    k_trsm_rows<<<cdiv(cols, 128), 128, 0, h->stream>>>(A, Y, N, rb); rso::note_launch();
  }
  k_gram_tiles<<<nt * (nt + 1) / 2, 256, sm2, h->stream>>>(Y, X, N, nt); rso::note_launch();
  return launch_check(h, "coarsest dense inverse");
}

__global__ void k_trace(const double* __restrict__ A, int N, double* out) {
  __shared__ double ws[32];
  double s = 0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) s += A[(long long)i * N + i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += ws[w];
    *out = t;
  }
}

rso_status dense_trace(rso_handle* h, const double* A, int N, double* out) {
  k_trace<<<1, 1024, 0, h->stream>>>(A, N, out); rso::note_launch();
  return launch_check(h, "coarsest trace");
}

rso_status dense_rank_update(rso_handle* h, double* A, int N, const double* R, int nr, double a) {
  k_rank_update<<<(unsigned)cdiv((long long)N * N, 256), 256, 0, h->stream>>>(A, N, R, nr, a); rso::note_launch();
  return launch_check(h, "coarsest rank update");
}

}  // namespace rso
