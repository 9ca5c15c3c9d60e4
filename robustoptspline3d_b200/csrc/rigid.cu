// Rigid motions of support-free problems (RSO_NO_SUPPORT_* modes).
//
// Without supports the stiffness operator is singular: its null space is the
// six rigid motions (three translations and three rotations p^) of the
// active nodes.  The reference handles this in three places, all mirrored
// here:
//  - forceProject removes the rigid motions of the load set from every
//    admissible load, after the tangential part in constrained-direction
//    modes (optimization/projection.cpp:289-360; the basis Rd, orthonormal by
//    Gram-Schmidt with nearly dependent motions dropped, :129-269);
//  - displacementProject removes the rigid motions of all active fine nodes
//    from the displacement (projection.cpp:374-411, basis _R of :47-110);
//  - the coarsest solve is a pseudo-inverse (BDCSVD, grid/Grid.cpp:4123-4185),
//    here (K + a R R^T)^-1 - R R^T / a with R the coarsest nodes' rigid
//    motions (coarse_op.cu, coarsest_factor).
// The load-set and coarsest bases are explicit (a few million doubles at
// most); the fine-node projection is formed from the node coordinates on the
// fly: u -= R G^-1 R^T u, G the 6 x 6 Gram matrix of the motions about the
// nodes' centroid (the projector onto the span the reference's orthonormal
// basis has).
#include "rso_internal.cuh"
#include <cmath>
#include <vector>

namespace rso {

constexpr int RG_BLOCKS = 296, RG_THREADS = 256;

// modified Gram-Schmidt over the 6 motions of `pos` (3 per node), in column
// order, optionally normal-projected per node and dropping columns whose
// residual is below 1e-6 of their norm (projection.cpp:235-262); returns the
// number of kept columns, stored column-major (3 n entries each) in Q
static int rigid_mgs(const std::vector<double>& pos, const double* nrm, bool drop, std::vector<double>& Q) {
  const size_t m = pos.size();
  std::vector<std::vector<double>> col(6, std::vector<double>(m, 0.0));
  for (size_t k = 0; k < m / 3; k++) {
    const double x = pos[3 * k], y = pos[3 * k + 1], z = pos[3 * k + 2];
    const double ph[3][3] = {{0, -z, y}, {z, 0, -x}, {-y, x, 0}};
    for (int c = 0; c < 3; c++) {
      col[c][3 * k + c] = 1.0;
      for (int j = 0; j < 3; j++) col[3 + j][3 * k + c] = ph[c][j];
    }
    if (nrm) {
      const double* nv = nrm + 3 * k;
      for (int j = 0; j < 6; j++) {
        double* b = &col[j][3 * k];
        const double s = b[0] * nv[0] + b[1] * nv[1] + b[2] * nv[2];
        for (int c = 0; c < 3; c++) b[c] = s * nv[c];
      }
    }
  }
  auto dotv = [&](const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0;
    for (size_t i = 0; i < m; i++) s += a[i] * b[i];
    return s;
  };
  bool invalid[6] = {false, false, false, false, false, false};
  for (int i = 0; i < 6; i++) {
    const double oldres = std::sqrt(dotv(col[i], col[i]));
    for (int j = 0; j < i; j++) {
      if (invalid[j]) continue;
      const double w = dotv(col[i], col[j]);
      for (size_t t = 0; t < m; t++) col[i][t] -= w * col[j][t];
    }
    const double res = std::sqrt(dotv(col[i], col[i]));
    if (drop && (!(oldres >= 1e-6) || res / oldres < 1e-6)) invalid[i] = true;
    if (!invalid[i])
      for (size_t t = 0; t < m; t++) col[i][t] /= res;
  }
  Q.clear();
  int k = 0;
  for (int i = 0; i < 6; i++) {
    if (invalid[i]) continue;
    Q.insert(Q.end(), col[i].begin(), col[i].end());
    k++;
  }
  return k;
}

// inverse of a 6 x 6 matrix (Gauss-Jordan with partial pivoting on the host)
static bool inv6(const double* G, double* M) {
  double A[6][12];
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 12; j++) A[i][j] = j < 6 ? G[i * 6 + j] : (j - 6 == i ? 1.0 : 0.0);
  for (int c = 0; c < 6; c++) {
    int p = c;
    for (int r = c + 1; r < 6; r++)
      if (std::fabs(A[r][c]) > std::fabs(A[p][c])) p = r;
    if (!(std::fabs(A[p][c]) > 0)) return false;
    for (int j = 0; j < 12; j++) std::swap(A[c][j], A[p][j]);
    const double d = A[c][c];
    for (int j = 0; j < 12; j++) A[c][j] /= d;
    for (int r = 0; r < 6; r++) {
      if (r == c) continue;
      const double f = A[r][c];
      for (int j = 0; j < 12; j++) A[r][j] -= f * A[c][j];
    }
  }
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) M[i * 6 + j] = A[i][j + 6];
  return true;
}

rso_status rigid_setup(rso_handle* h) {
  const Level& l0 = h->L[0];
  const int nl = h->n_load;
  const size_t ls = 3 * (size_t)std::max(nl, 1);
  // load set: positions and normals of the load nodes, in load order
  std::vector<double> pos(3 * (size_t)nl), nrm(ls);
  for (int k = 0; k < nl; k++) {
    const long long n = h->h_load_nodes[k];
    pos[3 * k] = (double)(n % l0.nx);
    pos[3 * k + 1] = (double)(n / l0.nx % l0.ny);
    pos[3 * k + 2] = (double)(n / ((long long)l0.nx * l0.ny));
  }
  RSO_CHECK_CUDA(h, cudaMemcpy(nrm.data(), h->load_normals, sizeof(double) * nrm.size(), cudaMemcpyDeviceToHost));
  RSO_CHECK_CUDA(h, cudaMalloc(&h->rigid_q, sizeof(double) * 2 * 6 * ls));
  RSO_CHECK_CUDA(h, cudaMemset(h->rigid_q, 0, sizeof(double) * 2 * 6 * ls));
  for (int cf = 0; cf < 2; cf++) {
    std::vector<double> Q;
    h->rigid_k[cf] = nl ? rigid_mgs(pos, cf ? nrm.data() : nullptr, true, Q) : 0;
    if (h->rigid_k[cf])
      RSO_CHECK_CUDA(h, cudaMemcpy(h->rigid_q + (size_t)cf * 6 * ls, Q.data(), sizeof(double) * Q.size(),
                                   cudaMemcpyHostToDevice));
  }
  // fine nodes: centroid and inverse Gram matrix of the motions about it
  const std::vector<uint8_t>& vm = h->h_vmask[0];
  double cnt = 0, cs[3] = {0, 0, 0};
  for (int z = 0; z < l0.nz; z++)
    for (int y = 0; y < l0.ny; y++)
      for (int x = 0; x < l0.nx; x++)
        if (vm[x + (size_t)l0.nx * (y + (size_t)l0.ny * z)]) { cnt++; cs[0] += x; cs[1] += y; cs[2] += z; }
  if (cnt < 1) { h->err = "no active node"; return RSO_ERR_INVALID_ARG; }
  const double ctr[3] = {cs[0] / cnt, cs[1] / cnt, cs[2] / cnt};
  double G[36] = {};
  for (int z = 0; z < l0.nz; z++)
    for (int y = 0; y < l0.ny; y++)
      for (int x = 0; x < l0.nx; x++) {
        if (!vm[x + (size_t)l0.nx * (y + (size_t)l0.ny * z)]) continue;
        const double X = x - ctr[0], Y = y - ctr[1], Z = z - ctr[2];
        // rows c of [I | p^] at this node
        const double R[3][6] = {{1, 0, 0, 0, -Z, Y}, {0, 1, 0, Z, 0, -X}, {0, 0, 1, -Y, X, 0}};
        for (int i = 0; i < 6; i++)
          for (int j = 0; j < 6; j++) G[i * 6 + j] += R[0][i] * R[0][j] + R[1][i] * R[1][j] + R[2][i] * R[2][j];
      }
  double M[39];
  if (!inv6(G, M)) { h->err = "rigid motions of the active nodes are degenerate"; return RSO_ERR_INVALID_ARG; }
  M[36] = ctr[0]; M[37] = ctr[1]; M[38] = ctr[2];
  RSO_CHECK_CUDA(h, cudaMalloc(&h->rigid_m, sizeof(M)));
  RSO_CHECK_CUDA(h, cudaMemcpy(h->rigid_m, M, sizeof(M), cudaMemcpyHostToDevice));
  RSO_CHECK_CUDA(h, cudaMalloc(&h->rigid_scr, sizeof(double) * 6 * RG_BLOCKS));
  // coarsest nodes: orthonormal motions (coarse node coordinates: positions
  // scaled by a common factor span the same motions)
  if (h->L.size() > 1 && h->nc > 0) {
    const Level& c = h->L.back();
    const std::vector<uint8_t>& cvm = h->h_vmask.back();
    std::vector<double> cpos;
    for (int z = 0; z < c.nz; z++)
      for (int y = 0; y < c.ny; y++)
        for (int x = 0; x < c.nx; x++)
          if (cvm[x + (size_t)c.nx * (y + (size_t)c.ny * z)]) {
            cpos.push_back(x);
            cpos.push_back(y);
            cpos.push_back(z);
          }
    std::vector<double> Q;
    const int k = rigid_mgs(cpos, nullptr, false, Q);
    const size_t N = cpos.size();
    std::vector<double> Rrow(N * 6, 0.0);  // row-major N x 6, the order of the coarsest node list
    for (int j = 0; j < k; j++)
      for (size_t i = 0; i < N; i++) Rrow[i * 6 + j] = Q[j * N + i];
    RSO_CHECK_CUDA(h, cudaMalloc(&h->c_R, sizeof(double) * Rrow.size()));
    RSO_CHECK_CUDA(h, cudaMemcpy(h->c_R, Rrow.data(), sizeof(double) * Rrow.size(), cudaMemcpyHostToDevice));
  }
  return RSO_OK;
}

// ---------------------------------------------------------------- load set
// s = Q^T v (fixed-order partial sums), then v -= Q s
__global__ void __launch_bounds__(RG_THREADS) k_ls_dots(const double* __restrict__ Q, long long ls,
                                                       const double* __restrict__ v, double* __restrict__ part) {
  const int j = blockIdx.y;
  double s = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ls; i += (long long)gridDim.x * blockDim.x)
    s += Q[ls * j + i] * v[i];
  __shared__ double ws[RG_THREADS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < RG_THREADS / 32; w++) t += ws[w];
    part[j * RG_BLOCKS + blockIdx.x] = t;
  }
}
__global__ void k_ls_sub(const double* __restrict__ Q, long long ls, int k, const double* __restrict__ part,
                         double* __restrict__ v) {
  __shared__ double s[6];
  if (threadIdx.x < k) {
    double t = 0;
    for (int b = 0; b < RG_BLOCKS; b++) t += part[threadIdx.x * RG_BLOCKS + b];
    s[threadIdx.x] = t;
  }
  __syncthreads();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ls; i += (long long)gridDim.x * blockDim.x) {
    double a = v[i];
    for (int j = 0; j < k; j++) a -= s[j] * Q[ls * j + i];
    v[i] = a;
  }
}

rso_status rigid_project_load(rso_handle* h, double* v, int cf) {
  if (h->has_support || h->n_load == 0) return RSO_OK;
  const int ci = cf ? 1 : 0, k = h->rigid_k[ci];
  if (k == 0) return RSO_OK;
  const long long ls = 3LL * h->n_load;
  const double* Q = h->rigid_q + (size_t)ci * 6 * ls;
  k_ls_dots<<<dim3(RG_BLOCKS, k), RG_THREADS, 0, h->stream>>>(Q, ls, v, h->rigid_scr); note_launch();
  k_ls_sub<<<RG_BLOCKS, RG_THREADS, 0, h->stream>>>(Q, ls, k, h->rigid_scr, v); note_launch();
  return launch_check(h, "rigid_project_load");
}

// ---------------------------------------------------------------- fine nodes
// R^T u at the active nodes, motions about the centroid m[36..38]
__global__ void __launch_bounds__(RG_THREADS) k_rigid_dots(const Level L, const double* __restrict__ u,
                                                          const double* __restrict__ m, double* __restrict__ part) {
  double s[6] = {0, 0, 0, 0, 0, 0};
  const long long pxy = (long long)L.px * L.py;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < L.NP;
       p += (long long)gridDim.x * blockDim.x) {
    if (!(L.vclass[p] & NC_ACTIVE)) continue;
    const long long zp = p / pxy, r = p - zp * pxy, yp = r / L.px, xp = r - yp * L.px;
    const double X = (double)(xp - 1) - m[36], Y = (double)(yp - 1) - m[37], Z = (double)(zp - 1) - m[38];
    const double a = u[p], b = u[p + L.NP], c = u[p + 2 * L.NP];
    s[0] += a; s[1] += b; s[2] += c;
    s[3] += Z * b - Y * c; s[4] += -Z * a + X * c; s[5] += Y * a - X * b;
  }
  __shared__ double ws[6][RG_THREADS / 32];
#pragma unroll
  for (int j = 0; j < 6; j++) {
    double t = s[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) ws[j][threadIdx.x >> 5] = t;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double t = 0;
    for (int w = 0; w < RG_THREADS / 32; w++) t += ws[threadIdx.x][w];
    part[threadIdx.x * RG_BLOCKS + blockIdx.x] = t;
  }
}
// u -= R (G^-1 R^T u) at the active nodes
__global__ void k_rigid_sub(const Level L, double* __restrict__ u, const double* __restrict__ m,
                            const double* __restrict__ part) {
  __shared__ double s[6], cf[6];
  if (threadIdx.x < 6) {
    double t = 0;
    for (int b = 0; b < RG_BLOCKS; b++) t += part[threadIdx.x * RG_BLOCKS + b];
    s[threadIdx.x] = t;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double t = 0;
    for (int j = 0; j < 6; j++) t += m[threadIdx.x * 6 + j] * s[j];
    cf[threadIdx.x] = t;
  }
  __syncthreads();
  const long long pxy = (long long)L.px * L.py;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < L.NP;
       p += (long long)gridDim.x * blockDim.x) {
    if (!(L.vclass[p] & NC_ACTIVE)) continue;
    const long long zp = p / pxy, r = p - zp * pxy, yp = r / L.px, xp = r - yp * L.px;
    const double X = (double)(xp - 1) - m[36], Y = (double)(yp - 1) - m[37], Z = (double)(zp - 1) - m[38];
    u[p] -= cf[0] - Z * cf[4] + Y * cf[5];
    u[p + L.NP] -= cf[1] + Z * cf[3] - X * cf[5];
    u[p + 2 * L.NP] -= cf[2] - Y * cf[3] + X * cf[4];
  }
}

rso_status displacement_project(rso_handle* h, double* u) {
  if (h->has_support) return RSO_OK;
  const Level& l0 = h->L[0];
  k_rigid_dots<<<RG_BLOCKS, RG_THREADS, 0, h->stream>>>(l0, u, h->rigid_m, h->rigid_scr); note_launch();
  k_rigid_sub<<<RG_BLOCKS, RG_THREADS, 0, h->stream>>>(l0, u, h->rigid_m, h->rigid_scr); note_launch();
  return launch_check(h, "displacement_project");
}

}  // namespace rso

using namespace rso;

extern "C" rso_status rso_displacement_project(rso_handle* h, double* u) {
  if (!h || !u) return RSO_ERR_INVALID_ARG;
  RSO_TRY(pad_nodes(h, 0, u, h->w));
  RSO_TRY(displacement_project(h, h->w));
  RSO_TRY(unpad_nodes(h, 0, h->w, u));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}
