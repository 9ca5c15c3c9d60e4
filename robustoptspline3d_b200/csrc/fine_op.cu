// Matrix-free SIMP elasticity operator on the finest level.
//
// r_i = f_i - sum_{e incident to i} rho_e^p sum_{j in e} K0[vi, vj] u_j
// (update_residual_OTFA_WS_kernel grid/Grid.cu:2320-2376, applyK_OTFA_kernel
// grid/Grid.cu:4358-4436, gs_relax_OTFA_WS_kernel grid/Grid.cu:1742-1885).
//
// One thread per node.  The 27 neighbour displacements are loaded once; each
// is multiplied by the K0 blocks of the (up to 8) incident elements that
// contain both nodes, accumulated per element, and the 8 partial sums are
// scaled by rho_e^p at the end: 576 FMA + 24 FMA per node.  K0 lives in
// constant memory and, with every loop unrolled, each K0 entry is a
// compile-time constant-bank operand of the FMA.  Support DOFs hold zero by
// construction, so neighbours need no Dirichlet test; support rows are
// handled from the node-class byte.
#include "rso_internal.cuh"
#include <cmath>

namespace rso {

__constant__ double cK0d[576];
__constant__ float cK0f[576];

template <typename T>
__device__ __forceinline__ T k0(int i);
template <>
__device__ __forceinline__ double k0<double>(int i) { return cK0d[i]; }
template <>
__device__ __forceinline__ float k0<float>(int i) { return cK0f[i]; }

rso_status upload_K0(rso_handle* h) {
  float kf[576];
  for (int i = 0; i < 576; i++) kf[i] = (float)h->K0[i];
  RSO_CHECK_CUDA(h, cudaMemcpyToSymbolAsync(cK0d, h->K0, sizeof(double) * 576, 0, cudaMemcpyHostToDevice, h->stream));
  RSO_CHECK_CUDA(h, cudaMemcpyToSymbolAsync(cK0f, kf, sizeof(float) * 576, 0, cudaMemcpyHostToDevice, h->stream));
  return RSO_OK;
}

// rho^p in FP64 (and its FP32 copy) for active elements, zero elsewhere
__global__ void k_penalise(Level L, const float* rho, float* rp32, double* rp64, double p) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= L.NQ) return;
  double v = 0.0;
  if (L.emask[i]) v = pow((double)rho[i], p);
  rp64[i] = v;
  rp32[i] = (float)v;
}

rso_status penalise(rso_handle* h) {
  Level& l = h->L[0];
  k_penalise<<<cdiv(l.NQ, 256), 256, 0, h->stream>>>(l, h->rho, h->rp32, h->rp64, h->cfg.penal); rso::note_launch();
  return launch_check(h, "penalise");
}

// MODE 0: out = f - K u;  MODE 1: out = K u (support rows pass u);
// MODE 2: out = u + omega D^-1 (f - K u)  (damped block Jacobi, D = 3x3 diagonal block)
template <typename T, int MODE>
__global__ void __launch_bounds__(256) k_fine(const Level L, const T* __restrict__ u, const T* __restrict__ f,
                                              T* __restrict__ out, const T* __restrict__ rp, T omega) {
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * 8 + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= L.nx || y >= L.ny) return;
  const long long NP = L.NP;
  const long long px = L.px, pxy = (long long)L.px * L.py;
  const long long n = L.nidx(x, y, z);
  const uint8_t cls = L.vclass[n];
  const bool work = (cls & NC_ACTIVE) && !(cls & NC_SUPPORT);
  T acc0 = 0, acc1 = 0, acc2 = 0;
  T D[6] = {0, 0, 0, 0, 0, 0};
  if (work) {
    const long long qx = L.qx, qxy = (long long)L.qx * L.qy;
    const long long e0 = L.eidx(x - 1, y - 1, z - 1);
    T r[8];
#pragma unroll
    for (int k = 0; k < 8; k++) r[k] = rp[e0 + (k & 1) + ((k >> 1) & 1) * qx + (k >> 2) * qxy];
    T a[8][3];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k][0] = a[k][1] = a[k][2] = 0;
#pragma unroll
    for (int d = 0; d < 27; d++) {
      const int dx = d % 3 - 1, dy = d / 3 % 3 - 1, dz = d / 9 - 1;
      const long long nb = n + dx + dy * px + dz * pxy;
      const T u0 = u[nb], u1 = u[nb + NP], u2 = u[nb + 2 * NP];
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const int kx = k & 1, ky = (k >> 1) & 1, kz = k >> 2;
        // element k spans node offsets {k?-1, k?} on each axis
        if ((dx == kx - 1 || dx == kx) && (dy == ky - 1 || dy == ky) && (dz == kz - 1 || dz == kz)) {
          const int vi = 7 - k;
          const int vj = (dx - kx + 1) + 2 * (dy - ky + 1) + 4 * (dz - kz + 1);
#pragma unroll
          for (int rr = 0; rr < 3; rr++)
            a[k][rr] += k0<T>((vi * 3 + rr) * 24 + vj * 3 + 0) * u0 + k0<T>((vi * 3 + rr) * 24 + vj * 3 + 1) * u1 +
                        k0<T>((vi * 3 + rr) * 24 + vj * 3 + 2) * u2;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < 8; k++) {
      acc0 += r[k] * a[k][0];
      acc1 += r[k] * a[k][1];
      acc2 += r[k] * a[k][2];
    }
    if (MODE == 2) {
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const int vi = 7 - k;
        D[0] += r[k] * k0<T>((vi * 3 + 0) * 24 + vi * 3 + 0);
        D[1] += r[k] * k0<T>((vi * 3 + 0) * 24 + vi * 3 + 1);
        D[2] += r[k] * k0<T>((vi * 3 + 0) * 24 + vi * 3 + 2);
        D[3] += r[k] * k0<T>((vi * 3 + 1) * 24 + vi * 3 + 1);
        D[4] += r[k] * k0<T>((vi * 3 + 1) * 24 + vi * 3 + 2);
        D[5] += r[k] * k0<T>((vi * 3 + 2) * 24 + vi * 3 + 2);
      }
    }
  }
  if (MODE == 0) {
    out[n] = f[n] - acc0;
    out[n + NP] = f[n + NP] - acc1;
    out[n + 2 * NP] = f[n + 2 * NP] - acc2;
  } else if (MODE == 1) {
    const bool pass = (cls & NC_SUPPORT) != 0;
    out[n] = pass ? u[n] : acc0;
    out[n + NP] = pass ? u[n + NP] : acc1;
    out[n + 2 * NP] = pass ? u[n + 2 * NP] : acc2;
  } else {
    if (!work) {
      out[n] = 0; out[n + NP] = 0; out[n + 2 * NP] = 0;
      return;
    }
    const T r0 = f[n] - acc0, r1 = f[n + NP] - acc1, r2 = f[n + 2 * NP] - acc2;
    // symmetric 3x3 inverse
    const T a = D[0], b = D[1], c = D[2], d = D[3], e = D[4], g = D[5];
    const T A = d * g - e * e, B = c * e - b * g, C = b * e - c * d;
    const T det = a * A + b * B + c * C;
    const T id = omega / det;
    const T E = a * g - c * c, F = b * c - a * e, I = a * d - b * b;
    out[n] = u[n] + id * (A * r0 + B * r1 + C * r2);
    out[n + NP] = u[n + NP] + id * (B * r0 + E * r1 + F * r2);
    out[n + 2 * NP] = u[n + 2 * NP] + id * (C * r0 + F * r1 + I * r2);
  }
}

// one colour of the 8-colour point Gauss-Seidel sweep (in place)
template <typename T>
__global__ void __launch_bounds__(256) k_fine_gs(const Level L, T* __restrict__ u, const T* __restrict__ f,
                                                 const T* __restrict__ rp, int cx, int cy, int cz, int rev) {
  const int x = 2 * (blockIdx.x * 32 + threadIdx.x) + cx;
  const int y = 2 * (blockIdx.y * 8 + threadIdx.y) + cy;
  const int z = 2 * blockIdx.z + cz;
  if (x >= L.nx || y >= L.ny || z >= L.nz) return;
  const long long NP = L.NP;
  const long long px = L.px, pxy = (long long)L.px * L.py;
  const long long n = L.nidx(x, y, z);
  const uint8_t cls = L.vclass[n];
  if (!(cls & NC_ACTIVE)) return;
  if (cls & NC_SUPPORT) {
    // S = n_e I and KeU = 0 at support nodes (grid/Grid.cu:1808-1833): u = f / n_e = 0
    u[n] = 0; u[n + NP] = 0; u[n + 2 * NP] = 0;
    return;
  }
  const long long qx = L.qx, qxy = (long long)L.qx * L.qy;
  const long long e0 = L.eidx(x - 1, y - 1, z - 1);
  T r[8];
#pragma unroll
  for (int k = 0; k < 8; k++) r[k] = rp[e0 + (k & 1) + ((k >> 1) & 1) * qx + (k >> 2) * qxy];
  T a[8][3];
#pragma unroll
  for (int k = 0; k < 8; k++) a[k][0] = a[k][1] = a[k][2] = 0;
#pragma unroll
  for (int d = 0; d < 27; d++) {
    if (d == 13) continue;
    const int dx = d % 3 - 1, dy = d / 3 % 3 - 1, dz = d / 9 - 1;
    const long long nb = n + dx + dy * px + dz * pxy;
    const T u0 = u[nb], u1 = u[nb + NP], u2 = u[nb + 2 * NP];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const int kx = k & 1, ky = (k >> 1) & 1, kz = k >> 2;
      if ((dx == kx - 1 || dx == kx) && (dy == ky - 1 || dy == ky) && (dz == kz - 1 || dz == kz)) {
        const int vi = 7 - k;
        const int vj = (dx - kx + 1) + 2 * (dy - ky + 1) + 4 * (dz - kz + 1);
#pragma unroll
        for (int rr = 0; rr < 3; rr++)
          a[k][rr] += k0<T>((vi * 3 + rr) * 24 + vj * 3 + 0) * u0 + k0<T>((vi * 3 + rr) * 24 + vj * 3 + 1) * u1 +
                      k0<T>((vi * 3 + rr) * 24 + vj * 3 + 2) * u2;
      }
    }
  }
  T KU[3] = {0, 0, 0};
  T S[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const int vi = 7 - k;
#pragma unroll
    for (int rr = 0; rr < 3; rr++) {
      KU[rr] += r[k] * a[k][rr];
#pragma unroll
      for (int c = 0; c < 3; c++) S[rr * 3 + c] += r[k] * k0<T>((vi * 3 + rr) * 24 + vi * 3 + c);
    }
  }
  T v[3] = {u[n], u[n + NP], u[n + 2 * NP]};
#pragma unroll
  for (int t = 0; t < 3; t++) {
    const int rr = rev ? 2 - t : t;
    T s = f[n + rr * NP] - KU[rr];
#pragma unroll
    for (int c = 0; c < 3; c++)
      if (c != rr) s -= S[rr * 3 + c] * v[c];
    v[rr] = s / S[rr * 3 + rr];
  }
  u[n] = v[0]; u[n + NP] = v[1]; u[n + 2 * NP] = v[2];
}

static inline dim3 fine_grid(const Level& l) { return dim3(cdiv(l.nx, 32), cdiv(l.ny, 8), l.nz); }

template <typename T>
static inline int pcls(int c32, int c64) { return sizeof(T) == 4 ? c32 : c64; }

template <typename T>
rso_status fine_residual(rso_handle* h, const T* u, const T* f, T* r, const T* rp) {
  const Level& l = h->L[0];
  const int cls = pcls<T>(PC_FINE_RES32, PC_FINE_RES64);
  if (h->prof_on) prof_begin(h, cls, (double)l.nn);
  k_fine<T, 0><<<fine_grid(l), dim3(32, 8), 0, h->stream>>>(l, u, f, r, rp, T(0));
  note_launch();
  if (h->prof_on) prof_end(h, cls);
  return launch_check(h, "fine_residual");
}
template <typename T>
rso_status fine_applyK(rso_handle* h, const T* u, T* f, const T* rp) {
  const Level& l = h->L[0];
  const int cls = pcls<T>(PC_FINE_RES32, PC_FINE_APPLYK64);
  if (h->prof_on) prof_begin(h, cls, (double)l.nn);
  k_fine<T, 1><<<fine_grid(l), dim3(32, 8), 0, h->stream>>>(l, u, u, f, rp, T(0));
  note_launch();
  if (h->prof_on) prof_end(h, cls);
  return launch_check(h, "fine_applyK");
}
template <typename T>
rso_status fine_jacobi(rso_handle* h, const T* u_in, const T* f, T* u_out, const T* rp, double omega) {
  const Level& l = h->L[0];
  const int cls = pcls<T>(PC_FINE_JAC32, PC_FINE_JAC64);
  if (h->prof_on) prof_begin(h, cls, (double)l.nn);
  k_fine<T, 2><<<fine_grid(l), dim3(32, 8), 0, h->stream>>>(l, u_in, f, u_out, rp, (T)omega);
  note_launch();
  if (h->prof_on) prof_end(h, cls);
  return launch_check(h, "fine_jacobi");
}
template <typename T>
rso_status fine_gs(rso_handle* h, T* u, const T* f, const T* rp, int colour, int reverse) {
  const Level& l = h->L[0];
  int cx = colour & 1, cy = (colour >> 1) & 1, cz = colour >> 2;
  dim3 g(cdiv((l.nx - cx + 1) / 2, 32), cdiv((l.ny - cy + 1) / 2, 8), (l.nz - cz + 1) / 2);
  if (g.x == 0 || g.y == 0 || g.z == 0) return RSO_OK;
  const int cls = pcls<T>(PC_FINE_GS32, PC_FINE_GS64);
  if (h->prof_on) prof_begin(h, cls, (double)l.nn / 8);
  k_fine_gs<T><<<g, dim3(32, 8), 0, h->stream>>>(l, u, f, rp, cx, cy, cz, reverse);
  note_launch();
  if (h->prof_on) prof_end(h, cls);
  return launch_check(h, "fine_gs");
}

template rso_status fine_residual<double>(rso_handle*, const double*, const double*, double*, const double*);
template rso_status fine_residual<float>(rso_handle*, const float*, const float*, float*, const float*);
template rso_status fine_applyK<double>(rso_handle*, const double*, double*, const double*);
template rso_status fine_applyK<float>(rso_handle*, const float*, float*, const float*);
template rso_status fine_jacobi<double>(rso_handle*, const double*, const double*, double*, const double*, double);
template rso_status fine_jacobi<float>(rso_handle*, const float*, const float*, float*, const float*, double);
template rso_status fine_gs<double>(rso_handle*, double*, const double*, const double*, int, int);
template rso_status fine_gs<float>(rso_handle*, float*, const float*, const float*, int, int);

}  // namespace rso
