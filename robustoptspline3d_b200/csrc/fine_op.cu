// Matrix-free SIMP elasticity operator on the finest level.
//
// r_i = f_i - sum_{e incident to i} rho_e^p sum_{j in e} K0[vi, vj] u_j
// (update_residual_OTFA_WS_kernel grid/Grid.cu:2320-2376, applyK_OTFA_kernel
// grid/Grid.cu:4358-4436, gs_relax_OTFA_WS_kernel grid/Grid.cu:1742-1885).
//
// Residual / apply / damped-Jacobi kernels march along z.  A CTA owns a
// TX x TY column of nodes and a chunk of z planes; it keeps a rolling window
// of four node planes of u (three in use, one being filled) and three element
// planes of rho^p in shared memory, filled with cp.async while the previous
// plane is computed, so every value is read from HBM about once per CTA
// (halo overhead (TX+2)(TY+2)/(TX*TY)).  Each thread computes one node per
// plane: the 27 neighbour displacements are multiplied by the K0 blocks of
// the incident elements that contain both nodes, accumulated per element and
// scaled by rho_e^p at the end (576 + 24 FMA per node).  K0 lives in constant
// memory; with every loop unrolled each entry is a compile-time constant-bank
// operand.  Support DOFs hold zero by construction, so neighbours need no
// Dirichlet test; support rows are handled from the node-class byte.
#include "rso_internal.cuh"
#include <cmath>
#include <cuda_pipeline.h>

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

constexpr int FTX = 32, FTY = 8, FZC = 32;

template <typename T>
constexpr int fine_smem_bytes() {
  return (int)sizeof(T) * (4 * 3 * (FTX + 2) * (FTY + 2) + 3 * (FTX + 1) * (FTY + 1));
}

// MODE 0: out = f - K u;  MODE 1: out = K u (support rows pass u);
// MODE 2: out = u + omega D^-1 (f - K u)  (damped block Jacobi, D = 3x3 diagonal block)
template <typename T, int MODE>
__global__ void __launch_bounds__(FTX* FTY, sizeof(T) == 8 ? 2 : 3)
    k_fine(const Level L, const T* __restrict__ u, const T* __restrict__ f,
                                                   T* __restrict__ out, const T* __restrict__ rp, T omega) {
  constexpr int SX = FTX + 2, SY = FTY + 2, SP = SX * SY;  // one component of a node plane
  constexpr int EX = FTX + 1, EY = FTY + 1, EP = EX * EY;  // an element plane
  constexpr int NT = FTX * FTY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* su = reinterpret_cast<T*>(smem_raw);  // [4 slots][3 comps][SP]
  T* sr = su + 4 * 3 * SP;                 // [3 slots][EP]
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * FTX + tx;
  const int x0 = blockIdx.x * FTX, y0 = blockIdx.y * FTY;
  const int z0 = blockIdx.z * FZC;
  const int z1 = min(z0 + FZC, L.nz);
  const long long NP = L.NP;

  // node plane zp (in [-1, nz]) -> slot; element plane ep (in [-1, ez]) -> slot
  auto load_u = [&](int zp, int slot) {
    for (int i = tid; i < 3 * SP; i += NT) {
      const int c = i / SP, r = i - c * SP, sy = r / SX, sx = r - sy * SX;
      const int gx = x0 - 1 + sx, gy = y0 - 1 + sy;
      T* dst = su + (slot * 3 + c) * SP + r;
      if (gx <= L.nx && gy <= L.ny && zp <= L.nz)
        __pipeline_memcpy_async(dst, u + L.nidx(gx, gy, zp) + c * NP, sizeof(T));
      else
        *dst = T(0);
    }
  };
  auto load_r = [&](int ep, int slot) {
    for (int i = tid; i < EP; i += NT) {
      const int sy = i / EX, sx = i - sy * EX;
      const int gx = x0 - 1 + sx, gy = y0 - 1 + sy;
      T* dst = sr + slot * EP + i;
      if (gx <= L.ex && gy <= L.ey && ep <= L.ez)
        __pipeline_memcpy_async(dst, rp + L.eidx(gx, gy, ep), sizeof(T));
      else
        *dst = T(0);
    }
  };

  // prologue: node planes z0-1, z0, z0+1 and element planes z0-1, z0
  load_u(z0 - 1, (z0 + 3) & 3);
  load_u(z0, z0 & 3);
  load_r(z0 - 1, (z0 + 2) % 3);
  __pipeline_commit();
  load_u(z0 + 1, (z0 + 1) & 3);
  load_r(z0, z0 % 3);
  __pipeline_commit();

  const int x = x0 + tx, y = y0 + ty;
  const bool inside = x < L.nx && y < L.ny;
  for (int z = z0; z < z1; z++) {
    // stage the next planes while this one is computed
    if (z + 2 <= L.nz && z + 1 < z1 + 1) load_u(z + 2, (z + 2) & 3);
    if (z + 1 <= L.ez) load_r(z + 1, (z + 1) % 3);
    __pipeline_commit();
    __pipeline_wait_prior(1);
    __syncthreads();
    if (inside) {
      const long long n = L.nidx(x, y, z);
      const uint8_t cls = L.vclass[n];
      const bool work = (cls & NC_ACTIVE) && !(cls & NC_SUPPORT);
      T acc0 = 0, acc1 = 0, acc2 = 0;
      T D[6] = {0, 0, 0, 0, 0, 0};
      if (work) {
        const T* pu[3] = {su + ((z + 3) & 3) * 3 * SP, su + (z & 3) * 3 * SP, su + ((z + 1) & 3) * 3 * SP};
        const T* pr[2] = {sr + ((z + 2) % 3) * EP, sr + (z % 3) * EP};
        T r[8];
#pragma unroll
        for (int k = 0; k < 8; k++) r[k] = pr[k >> 2][(ty + ((k >> 1) & 1)) * EX + tx + (k & 1)];
        T a[8][3];
#pragma unroll
        for (int k = 0; k < 8; k++) a[k][0] = a[k][1] = a[k][2] = 0;
#pragma unroll
        for (int d = 0; d < 27; d++) {
          const int dx = d % 3 - 1, dy = d / 3 % 3 - 1, dz = d / 9 - 1;
          const T* q = pu[dz + 1] + (ty + 1 + dy) * SX + (tx + 1 + dx);
          const T u0 = q[0], u1 = q[SP], u2 = q[2 * SP];
#pragma unroll
          for (int k = 0; k < 8; k++) {
            const int kx = k & 1, ky = (k >> 1) & 1, kz = k >> 2;
            if ((dx == kx - 1 || dx == kx) && (dy == ky - 1 || dy == ky) && (dz == kz - 1 || dz == kz)) {
              const int vi = 7 - k;
              const int vj = (dx - kx + 1) + 2 * (dy - ky + 1) + 4 * (dz - kz + 1);
#pragma unroll
              for (int rr = 0; rr < 3; rr++) {
                // explicit fused chain: one FMA per matrix entry
                T s = a[k][rr];
                s = fma(k0<T>((vi * 3 + rr) * 24 + vj * 3 + 0), u0, s);
                s = fma(k0<T>((vi * 3 + rr) * 24 + vj * 3 + 1), u1, s);
                s = fma(k0<T>((vi * 3 + rr) * 24 + vj * 3 + 2), u2, s);
                a[k][rr] = s;
              }
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
        const T* c0 = su + (z & 3) * 3 * SP + (ty + 1) * SX + (tx + 1);
        out[n] = pass ? c0[0] : acc0;
        out[n + NP] = pass ? c0[SP] : acc1;
        out[n + 2 * NP] = pass ? c0[2 * SP] : acc2;
      } else {
        if (!work) {
          out[n] = 0; out[n + NP] = 0; out[n + 2 * NP] = 0;
        } else {
          const T* c0 = su + (z & 3) * 3 * SP + (ty + 1) * SX + (tx + 1);
          const T r0 = f[n] - acc0, r1 = f[n + NP] - acc1, r2 = f[n + 2 * NP] - acc2;
          // symmetric 3x3 inverse
          const T a = D[0], b = D[1], c = D[2], d = D[3], e = D[4], g = D[5];
          const T A = d * g - e * e, B = c * e - b * g, C = b * e - c * d;
          const T det = a * A + b * B + c * C;
          const T id = omega / det;
          const T E = a * g - c * c, F = b * c - a * e, I = a * d - b * b;
          out[n] = c0[0] + id * (A * r0 + B * r1 + C * r2);
          out[n + NP] = c0[SP] + id * (B * r0 + E * r1 + F * r2);
          out[n + 2 * NP] = c0[2 * SP] + id * (C * r0 + F * r1 + I * r2);
        }
      }
    }
    __syncthreads();
  }
  __pipeline_wait_prior(0);
}

// damped Jacobi from a zero iterate: out = omega D^-1 f (no neighbour reads)
template <typename T>
__global__ void __launch_bounds__(256) k_fine_jacobi0(const Level L, const T* __restrict__ f, T* __restrict__ out,
                                                      const T* __restrict__ rp, T omega) {
  const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
  if (x >= L.nx || y >= L.ny) return;
  const long long NP = L.NP, qx = L.qx, qxy = (long long)L.qx * L.qy;
  const long long n = L.nidx(x, y, z);
  const uint8_t cls = L.vclass[n];
  if (!(cls & NC_ACTIVE) || (cls & NC_SUPPORT)) {
    out[n] = 0; out[n + NP] = 0; out[n + 2 * NP] = 0;
    return;
  }
  const long long e0 = L.eidx(x - 1, y - 1, z - 1);
  T D[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const T r = rp[e0 + (k & 1) + ((k >> 1) & 1) * qx + (k >> 2) * qxy];
    const int vi = 7 - k;
    D[0] += r * k0<T>((vi * 3 + 0) * 24 + vi * 3 + 0);
    D[1] += r * k0<T>((vi * 3 + 0) * 24 + vi * 3 + 1);
    D[2] += r * k0<T>((vi * 3 + 0) * 24 + vi * 3 + 2);
    D[3] += r * k0<T>((vi * 3 + 1) * 24 + vi * 3 + 1);
    D[4] += r * k0<T>((vi * 3 + 1) * 24 + vi * 3 + 2);
    D[5] += r * k0<T>((vi * 3 + 2) * 24 + vi * 3 + 2);
  }
  const T r0 = f[n], r1 = f[n + NP], r2 = f[n + 2 * NP];
  const T a = D[0], b = D[1], c = D[2], d = D[3], e = D[4], g = D[5];
  const T A = d * g - e * e, B = c * e - b * g, C = b * e - c * d;
  const T det = a * A + b * B + c * C;
  const T id = omega / det;
  const T E = a * g - c * c, F = b * c - a * e, I = a * d - b * b;
  out[n] = id * (A * r0 + B * r1 + C * r2);
  out[n + NP] = id * (B * r0 + E * r1 + F * r2);
  out[n + 2 * NP] = id * (C * r0 + F * r1 + I * r2);
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
        for (int rr = 0; rr < 3; rr++) {
          T s = a[k][rr];
          s = fma(k0<T>((vi * 3 + rr) * 24 + vj * 3 + 0), u0, s);
          s = fma(k0<T>((vi * 3 + rr) * 24 + vj * 3 + 1), u1, s);
          s = fma(k0<T>((vi * 3 + rr) * 24 + vj * 3 + 2), u2, s);
          a[k][rr] = s;
        }
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

static inline dim3 plane_grid(const Level& l) { return dim3(cdiv(l.nx, 32), cdiv(l.ny, 8), l.nz); }
static inline dim3 march_grid(const Level& l) { return dim3(cdiv(l.nx, FTX), cdiv(l.ny, FTY), cdiv(l.nz, FZC)); }

template <typename T>
static inline int pcls(int c32, int c64) { return sizeof(T) == 4 ? c32 : c64; }

template <typename T, int MODE>
static rso_status launch_fine(rso_handle* h, const T* u, const T* f, T* out, const T* rp, double omega, int cls,
                              const char* what) {
  const Level& l = h->L[0];
  constexpr int smem = fine_smem_bytes<T>();
  static bool attr = false;
  if (!attr) {
    RSO_CHECK_CUDA(h, cudaFuncSetAttribute(k_fine<T, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr = true;
  }
  if (h->prof_on) prof_begin(h, cls, (double)l.nn);
  k_fine<T, MODE><<<march_grid(l), dim3(FTX, FTY), smem, h->stream>>>(l, u, f, out, rp, (T)omega);
  rso::note_launch();
  if (h->prof_on) prof_end(h, cls);
  return launch_check(h, what);
}

template <typename T>
rso_status fine_residual(rso_handle* h, const T* u, const T* f, T* r, const T* rp) {
  return launch_fine<T, 0>(h, u, f, r, rp, 0.0, pcls<T>(PC_FINE_RES32, PC_FINE_RES64), "fine_residual");
}
template <typename T>
rso_status fine_applyK(rso_handle* h, const T* u, T* f, const T* rp) {
  return launch_fine<T, 1>(h, u, u, f, rp, 0.0, pcls<T>(PC_FINE_RES32, PC_FINE_APPLYK64), "fine_applyK");
}
template <typename T>
rso_status fine_jacobi(rso_handle* h, const T* u_in, const T* f, T* u_out, const T* rp, double omega) {
  return launch_fine<T, 2>(h, u_in, f, u_out, rp, omega, pcls<T>(PC_FINE_JAC32, PC_FINE_JAC64), "fine_jacobi");
}
template <typename T>
rso_status fine_jacobi0(rso_handle* h, const T* f, T* u_out, const T* rp, double omega) {
  const Level& l = h->L[0];
  k_fine_jacobi0<T><<<plane_grid(l), dim3(32, 8), 0, h->stream>>>(l, f, u_out, rp, (T)omega);
  rso::note_launch();
  return launch_check(h, "fine_jacobi0");
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
  rso::note_launch();
  if (h->prof_on) prof_end(h, cls);
  return launch_check(h, "fine_gs");
}

template rso_status fine_residual<double>(rso_handle*, const double*, const double*, double*, const double*);
template rso_status fine_residual<float>(rso_handle*, const float*, const float*, float*, const float*);
template rso_status fine_applyK<double>(rso_handle*, const double*, double*, const double*);
template rso_status fine_applyK<float>(rso_handle*, const float*, float*, const float*);
template rso_status fine_jacobi<double>(rso_handle*, const double*, const double*, double*, const double*, double);
template rso_status fine_jacobi<float>(rso_handle*, const float*, const float*, float*, const float*, double);
template rso_status fine_jacobi0<double>(rso_handle*, const double*, double*, const double*, double);
template rso_status fine_jacobi0<float>(rso_handle*, const float*, float*, const float*, double);
template rso_status fine_gs<double>(rso_handle*, double*, const double*, const double*, int, int);
template rso_status fine_gs<float>(rso_handle*, float*, const float*, const float*, int, int);

}  // namespace rso
