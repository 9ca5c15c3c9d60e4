// Coarse levels: Galerkin operators, stencil smoothing/residuals, transfer
// operators and the coarsest dense FP64 solve.
//
// Galerkin operators are built element by element: a coarse element matrix
// is K_E = sum_children P_c^T K_c P_c with P_c the trilinear interpolation
// from the 8 coarse corners to a child's 8 nodes.  For the first coarsening
// the children are fine voxels, K_c = rho^p K0 with the rows/columns of
// support DOFs zeroed and 1e6 on their diagonal (the matrix behind
// restrict_stencil_nondyadic_OTFA_WS_kernel, grid/Grid.cu:1154-1268); for
// unconstrained voxels P^T (rho^p K0) P = rho^p T_pos with T_pos tabulated
// once per coarsening factor.  Deeper levels recurse on the coarse element
// matrices (equivalent to restrict_stencil_dyadic_kernel, grid/Grid.cu:882-939,
// which applies R K P to assembled stencils).  Stencils are then assembled
// from the element matrices, in FP64 and FP32.
#include "rso_internal.cuh"
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cooperative_groups.h>
#include <vector>

namespace cg = cooperative_groups;

namespace rso {

static const double DIRICHLET_W = 1e6;  // grid/Grid.cu:14

// ---------------------------------------------------------------- stencil kernels
// u is a plain pointer: the bottom kernels write it in earlier phases of the
// same launch, so its loads must be coherent ones
template <typename T>
__device__ __forceinline__ void stencil_apply(const Level& L, const T* __restrict__ st, const T* u,
                                              long long n, bool skip_centre, T acc[3]) {
  const long long NP = L.NP, px = L.px, pxy = (long long)L.px * L.py;
#pragma unroll
  for (int d = 0; d < 27; d++) {
    if (skip_centre && d == 13) continue;
    const long long nb = n + (d % 3 - 1) + (d / 3 % 3 - 1) * px + (d / 9 - 1) * pxy;
    const T u0 = u[nb], u1 = u[nb + NP], u2 = u[nb + 2 * NP];
#pragma unroll
    for (int r = 0; r < 3; r++) {
      T s = acc[r];
      s = fma(st[st_at<T>(NP, d * 9 + r * 3 + 0, n)], u0, s);
      s = fma(st[st_at<T>(NP, d * 9 + r * 3 + 1, n)], u1, s);
      s = fma(st[st_at<T>(NP, d * 9 + r * 3 + 2, n)], u2, s);
      acc[r] = s;
    }
  }
}

// Per-node variant for the large coarse levels, which are bandwidth-bound:
// one thread reads a node's 243 stencil entries and 27 neighbours once.
// MODE 0 residual, MODE 2 damped block Jacobi (out of place).
template <typename T, int MODE, int KB>
__global__ void __launch_bounds__(256) k_coarse(const Level L, const T* __restrict__ st, const T* __restrict__ u,
                                                const T* __restrict__ f, T* __restrict__ out, T omega,
                                                const T* __restrict__ uprev, T c1) {
  // blockIdx.z = z + nz * (chunk of KB systems): each stencil entry is read
  // once and applied to the chunk's systems
  const int chunk = blockIdx.z / L.nz;
  const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z - chunk * L.nz;
  if (x >= L.nx || y >= L.ny) return;
  const long long NP = L.NP, px = L.px, pxy = (long long)L.px * L.py, VS = 3 * NP;
  const int b0 = chunk * KB, nv = min(KB, L.nb - b0);
  const long long n = L.nidx(x, y, z);
  const bool act = (L.vclass[n] & NC_ACTIVE) != 0;
  T acc[KB][3];
#pragma unroll
  for (int j = 0; j < KB; j++) acc[j][0] = acc[j][1] = acc[j][2] = T(0);
  if (act) {
#pragma unroll
    for (int d = 0; d < 27; d++) {
      const long long nbr = n + (d % 3 - 1) + (d / 3 % 3 - 1) * px + (d / 9 - 1) * pxy;
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const T sv = st[st_at<T>(NP, d * 9 + r * 3 + c, n)];
#pragma unroll
          for (int j = 0; j < KB; j++)
            if (j < nv) acc[j][r] = fma(sv, u[(b0 + j) * VS + nbr + c * NP], acc[j][r]);
        }
    }
  }
  T S[9];
  if (MODE == 2 && act) {
#pragma unroll
    for (int i = 0; i < 9; i++) S[i] = st[st_at<T>(NP, 13 * 9 + i, n)];
  }
#pragma unroll
  for (int j = 0; j < KB; j++) {
    if (j >= nv) break;
    const long long o = (b0 + j) * VS + n;
    if (MODE == 0) {
#pragma unroll
      for (int r = 0; r < 3; r++) out[o + r * NP] = f[o + r * NP] - acc[j][r];
    } else {
      if (!act) { out[o] = 0; out[o + NP] = 0; out[o + 2 * NP] = 0; continue; }
      const T r0 = f[o] - acc[j][0], r1 = f[o + NP] - acc[j][1], r2 = f[o + 2 * NP] - acc[j][2];
      const T A = S[4] * S[8] - S[5] * S[7], B = -(S[3] * S[8] - S[5] * S[6]), C = S[3] * S[7] - S[4] * S[6];
      const T det = S[0] * A + S[1] * B + S[2] * C;
      const T id = omega / det;
      const T i01 = -(S[1] * S[8] - S[2] * S[7]), i02 = S[1] * S[5] - S[2] * S[4];
      const T i11 = S[0] * S[8] - S[2] * S[6], i12 = -(S[0] * S[5] - S[2] * S[3]);
      const T i21 = -(S[0] * S[7] - S[1] * S[6]), i22 = S[0] * S[4] - S[1] * S[3];
      const T p0 = uprev ? uprev[o] : T(0), p1 = uprev ? uprev[o + NP] : T(0), p2 = uprev ? uprev[o + 2 * NP] : T(0);
      out[o] = u[o] + c1 * (u[o] - p0) + id * (A * r0 + i01 * r1 + i02 * r2);
      out[o + NP] = u[o + NP] + c1 * (u[o + NP] - p1) + id * (B * r0 + i11 * r1 + i12 * r2);
      out[o + 2 * NP] = u[o + 2 * NP] + c1 * (u[o + 2 * NP] - p2) + id * (C * r0 + i21 * r1 + i22 * r2);
    }
  }
}

// FP32 variant for large single-system levels.  A group of four consecutive
// padded nodes (px is a multiple of 4, so a group never spans two rows and
// starts on 16 bytes) is taken by three threads, one per neighbour plane
// dz = -1, 0, +1: each streams the 81 stencil entries of its 9 neighbours
// (16-byte loads from the tiled FP32 stencil) and their values (one 16-byte
// load and two scalars per neighbour row), so three times the threads are in
// flight and each one's chain of loads is a third as long (the levels are a
// few hundred thousand nodes: one thread per group left the GPU under a wave,
// bound by each thread's latency).  The partial sums of planes -1 and +1 meet
// the centre plane's thread in shared memory, which adds them in a fixed
// order and finishes the node (residual, or damped block Jacobi / Chebyshev
// step with the diagonal block of its own plane).  Halo rows are skipped;
// halo and inactive nodes of a group are written as the per-node kernel
// leaves them (zero, or f for the residual).
constexpr int C4G = 64;  // node groups per CTA (blockDim (C4G, 3))
template <int MODE>
__global__ void __launch_bounds__(C4G * 3, 3) k_coarse4(const Level L, const float* __restrict__ st,
                                                     const float* __restrict__ u, const float* __restrict__ f,
                                                     float* __restrict__ out, float omega,
                                                     const float* __restrict__ uprev, float c1) {
  __shared__ float red[2][12][C4G];
  const int tg = threadIdx.x, pz = threadIdx.y;  // neighbour plane dz = pz - 1
  const long long g = blockIdx.x * (long long)C4G + tg;
  const long long NP = L.NP, px = L.px, pxy = (long long)L.px * L.py;
  const long long p0 = 4 * g;
  bool work = p0 < NP;
  int xp = 0;
  bool act[4] = {false, false, false, false};
  if (work) {
    // NP < 2^31 (checked by the launchers): 32-bit divisions
    const unsigned p0u = (unsigned)p0, pxyu = (unsigned)pxy, pxu = (unsigned)px;
    const int zp = (int)(p0u / pxyu);
    const unsigned rem = p0u - (unsigned)zp * pxyu;
    const int yp = (int)(rem / pxu);
    xp = (int)(rem - (unsigned)yp * pxu);
    work = !(zp < 1 || zp > L.nz || yp < 1 || yp > L.ny);  // halo row: stays zero
  }
  bool any = false;
  if (work) {
    const uchar4 cl4 = *reinterpret_cast<const uchar4*>(L.vclass + p0);
    const uint8_t cls[4] = {cl4.x, cl4.y, cl4.z, cl4.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int x = xp + k - 1;  // node x index
      act[k] = x >= 0 && x < L.nx && (cls[k] & NC_ACTIVE);
      any = any || act[k];
    }
  }
  float acc[3][4];
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int k = 0; k < 4; k++) acc[r][k] = 0.f;
  if (any) {
    const long long pl = p0 + (long long)(pz - 1) * pxy;
#pragma unroll
    for (int e = 0; e < 9; e++) {
      const int d = pz * 9 + e;
      const long long nb = pl + (e / 3 - 1) * px;  // same row offset, dx below
      const int dx = e % 3 - 1;
      float un[3][4];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const float* uc = u + nb + c * NP;
        const float4 m = *reinterpret_cast<const float4*>(uc);
        if (dx == 0) {
          un[c][0] = m.x; un[c][1] = m.y; un[c][2] = m.z; un[c][3] = m.w;
        } else if (dx < 0) {
          // the left neighbour of the group's first node; at xp = 0 that node
          // is halo (its result is discarded) and the read would leave the row
          un[c][0] = xp > 0 ? uc[-1] : 0.f; un[c][1] = m.x; un[c][2] = m.y; un[c][3] = m.z;
        } else {
          // likewise at the row's end: xp + 3 = px - 1 is halo
          un[c][0] = m.y; un[c][1] = m.z; un[c][2] = m.w; un[c][3] = xp + 4 < px ? uc[4] : 0.f;
        }
      }
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const float4 sv = *reinterpret_cast<const float4*>(st + st_at<float>(NP, d * 9 + r * 3 + c, p0));
          acc[r][0] = fmaf(sv.x, un[c][0], acc[r][0]);
          acc[r][1] = fmaf(sv.y, un[c][1], acc[r][1]);
          acc[r][2] = fmaf(sv.z, un[c][2], acc[r][2]);
          acc[r][3] = fmaf(sv.w, un[c][3], acc[r][3]);
        }
    }
  }
  if (pz != 1) {
    const int slot = pz >> 1;  // plane -1 -> 0, plane +1 -> 1
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int k = 0; k < 4; k++) red[slot][r * 4 + k][tg] = acc[r][k];
  }
  __syncthreads();
  if (pz != 1 || !work) return;
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int k = 0; k < 4; k++) acc[r][k] = (red[0][r * 4 + k][tg] + acc[r][k]) + red[1][r * 4 + k][tg];
  float res[3][4];
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const float4 fv = *reinterpret_cast<const float4*>(f + p0 + r * NP);
    // K u is zero at inactive nodes, as in the per-node kernel
    res[r][0] = fv.x - (act[0] ? acc[r][0] : 0.f); res[r][1] = fv.y - (act[1] ? acc[r][1] : 0.f);
    res[r][2] = fv.z - (act[2] ? acc[r][2] : 0.f); res[r][3] = fv.w - (act[3] ? acc[r][3] : 0.f);
  }
  if (MODE == 0) {
    // out = f - K u; at the halo nodes of the group f is zero, so they keep their zero
#pragma unroll
    for (int r = 0; r < 3; r++)
      *reinterpret_cast<float4*>(out + p0 + r * NP) = make_float4(res[r][0], res[r][1], res[r][2], res[r][3]);
    return;
  }
  float uo[3][4], up[3][4];
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const float4 uv = *reinterpret_cast<const float4*>(u + p0 + r * NP);
    uo[r][0] = uv.x; uo[r][1] = uv.y; uo[r][2] = uv.z; uo[r][3] = uv.w;
    float4 pv = make_float4(0.f, 0.f, 0.f, 0.f);
    if (uprev) pv = *reinterpret_cast<const float4*>(uprev + p0 + r * NP);
    up[r][0] = pv.x; up[r][1] = pv.y; up[r][2] = pv.z; up[r][3] = pv.w;
  }
  // the diagonal blocks, re-read (the centre plane's thread streamed them a
  // moment ago: cache hits) rather than held in registers through the loop
  float S[9][4];
#pragma unroll
  for (int i = 0; i < 9; i++) {
    const float4 sv = *reinterpret_cast<const float4*>(st + st_at<float>(NP, 13 * 9 + i, p0));
    S[i][0] = sv.x; S[i][1] = sv.y; S[i][2] = sv.z; S[i][3] = sv.w;
  }
  float o[3][4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    if (!act[k]) {
      o[0][k] = o[1][k] = o[2][k] = 0.f;
      continue;
    }
    float Sk[9];
#pragma unroll
    for (int i = 0; i < 9; i++) Sk[i] = S[i][k];
    const float r0 = res[0][k], r1 = res[1][k], r2 = res[2][k];
    const float A = Sk[4] * Sk[8] - Sk[5] * Sk[7], B = -(Sk[3] * Sk[8] - Sk[5] * Sk[6]),
                C = Sk[3] * Sk[7] - Sk[4] * Sk[6];
    const float det = Sk[0] * A + Sk[1] * B + Sk[2] * C;
    const float id = omega / det;
    const float i01 = -(Sk[1] * Sk[8] - Sk[2] * Sk[7]), i02 = Sk[1] * Sk[5] - Sk[2] * Sk[4];
    const float i11 = Sk[0] * Sk[8] - Sk[2] * Sk[6], i12 = -(Sk[0] * Sk[5] - Sk[2] * Sk[3]);
    const float i21 = -(Sk[0] * Sk[7] - Sk[1] * Sk[6]), i22 = Sk[0] * Sk[4] - Sk[1] * Sk[3];
    o[0][k] = uo[0][k] + c1 * (uo[0][k] - up[0][k]) + id * (A * r0 + i01 * r1 + i02 * r2);
    o[1][k] = uo[1][k] + c1 * (uo[1][k] - up[1][k]) + id * (B * r0 + i11 * r1 + i12 * r2);
    o[2][k] = uo[2][k] + c1 * (uo[2][k] - up[2][k]) + id * (C * r0 + i21 * r1 + i22 * r2);
  }
#pragma unroll
  for (int r = 0; r < 3; r++)
    *reinterpret_cast<float4*>(out + p0 + r * NP) = make_float4(o[r][0], o[r][1], o[r][2], o[r][3]);
}

// Row-split variant for the small, latency-bound levels (MODE as above).
// Thread (x, y, r) owns
// output component r of node (x, y, z), so each node's 243 stencil entries
// are read by three threads (81 each) and the small, latency-bound coarse
// levels get three times the independent loads in flight.  The damped
// Jacobi update exchanges the three residual components through shared
// memory.
constexpr int CTY = 4;
// thread (x, y, r) of a 32 x CTY x 3 tile at plane z of system bsys; ZERO:
// u read as zero (a first step from a zero iterate).  sres is the tile's
// shared exchange; every thread of the CTA calls this (MODE 2 synchronises it)
// The vectors are plain pointers here: the persistent bottom kernel writes
// them in earlier phases of the same launch, so their loads must be coherent
// ones (the per-level kernel's own parameters carry __restrict__).
template <typename T, int MODE, bool ZERO = false>
__device__ __forceinline__ void coarse_r_node(const Level& L, const T* __restrict__ st, const T* u, const T* f,
                                              T* out, T omega, const T* uprev, T c1, int x, int y, int z, int bsys,
                                              T (*sres)[CTY][32]) {
  {
    const long long off = (long long)bsys * 3 * L.NP;
    u += off;
    f += off;
    out += off;
    if (uprev != nullptr) uprev += off;
  }
  const int r = threadIdx.z;
  const bool in = x < L.nx && y < L.ny;
  const long long NP = L.NP, px = L.px, pxy = (long long)L.px * L.py;
  const long long n = in ? L.nidx(x, y, z) : 0;
  const bool act = in && (L.vclass[n] & NC_ACTIVE) != 0;
  T acc = 0;
  if (act && !ZERO) {
#pragma unroll
    for (int d = 0; d < 27; d++) {
      const long long nb = n + (d % 3 - 1) + (d / 3 % 3 - 1) * px + (d / 9 - 1) * pxy;
      acc = fma(st[st_at<T>(NP, d * 9 + r * 3 + 0, n)], u[nb], acc);
      acc = fma(st[st_at<T>(NP, d * 9 + r * 3 + 1, n)], u[nb + NP], acc);
      acc = fma(st[st_at<T>(NP, d * 9 + r * 3 + 2, n)], u[nb + 2 * NP], acc);
    }
  }
  if (MODE == 0) {
    if (in) out[n + r * NP] = f[n + r * NP] - acc;
    return;
  }
  const T res = act ? f[n + r * NP] - acc : T(0);
  sres[r][threadIdx.y][threadIdx.x] = res;
  __syncthreads();
  if (!in) return;
  if (!act) { out[n + r * NP] = 0; return; }
  T S[9];
#pragma unroll
  for (int i = 0; i < 9; i++) S[i] = st[st_at<T>(NP, 13 * 9 + i, n)];
  // row r of the adjugate of the 3x3 diagonal block
  const T c00 = S[4] * S[8] - S[5] * S[7], c01 = -(S[3] * S[8] - S[5] * S[6]), c02 = S[3] * S[7] - S[4] * S[6];
  const T det = S[0] * c00 + S[1] * c01 + S[2] * c02;
  T a0, a1, a2;
  if (r == 0) { a0 = c00; a1 = -(S[1] * S[8] - S[2] * S[7]); a2 = S[1] * S[5] - S[2] * S[4]; }
  else if (r == 1) { a0 = c01; a1 = S[0] * S[8] - S[2] * S[6]; a2 = -(S[0] * S[5] - S[2] * S[3]); }
  else { a0 = c02; a1 = -(S[0] * S[7] - S[1] * S[6]); a2 = S[0] * S[4] - S[1] * S[3]; }
  const T r0 = sres[0][threadIdx.y][threadIdx.x], r1 = sres[1][threadIdx.y][threadIdx.x],
          r2 = sres[2][threadIdx.y][threadIdx.x];
  const T ur = ZERO ? T(0) : u[n + r * NP], pr = uprev ? uprev[n + r * NP] : T(0);
  out[n + r * NP] = ur + c1 * (ur - pr) + (omega / det) * (a0 * r0 + a1 * r1 + a2 * r2);
}
template <typename T, int MODE>
__global__ void __launch_bounds__(32 * CTY * 3) k_coarse_r(const Level L, const T* __restrict__ st,
                                                           const T* __restrict__ u, const T* __restrict__ f,
                                                           T* __restrict__ out, T omega,
                                                           const T* __restrict__ uprev, T c1) {
  __shared__ T sres[3][CTY][32];
  const int bsys = blockIdx.z / L.nz;
  coarse_r_node<T, MODE>(L, st, u, f, out, omega, uprev, c1, blockIdx.x * 32 + threadIdx.x,
                         blockIdx.y * CTY + threadIdx.y, blockIdx.z - bsys * L.nz, bsys, sres);
}

// Small levels (a few thousand to a few ten thousand nodes): the per-row
// kernel above leaves most of the GPU idle and each thread with a chain of 81
// stencil and 81 vector loads.  Here nine threads share a node: thread (r, pz)
// takes row r over the nine neighbours of plane z - 1 + pz (27 loads of each),
// and the three planes' partial sums meet in shared memory.  Same arithmetic
// per plane as k_coarse_r, summed plane by plane (the FP32 result may differ in
// the last bits).  MODE 0 residual, MODE 2 damped block Jacobi / Chebyshev step.
constexpr int CTY9 = 2;
template <typename T, int MODE>
__global__ void __launch_bounds__(32 * CTY9 * 9) k_coarse_r9(const Level L, const T* __restrict__ st,
                                                             const T* __restrict__ u, const T* __restrict__ f,
                                                             T* __restrict__ out, T omega,
                                                             const T* __restrict__ uprev, T c1) {
  __shared__ T spart[3][3][CTY9][32];  // [plane][row]
  __shared__ T sres[3][CTY9][32];
  const int bsys = blockIdx.z / L.nz;
  const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * CTY9 + threadIdx.y, z = blockIdx.z - bsys * L.nz;
  {
    const long long off = (long long)bsys * 3 * L.NP;
    u += off;
    f += off;
    out += off;
    if (uprev != nullptr) uprev += off;
  }
  const int r = threadIdx.z % 3, pz = threadIdx.z / 3;
  const bool in = x < L.nx && y < L.ny;
  const long long NP = L.NP, px = L.px, pxy = (long long)L.px * L.py;
  const long long n = in ? L.nidx(x, y, z) : 0;
  const bool act = in && (L.vclass[n] & NC_ACTIVE) != 0;
  T acc = 0;
  if (act) {
#pragma unroll
    for (int d9 = 0; d9 < 9; d9++) {
      const int d = pz * 9 + d9;
      const long long nb = n + (d % 3 - 1) + (d / 3 % 3 - 1) * px + (d / 9 - 1) * pxy;
      acc = fma(st[st_at<T>(NP, d * 9 + r * 3 + 0, n)], u[nb], acc);
      acc = fma(st[st_at<T>(NP, d * 9 + r * 3 + 1, n)], u[nb + NP], acc);
      acc = fma(st[st_at<T>(NP, d * 9 + r * 3 + 2, n)], u[nb + 2 * NP], acc);
    }
  }
  spart[pz][r][threadIdx.y][threadIdx.x] = acc;
  __syncthreads();
  if (pz == 0) {
    const T a = spart[0][r][threadIdx.y][threadIdx.x] + spart[1][r][threadIdx.y][threadIdx.x] +
                spart[2][r][threadIdx.y][threadIdx.x];
    if (MODE == 0) {
      if (in) out[n + r * NP] = f[n + r * NP] - a;
      return;
    }
    sres[r][threadIdx.y][threadIdx.x] = act ? f[n + r * NP] - a : T(0);
  }
  if (MODE == 0) return;
  __syncthreads();
  if (pz != 0 || !in) return;
  if (!act) { out[n + r * NP] = 0; return; }
  T S[9];
#pragma unroll
  for (int i = 0; i < 9; i++) S[i] = st[st_at<T>(NP, 13 * 9 + i, n)];
  // row r of the adjugate of the 3x3 diagonal block
  const T c00 = S[4] * S[8] - S[5] * S[7], c01 = -(S[3] * S[8] - S[5] * S[6]), c02 = S[3] * S[7] - S[4] * S[6];
  const T det = S[0] * c00 + S[1] * c01 + S[2] * c02;
  T a0, a1, a2;
  if (r == 0) { a0 = c00; a1 = -(S[1] * S[8] - S[2] * S[7]); a2 = S[1] * S[5] - S[2] * S[4]; }
  else if (r == 1) { a0 = c01; a1 = S[0] * S[8] - S[2] * S[6]; a2 = -(S[0] * S[5] - S[2] * S[3]); }
  else { a0 = c02; a1 = -(S[0] * S[7] - S[1] * S[6]); a2 = S[0] * S[4] - S[1] * S[3]; }
  const T r0 = sres[0][threadIdx.y][threadIdx.x], r1 = sres[1][threadIdx.y][threadIdx.x],
          r2 = sres[2][threadIdx.y][threadIdx.x];
  const T ur = u[n + r * NP], pr = uprev ? uprev[n + r * NP] : T(0);
  out[n + r * NP] = ur + c1 * (ur - pr) + (omega / det) * (a0 * r0 + a1 * r1 + a2 * r2);
}

// one colour of the point Gauss-Seidel sweep on stored stencils (gs_relax_kernel grid/Grid.cu:1497-1609)
template <typename T>
__global__ void __launch_bounds__(256) k_coarse_gs(const Level L, const T* __restrict__ st, T* __restrict__ u,
                                                   const T* __restrict__ f, int cx, int cy, int cz, int rev) {
  const int x = 2 * (blockIdx.x * 32 + threadIdx.x) + cx;
  const int y = 2 * (blockIdx.y * 8 + threadIdx.y) + cy;
  const int z = 2 * blockIdx.z + cz;
  if (x >= L.nx || y >= L.ny || z >= L.nz) return;
  const long long NP = L.NP;
  const long long n = L.nidx(x, y, z);
  if (!(L.vclass[n] & NC_ACTIVE)) return;
  T acc[3] = {0, 0, 0};
  stencil_apply<T>(L, st, u, n, true, acc);
  T v[3] = {u[n], u[n + NP], u[n + 2 * NP]};
#pragma unroll
  for (int t = 0; t < 3; t++) {
    const int r = rev ? 2 - t : t;
    T s = f[n + r * NP] - acc[r];
#pragma unroll
    for (int c = 0; c < 3; c++)
      if (c != r) s -= st[st_at<T>(NP, 13 * 9 + r * 3 + c, n)] * v[c];
    v[r] = s / st[st_at<T>(NP, 13 * 9 + r * 3 + r, n)];
  }
  u[n] = v[0]; u[n + NP] = v[1]; u[n + 2 * NP] = v[2];
}

// ---------------------------------------------------------------- transfers
// f_c(X) = sum_x w(x - F X) r_f(x), w = prod (F-|d|)/F  (R = P^T)
// Restriction in two separable passes.  Pass 1 (one thread per fine column
// (x, y) and coarse plane Z) filters along z into the scratch array
// t[c][Z][y][x]; pass 2 (one thread per coarse node) filters along y and x.
// Weights (F - |d|) / F per axis, d in (-F, F).
template <typename T, int F>
__global__ void k_restrict_z(const Level Fl, int nZ, const T* __restrict__ rf, T* __restrict__ t) {
  const int bsys = blockIdx.z / nZ;
  const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y, Z = blockIdx.z - bsys * nZ;
  if (x >= Fl.nx || y >= Fl.ny) return;
  rf += (long long)bsys * 3 * Fl.NP;
  t += (long long)bsys * 3 * Fl.nx * Fl.ny * nZ;
  T s0 = 0, s1 = 0, s2 = 0;
#pragma unroll
  for (int dz = -F + 1; dz < F; dz++) {
    const int z = F * Z + dz;
    if (z < 0 || z >= Fl.nz) continue;
    const long long n = Fl.nidx(x, y, z);
    const T w = (T)(F - (dz < 0 ? -dz : dz)) / (T)F;
    s0 += w * rf[n]; s1 += w * rf[n + Fl.NP]; s2 += w * rf[n + 2 * Fl.NP];
  }
  const long long plane = (long long)Fl.nx * Fl.ny, comp = plane * nZ;
  const long long i = (long long)Z * plane + (long long)y * Fl.nx + x;
  t[i] = s0; t[i + comp] = s1; t[i + 2 * comp] = s2;
}

// FP32, single system: pass 1 over four consecutive padded fine nodes per
// thread (16-byte loads and stores; px is a multiple of 4), into t laid out
// like the fine level's padded planes, t[c][Z][py][px].  Same arithmetic, in
// the same order, as k_restrict_z; the padding entries of t are never read.
template <int F>
__global__ void __launch_bounds__(256) k_restrict_z_v4(const Level Fl, int nZ, const float* __restrict__ rf,
                                                       float* __restrict__ t) {
  const long long pxy = (long long)Fl.px * Fl.py, off = 4 * (blockIdx.x * (long long)blockDim.x + threadIdx.x);
  const int Z = blockIdx.y;
  if (off >= pxy) return;
  float4 s[3];
#pragma unroll
  for (int c = 0; c < 3; c++) s[c] = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
  for (int dz = -F + 1; dz < F; dz++) {
    const int z = F * Z + dz;
    if (z < 0 || z >= Fl.nz) continue;
    const float* src = rf + pxy * (z + 1) + off;
    const float w = (float)(F - (dz < 0 ? -dz : dz)) / (float)F;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float4 v = *reinterpret_cast<const float4*>(src + c * Fl.NP);
      s[c].x += w * v.x; s[c].y += w * v.y; s[c].z += w * v.z; s[c].w += w * v.w;
    }
  }
  const long long comp = pxy * nZ;
#pragma unroll
  for (int c = 0; c < 3; c++) *reinterpret_cast<float4*>(t + c * comp + Z * pxy + off) = s[c];
}

// FP32, single system: the xy filter of the padded-plane t as two separable
// passes, y into ty[c][Z][Yc][px] (16-byte vectors along x) and x into the
// coarse nodes, 7 + 7 loads per output where the fused pass makes 49 (the
// sums grouped by axis, so the last bits may differ from k_restrict_xy)
template <int F>
__global__ void __launch_bounds__(256) k_restrict_y_v4(const Level Fl, const Level C, const float* __restrict__ t,
                                                       float* __restrict__ ty) {
  const int ng = Fl.px / 4;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x, Z = blockIdx.y;
  if (idx >= ng * C.ny) return;
  const int Yc = idx / ng, g = idx - Yc * ng;
  const long long plane = (long long)Fl.px * Fl.py, comp = plane * C.nz;
  const long long ocomp = (long long)C.nz * C.ny * Fl.px;
  float4 acc[3];
#pragma unroll
  for (int c = 0; c < 3; c++) acc[c] = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
  for (int dy = -F + 1; dy < F; dy++) {
    const int y = F * Yc + dy;
    if (y < 0 || y >= Fl.ny) continue;
    const float w = (float)(F - (dy < 0 ? -dy : dy)) / (float)F;
    const float* src = t + (long long)Z * plane + (long long)(y + 1) * Fl.px + 4 * g;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float4 v = *reinterpret_cast<const float4*>(src + c * comp);
      acc[c].x += w * v.x; acc[c].y += w * v.y; acc[c].z += w * v.z; acc[c].w += w * v.w;
    }
  }
  float* dst = ty + ((long long)Z * C.ny + Yc) * Fl.px + 4 * g;
#pragma unroll
  for (int c = 0; c < 3; c++) *reinterpret_cast<float4*>(dst + c * ocomp) = acc[c];
}
template <int F>
__global__ void k_restrict_x(const Level Fl, const Level C, const float* __restrict__ ty, float* __restrict__ fc) {
  const int X = blockIdx.x * 32 + threadIdx.x, Y = blockIdx.y * 8 + threadIdx.y, Z = blockIdx.z;
  if (X >= C.nx || Y >= C.ny) return;
  const long long nC = C.nidx(X, Y, Z);
  const long long ocomp = (long long)C.nz * C.ny * Fl.px;
  float s0 = 0.f, s1 = 0.f, s2 = 0.f;
  if (C.vclass[nC] & NC_ACTIVE) {
    const float* row = ty + ((long long)Z * C.ny + Y) * Fl.px + 1;  // padded x: fine x + 1
#pragma unroll
    for (int dx = -F + 1; dx < F; dx++) {
      const int x = F * X + dx;
      if (x < 0 || x >= Fl.nx) continue;
      const float w = (float)(F - (dx < 0 ? -dx : dx)) / (float)F;
      s0 += w * row[x]; s1 += w * row[x + ocomp]; s2 += w * row[x + 2 * ocomp];
    }
  }
  fc[nC] = s0; fc[nC + C.NP] = s1; fc[nC + 2 * C.NP] = s2;
}

// PAD: t laid out like the fine level's padded planes, t[c][Z][py][px] (the
// layout k_restrict_z_v4 writes)
template <typename T, int F, bool PAD = false>
__global__ void k_restrict_xy(const Level Fl, const Level C, const T* __restrict__ t, T* __restrict__ fc) {
  const int bsys = blockIdx.z / C.nz;
  const int X = blockIdx.x * 32 + threadIdx.x, Y = blockIdx.y * 8 + threadIdx.y, Z = blockIdx.z - bsys * C.nz;
  if (X >= C.nx || Y >= C.ny) return;
  const long long plane = PAD ? (long long)Fl.px * Fl.py : (long long)Fl.nx * Fl.ny, comp = plane * C.nz;
  const long long rowl = PAD ? Fl.px : Fl.nx, o0 = PAD ? Fl.px + 1 : 0;  // t index of fine (x, y): o0 + y rowl + x
  t += (long long)bsys * 3 * comp;
  fc += (long long)bsys * 3 * C.NP;
  const long long nC = C.nidx(X, Y, Z);
  T s0 = 0, s1 = 0, s2 = 0;
  if (C.vclass[nC] & NC_ACTIVE) {
    const T* tz = t + (long long)Z * plane + o0;
#pragma unroll
    for (int dy = -F + 1; dy < F; dy++) {
      const int y = F * Y + dy;
      if (y < 0 || y >= Fl.ny) continue;
      const T wy = (T)(F - (dy < 0 ? -dy : dy)) / (T)F;
#pragma unroll
      for (int dx = -F + 1; dx < F; dx++) {
        const int x = F * X + dx;
        if (x < 0 || x >= Fl.nx) continue;
        const T w = wy * ((T)(F - (dx < 0 ? -dx : dx)) / (T)F);
        const long long i = (long long)y * rowl + x;
        s0 += w * tz[i]; s1 += w * tz[i + comp]; s2 += w * tz[i + 2 * comp];
      }
    }
  }
  fc[nC] = s0; fc[nC + C.NP] = s1; fc[nC + 2 * C.NP] = s2;
}

// u_f += P u_c at active, non-support fine nodes (trilinear, F = 2 or 4).
// One thread per fine node, so fine loads and stores are coalesced.  The
// warp's 32 nodes span 32/F + 1 coarse x positions: lane l folds the coarse
// column X = xb + l along y and z (12 loads), and each node takes its two
// x-corners from the lanes that hold them by shuffle.
template <typename T, int F>
__global__ void k_prolong(const Level Fl, const Level C, const T* __restrict__ uc, T* __restrict__ uf) {
  const int lane = threadIdx.x;
  const int bsys = blockIdx.z / Fl.nz;
  const int x = blockIdx.x * 32 + lane, y = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z - bsys * Fl.nz;
  uc += (long long)bsys * 3 * C.NP;
  uf += (long long)bsys * 3 * Fl.NP;
  const bool yok = y < Fl.ny;
  const int xb = blockIdx.x * (32 / F);
  const int Y0 = y / F, Z0 = z / F, oy = y - F * Y0, oz = z - F * Z0;
  const T wy[2] = {(T)(F - oy) / (T)F, (T)oy / (T)F};
  const T wz[2] = {(T)(F - oz) / (T)F, (T)oz / (T)F};
  T E[3] = {T(0), T(0), T(0)};
  const int X = xb + lane;
  if (yok && X <= C.nx) {  // index C.nx is the padded halo (zero)
    const long long c0 = C.nidx(X, Y0, Z0), cpx = C.px, cpxy = (long long)C.px * C.py;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      T s = 0;
#pragma unroll
      for (int k = 0; k < 4; k++) s += wy[k & 1] * wz[k >> 1] * uc[c0 + (k & 1) * cpx + (k >> 1) * cpxy + c * C.NP];
      E[c] = s;
    }
  }
  const int X0 = x / F - xb, ox = x - F * (x / F);
  T e0[3], e1[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    e0[c] = __shfl_sync(0xffffffffu, E[c], X0);
    e1[c] = __shfl_sync(0xffffffffu, E[c], X0 + 1);
  }
  if (x >= Fl.nx || !yok) return;
  const long long n = Fl.nidx(x, y, z);
  const uint8_t cls = Fl.vclass[n];
  const T u0 = uf[n], u1 = uf[n + Fl.NP], u2 = uf[n + 2 * Fl.NP];
  if (!(cls & NC_ACTIVE) || (cls & NC_SUPPORT)) return;
  const T w1 = (T)ox / (T)F, w0 = (T)(F - ox) / (T)F;
  uf[n] = u0 + (w0 * e0[0] + w1 * e1[0]);
  uf[n + Fl.NP] = u1 + (w0 * e0[1] + w1 * e1[1]);
  uf[n + 2 * Fl.NP] = u2 + (w0 * e0[2] + w1 * e1[2]);
}

// FP32, single system: four consecutive padded fine nodes per thread (px is a
// multiple of 4), the fine vector and node classes as 16-byte vectors, the
// yz-interpolated coarse values of the (at most four) coarse columns the group
// touches computed once.  Same arithmetic, in the same order, as k_prolong.
template <int F>
__global__ void __launch_bounds__(256) k_prolong_v4(const Level Fl, const Level C, const float* __restrict__ uc,
                                                    float* __restrict__ uf) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long NP = Fl.NP, px = Fl.px, pxy = (long long)Fl.px * Fl.py;
  const long long p0 = 4 * g;
  if (p0 >= NP) return;
  const int zp = (int)(p0 / pxy);
  const long long rem = p0 - zp * pxy;
  const int yp = (int)(rem / px), xp = (int)(rem - yp * px);
  if (zp < 1 || zp > Fl.nz || yp < 1 || yp > Fl.ny) return;
  const uchar4 cl4 = *reinterpret_cast<const uchar4*>(Fl.vclass + p0);
  const uint8_t cls[4] = {cl4.x, cl4.y, cl4.z, cl4.w};
  bool upd[4];
  bool any = false;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int x = xp - 1 + k;
    upd[k] = x >= 0 && x < Fl.nx && (cls[k] & NC_ACTIVE) && !(cls[k] & NC_SUPPORT);
    any = any || upd[k];
  }
  if (!any) return;
  const int y = yp - 1, z = zp - 1;
  const int Y0 = y / F, Z0 = z / F, oy = y - F * Y0, oz = z - F * Z0;
  const float wy[2] = {(float)(F - oy) / (float)F, (float)oy / (float)F};
  const float wz[2] = {(float)(F - oz) / (float)F, (float)oz / (float)F};
  const int x_first = max(xp - 1, 0), x_last = min(xp + 2, Fl.nx - 1);
  const int Xa = x_first / F, Xb = x_last / F + 1;
  const long long cpx = C.px, cpxy = (long long)C.px * C.py;
  float E[4][3];
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int X = Xa + j;
#pragma unroll
    for (int c = 0; c < 3; c++) E[j][c] = 0.f;
    if (X <= Xb && X <= C.nx) {  // index C.nx is the padded halo (zero)
      const long long c0 = C.nidx(X, Y0, Z0);
#pragma unroll
      for (int c = 0; c < 3; c++) {
        float s = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) s += wy[k & 1] * wz[k >> 1] * uc[c0 + (k & 1) * cpx + (k >> 1) * cpxy + c * C.NP];
        E[j][c] = s;
      }
    }
  }
  float u[3][4];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float4 m = *reinterpret_cast<const float4*>(uf + p0 + c * NP);
    u[c][0] = m.x; u[c][1] = m.y; u[c][2] = m.z; u[c][3] = m.w;
  }
#pragma unroll
  for (int k = 0; k < 4; k++) {
    if (!upd[k]) continue;
    const int x = xp - 1 + k, X0 = x / F, ox = x - F * X0, j = X0 - Xa;
    const float w1 = (float)ox / (float)F, w0 = (float)(F - ox) / (float)F;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      float e0 = 0.f, e1 = 0.f;
#pragma unroll
      for (int q = 0; q < 3; q++)
        if (q == j) { e0 = E[q][c]; e1 = E[q + 1][c]; }
      u[c][k] = u[c][k] + (w0 * e0 + w1 * e1);
    }
  }
#pragma unroll
  for (int c = 0; c < 3; c++)
    *reinterpret_cast<float4*>(uf + p0 + c * NP) = make_float4(u[c][0], u[c][1], u[c][2], u[c][3]);
}

// FP32, single system: one warp per fine row (y, z).  The lanes first fold the
// row's coarse columns along y and z into shared memory (E[c][X], X = 0..C.nx,
// index C.nx the zero halo), then update four consecutive padded fine nodes
// each with 16-byte loads and stores, taking every node's two x-corners from
// E: 12 coarse loads per coarse column instead of up to 36 per four nodes.
// Same arithmetic, in the same order, as k_prolong.
constexpr int PROW_WARPS = 8;
template <int F>
__global__ void __launch_bounds__(32 * PROW_WARPS) k_prolong_row(const Level Fl, const Level C,
                                                                 const float* __restrict__ uc, float* __restrict__ uf) {
  extern __shared__ float sE_all[];  // [PROW_WARPS][3][C.nx + 1]
  const int lane = threadIdx.x, w = threadIdx.y;
  const int y = blockIdx.x * PROW_WARPS + w, z = blockIdx.y;
  if (y >= Fl.ny) return;  // whole warp
  const int ncol = C.nx + 1;
  float* sE = sE_all + w * 3 * ncol;
  const int Y0 = y / F, Z0 = z / F, oy = y - F * Y0, oz = z - F * Z0;
  const float wy[2] = {(float)(F - oy) / (float)F, (float)oy / (float)F};
  const float wz[2] = {(float)(F - oz) / (float)F, (float)oz / (float)F};
  const long long cpx = C.px, cpxy = (long long)C.px * C.py;
  for (int X = lane; X < ncol; X += 32) {
    const long long c0 = C.nidx(X, Y0, Z0);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      float s = 0;
#pragma unroll
      for (int k = 0; k < 4; k++) s += wy[k & 1] * wz[k >> 1] * uc[c0 + (k & 1) * cpx + (k >> 1) * cpxy + c * C.NP];
      sE[c * ncol + X] = s;
    }
  }
  __syncwarp();
  const long long NP = Fl.NP, rb = (long long)Fl.px * ((y + 1) + (long long)Fl.py * (z + 1));
  for (int gq = lane; 4 * gq < Fl.px; gq += 32) {
    const long long p0 = rb + 4 * gq;
    const uchar4 cl4 = *reinterpret_cast<const uchar4*>(Fl.vclass + p0);
    const uint8_t cls[4] = {cl4.x, cl4.y, cl4.z, cl4.w};
    bool upd[4];
    bool any = false;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int x = 4 * gq - 1 + k;
      upd[k] = x >= 0 && x < Fl.nx && (cls[k] & NC_ACTIVE) && !(cls[k] & NC_SUPPORT);
      any = any || upd[k];
    }
    if (!any) continue;
    float u[3][4];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float4 m = *reinterpret_cast<const float4*>(uf + p0 + c * NP);
      u[c][0] = m.x; u[c][1] = m.y; u[c][2] = m.z; u[c][3] = m.w;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      if (!upd[k]) continue;
      const int x = 4 * gq - 1 + k, X0 = x / F, ox = x - F * X0;
      const float w1 = (float)ox / (float)F, w0 = (float)(F - ox) / (float)F;
#pragma unroll
      for (int c = 0; c < 3; c++) u[c][k] = u[c][k] + (w0 * sE[c * ncol + X0] + w1 * sE[c * ncol + X0 + 1]);
    }
#pragma unroll
    for (int c = 0; c < 3; c++)
      *reinterpret_cast<float4*>(uf + p0 + c * NP) = make_float4(u[c][0], u[c][1], u[c][2], u[c][3]);
  }
}

// ---------------------------------------------------------------- Galerkin
__device__ __forceinline__ double pw(int F, int o, int A) { return A ? (double)o / F : (double)(F - o) / F; }

// Support-free children enter the first-level coarse element matrices as a
// product KE[E] = sum_pos w[E][pos] T1[pos] (w = rho^p of child pos, 0 for
// inactive or support-touching children; T1[pos] the 576 entries of child
// pos's element matrix seen from the coarse element's nodes), done by
// k_galerkin_first; the support-touching children are added by
// k_galerkin_fix on the few coarse elements that have them.
__global__ void k_elem_fixmask(const Level Fl, uint8_t* __restrict__ efix) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= Fl.ne) return;
  const int x = i % Fl.ex, y = (i / Fl.ex) % Fl.ey, z = i / ((long long)Fl.ex * Fl.ey);
  unsigned m = 0;
#pragma unroll
  for (int a = 0; a < 8; a++)
    if (Fl.vclass[Fl.nidx(x + (a & 1), y + ((a >> 1) & 1), z + (a >> 2))] & NC_SUPPORT) m |= 1u << a;
  efix[Fl.eidx(x, y, z)] = (uint8_t)m;
}

// KE (576 x ne, column per coarse element) = T1 (576 x F3) . w (F3 x ne),
// w formed on the fly from the children's rho^p.  A CTA takes GE coarse
// elements: their weights go to shared memory once, then the 576 rows pass
// in chunks of 64 staged from T1; a thread accumulates 4 rows x 2 elements
// in FP64 (each output is one ordered sum over the F3 children).
constexpr int GE = 32, GM = 64;
template <int F>
__global__ void __launch_bounds__(256) k_galerkin_first(const Level Fl, const Level C, const double* __restrict__ rp,
                                                        const uint8_t* __restrict__ efix,
                                                        const double* __restrict__ T1, double* __restrict__ KE) {
  constexpr int F3 = F * F * F;
  __shared__ __align__(16) double Ws[F3][GE];
  __shared__ __align__(16) double Ts[F3][GM];
  const int t = threadIdx.x;
  const long long E0 = (long long)blockIdx.x * GE;
  for (int idx = t; idx < F3 * GE; idx += 256) {
    const int pos = idx / GE, j = idx - pos * GE;
    const long long E = E0 + j;
    double r = 0.0;
    if (E < C.ne) {
      const int X = E % C.ex, Y = (E / C.ex) % C.ey, Z = E / ((long long)C.ex * C.ey);
      const int x = X * F + pos % F, y = Y * F + (pos / F) % F, z = Z * F + pos / (F * F);
      if (x < Fl.ex && y < Fl.ey && z < Fl.ez) {
        const long long e = Fl.eidx(x, y, z);
        if (Fl.emask[e] && !efix[e]) r = rp[e];
      }
    }
    Ws[pos][j] = r;
  }
  const int ti = t & 15, te = t >> 4;  // rows 4 ti .. 4 ti + 3 of the chunk, elements 2 te, 2 te + 1
  for (int m0 = 0; m0 < 576; m0 += GM) {
    __syncthreads();  // Ws complete (first chunk); Ts free (later chunks)
    for (int idx = t; idx < F3 * GM; idx += 256) {
      const int k = idx / GM, i = idx - k * GM;
      Ts[k][i] = T1[(long long)k * 576 + m0 + i];
    }
    __syncthreads();
    double acc[4][2] = {};
#pragma unroll 8
    for (int k = 0; k < F3; k++) {
      const double2 a01 = *reinterpret_cast<const double2*>(&Ts[k][4 * ti]);
      const double2 a23 = *reinterpret_cast<const double2*>(&Ts[k][4 * ti + 2]);
      const double2 b = *reinterpret_cast<const double2*>(&Ws[k][2 * te]);
      const double a[4] = {a01.x, a01.y, a23.x, a23.y};
#pragma unroll
      for (int r = 0; r < 4; r++) {
        acc[r][0] = fma(a[r], b.x, acc[r][0]);
        acc[r][1] = fma(a[r], b.y, acc[r][1]);
      }
    }
#pragma unroll
    for (int c = 0; c < 2; c++) {
      const long long E = E0 + 2 * te + c;
      if (E >= C.ne) continue;
      double* o = KE + E * 576 + m0 + 4 * ti;
      *reinterpret_cast<double2*>(o) = make_double2(acc[0][c], acc[1][c]);
      *reinterpret_cast<double2*>(o + 2) = make_double2(acc[2][c], acc[3][c]);
    }
  }
}

// support-touching children of listed coarse elements, added to KE
__global__ void __launch_bounds__(288) k_galerkin_fix(const Level Fl, const Level C, int F,
                                                      const double* __restrict__ rp, const double* __restrict__ K0g,
                                                      const uint8_t* __restrict__ efix, const int* __restrict__ list,
                                                      double* __restrict__ KE) {
  const long long E = list[blockIdx.x];
  const int X = E % C.ex, Y = (E / C.ex) % C.ey, Z = E / ((long long)C.ex * C.ey);
  const int t = threadIdx.x;
  double acc[2] = {0, 0};
  for (int pz = 0; pz < F; pz++)
    for (int py = 0; py < F; py++)
      for (int px = 0; px < F; px++) {
        const int x = X * F + px, y = Y * F + py, z = Z * F + pz;
        if (x >= Fl.ex || y >= Fl.ey || z >= Fl.ez) continue;
        const long long e = Fl.eidx(x, y, z);
        const unsigned fixmask = efix[e];
        if (!Fl.emask[e] || !fixmask) continue;
        const double r = rp[e];
        for (int h2 = 0; h2 < 2; h2++) {
          const int ent = t + 288 * h2;
          const int row = ent / 24, col = ent % 24;
          const int A = row / 3, i = row % 3, B = col / 3, j = col % 3;
          double s = 0;
          for (int a = 0; a < 8; a++) {
            const double wa = pw(F, px + (a & 1), A & 1) * pw(F, py + ((a >> 1) & 1), (A >> 1) & 1) *
                              pw(F, pz + (a >> 2), A >> 2);
            if (wa == 0) continue;
            for (int b = 0; b < 8; b++) {
              const double wb = pw(F, px + (b & 1), B & 1) * pw(F, py + ((b >> 1) & 1), (B >> 1) & 1) *
                                pw(F, pz + (b >> 2), B >> 2);
              if (wb == 0) continue;
              double kv;
              if ((fixmask >> a & 1u) || (fixmask >> b & 1u)) kv = (a == b && i == j) ? DIRICHLET_W : 0.0;
              else kv = r * K0g[(a * 3 + i) * 24 + b * 3 + j];
              s += wa * wb * kv;
            }
          }
          acc[h2] += s;
        }
      }
  KE[E * 576 + t] += acc[0];
  KE[E * 576 + t + 288] += acc[1];
}

// dyadic recursion on element matrices
__global__ void __launch_bounds__(288) k_galerkin_next(const Level Fl, const Level C, const double* __restrict__ KEf,
                                                       double* __restrict__ KEc) {
  __shared__ double K[576];
  __shared__ double Tm[576];
  const long long E = blockIdx.x;
  const int X = E % C.ex, Y = (E / C.ex) % C.ey, Z = E / ((long long)C.ex * C.ey);
  const int t = threadIdx.x;
  double acc[2] = {0, 0};
  if (C.emask[C.eidx(X, Y, Z)]) {
    for (int c = 0; c < 8; c++) {
      const int px = c & 1, py = (c >> 1) & 1, pz = c >> 2;
      const int x = 2 * X + px, y = 2 * Y + py, z = 2 * Z + pz;
      if (x >= Fl.ex || y >= Fl.ey || z >= Fl.ez) continue;
      if (!Fl.emask[Fl.eidx(x, y, z)]) continue;
      const long long ef = x + (long long)Fl.ex * (y + (long long)Fl.ey * z);
      __syncthreads();
      K[t] = KEf[ef * 576 + t];
      K[t + 288] = KEf[ef * 576 + t + 288];
      __syncthreads();
      // Tm[(a,i),(B,j)] = sum_b K[(a,i),(b,j)] P[b][B]
      for (int h2 = 0; h2 < 2; h2++) {
        const int ent = t + 288 * h2;
        const int row = ent / 24, col = ent % 24, B = col / 3, j = col % 3;
        double s = 0;
#pragma unroll
        for (int b = 0; b < 8; b++) {
          const double wb = pw(2, px + (b & 1), B & 1) * pw(2, py + ((b >> 1) & 1), (B >> 1) & 1) *
                            pw(2, pz + (b >> 2), B >> 2);
          s += K[row * 24 + b * 3 + j] * wb;
        }
        Tm[ent] = s;
      }
      __syncthreads();
      for (int h2 = 0; h2 < 2; h2++) {
        const int ent = t + 288 * h2;
        const int row = ent / 24, col = ent % 24, A = row / 3, i = row % 3;
        double s = 0;
#pragma unroll
        for (int a = 0; a < 8; a++) {
          const double wa = pw(2, px + (a & 1), A & 1) * pw(2, py + ((a >> 1) & 1), (A >> 1) & 1) *
                            pw(2, pz + (a >> 2), A >> 2);
          s += wa * Tm[(a * 3 + i) * 24 + col];
        }
        acc[h2] += s;
      }
    }
  }
  KEc[E * 576 + t] = acc[0];
  KEc[E * 576 + t + 288] = acc[1];
}

// stencil assembly from element matrices: one thread per (node, neighbour d),
// summing the 3x3 blocks of the incident elements that contain both nodes
__global__ void k_assemble(const Level C, const double* __restrict__ KE, double* __restrict__ st64,
                           float* __restrict__ st32) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= 27 * C.nn) return;
  const int d = t / C.nn;
  const long long nl = t % C.nn;
  const int x = nl % C.nx, y = (nl / C.nx) % C.ny, z = nl / ((long long)C.nx * C.ny);
  const int dx = d % 3 - 1, dy = d / 3 % 3 - 1, dz = d / 9 - 1;
  const long long NP = C.NP;
  const long long n = C.nidx(x, y, z);
  double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = 0; k < 8; k++) {
    const int kx = k & 1, ky = (k >> 1) & 1, kz = k >> 2;
    if (!((dx == kx - 1 || dx == kx) && (dy == ky - 1 || dy == ky) && (dz == kz - 1 || dz == kz))) continue;
    const int ex = x - 1 + kx, ey = y - 1 + ky, ez = z - 1 + kz;
    if (!C.emask[C.eidx(ex, ey, ez)]) continue;
    const long long E = ex + (long long)C.ex * (ey + (long long)C.ey * ez);
    const int a = 7 - k;
    const int b = (dx - kx + 1) + 2 * (dy - ky + 1) + 4 * (dz - kz + 1);
    const double* K = KE + E * 576;
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int c = 0; c < 3; c++) s[r * 3 + c] += K[(a * 3 + r) * 24 + b * 3 + c];
  }
#pragma unroll
  for (int i = 0; i < 9; i++) {
    st64[(d * 9 + i) * NP + n] = s[i];
    st32[st_at<float>(NP, d * 9 + i, n)] = (float)s[i];
  }
}

// ---------------------------------------------------------------- coarsest dense solve
__global__ void k_coarse_dense(const Level C, const double* __restrict__ st, const int* __restrict__ cnodes,
                               const int* __restrict__ crow, int nc, double* __restrict__ K) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long tot = (long long)nc * 243;
  if (t >= tot) return;
  const int i = t / 243, rem = t % 243, d = rem / 9, r = (rem % 9) / 3, c = rem % 3;
  const long long n = cnodes[i];
  const long long nb = n + (d % 3 - 1) + (d / 3 % 3 - 1) * (long long)C.px + (d / 9 - 1) * (long long)C.px * C.py;
  const int j = crow[nb];
  if (j < 0) return;
  const int N = 3 * nc;
  K[(long long)(3 * i + r) * N + 3 * j + c] = st[(long long)(d * 9 + r * 3 + c) * C.NP + n];
}

template <typename T>
__global__ void k_gather_coarse(const Level C, const T* __restrict__ f, const int* __restrict__ cnodes, int nc,
                                double* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nc) return;
  const long long n = cnodes[i];
  b[3 * i + 0] = (double)f[n];
  b[3 * i + 1] = (double)f[n + C.NP];
  b[3 * i + 2] = (double)f[n + 2 * C.NP];
}

// u = Kinv b, one warp per row; result scattered to the padded coarsest vector
template <typename T>
__global__ void k_gemv_scatter(const Level C, const double* __restrict__ Kinv, const double* __restrict__ b, int nc,
                               const int* __restrict__ cnodes, T* __restrict__ u) {
  const int N = 3 * nc;
  const int row = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (row >= N) return;
  double s = 0;
  for (int j = lane; j < N; j += 32) s += Kinv[(long long)row * N + j] * b[j];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) u[cnodes[row / 3] + (row % 3) * C.NP] = (T)s;
}

// ---------------------------------------------------------------- bottom of the V-cycle
// The small levels and the coarsest solve as one kernel on an 8-CTA
// thread-block cluster: every phase (Jacobi / Chebyshev sweeps, residual,
// restriction, dense coarsest solve, prolongation) is separated by a cluster
// barrier instead of a launch.  Results are left in the levels' u vectors
// exactly as the per-level launches leave them.  Measured on cubes from 32^3
// to 256^3 the phases wait on load latency with 8 SMs working, and the
// per-level launches over the whole GPU are faster (the 17^3 to 5^3 levels of
// a 256^3 hierarchy: 3 % of a solve), so it runs only when rso_autotune finds
// it faster on the handle's own problem.
constexpr int BOT_CTAS = 8, BOT_THREADS = 1024, BOT_MAX_LEVELS = 12;

constexpr int BOT_MAX_SWEEPS = 8;
template <typename T>
struct BottomArgs {
  Level L[BOT_MAX_LEVELS];
  T om[BOT_MAX_LEVELS][BOT_MAX_SWEEPS];  // smoother step coefficients per level and step
  T c1[BOT_MAX_LEVELS][BOT_MAX_SWEEPS];
  int lb, nl, pre, post;
  const double* kinv;  // coarsest inverse, N x N, N = 3 nc
  const int* cnodes;
  int nc;
  double* cf;          // coarsest right-hand side (N doubles)
};

template <typename T>
__device__ __forceinline__ T* bv_u(const Level& L) { if constexpr (sizeof(T) == 4) return (T*)L.u32; else return (T*)L.u64; }
template <typename T>
__device__ __forceinline__ T* bv_f(const Level& L) { if constexpr (sizeof(T) == 4) return (T*)L.f32; else return (T*)L.f64; }
template <typename T>
__device__ __forceinline__ T* bv_r(const Level& L) { if constexpr (sizeof(T) == 4) return (T*)L.r32; else return (T*)L.r64; }
template <typename T>
__device__ __forceinline__ T* bv_t(const Level& L) { if constexpr (sizeof(T) == 4) return (T*)L.t32; else return (T*)L.t64; }
template <typename T>
__device__ __forceinline__ const T* bv_st(const Level& L) {
  if constexpr (sizeof(T) == 4) return (const T*)L.st32; else return (const T*)L.st64;
}

__device__ __forceinline__ long long bot_node(const Level& L, long long i) {
  const int x = (int)(i % L.nx), y = (int)((i / L.nx) % L.ny), z = (int)(i / ((long long)L.nx * L.ny));
  return L.nidx(x, y, z);
}

// out = u + c1 (u - up) + om D^-1 (f - K u), u read as 0 when zero and up as
// 0 when NULL; inactive nodes 0
template <typename T>
__device__ void bot_jacobi(const Level& L, const T* st, const T* u0v, const T* f0v, T* out0v, T om, bool zero,
                           const T* up0v, T c1, int g0, int gs) {
  const long long NP = L.NP;
  for (long long ib = g0; ib < L.nn * L.nb; ib += gs) {
    const long long b = ib / L.nn, i = ib - b * L.nn, vo = b * 3 * NP;
    const T* u = u0v + vo;
    const T* f = f0v + vo;
    T* out = out0v + vo;
    const T* up = up0v ? up0v + vo : nullptr;
    const long long n = bot_node(L, i);
    if (!(L.vclass[n] & NC_ACTIVE)) { out[n] = 0; out[n + NP] = 0; out[n + 2 * NP] = 0; continue; }
    T acc[3] = {0, 0, 0};
    if (!zero) stencil_apply<T>(L, st, u, n, false, acc);
    T S[9];
#pragma unroll
    for (int k = 0; k < 9; k++) S[k] = st[st_at<T>(NP, 13 * 9 + k, n)];
    const T r0 = f[n] - acc[0], r1 = f[n + NP] - acc[1], r2 = f[n + 2 * NP] - acc[2];
    const T A = S[4] * S[8] - S[5] * S[7], B = -(S[3] * S[8] - S[5] * S[6]), C = S[3] * S[7] - S[4] * S[6];
    const T det = S[0] * A + S[1] * B + S[2] * C;
    const T id = om / det;
    const T i01 = -(S[1] * S[8] - S[2] * S[7]), i02 = S[1] * S[5] - S[2] * S[4];
    const T i11 = S[0] * S[8] - S[2] * S[6], i12 = -(S[0] * S[5] - S[2] * S[3]);
    const T i21 = -(S[0] * S[7] - S[1] * S[6]), i22 = S[0] * S[4] - S[1] * S[3];
    const T u0 = zero ? T(0) : u[n], u1 = zero ? T(0) : u[n + NP], u2 = zero ? T(0) : u[n + 2 * NP];
    const T p0 = up ? up[n] : T(0), p1 = up ? up[n + NP] : T(0), p2 = up ? up[n + 2 * NP] : T(0);
    out[n] = u0 + c1 * (u0 - p0) + id * (A * r0 + i01 * r1 + i02 * r2);
    out[n + NP] = u1 + c1 * (u1 - p1) + id * (B * r0 + i11 * r1 + i12 * r2);
    out[n + 2 * NP] = u2 + c1 * (u2 - p2) + id * (C * r0 + i21 * r1 + i22 * r2);
  }
}

template <typename T>
__device__ void bot_residual(const Level& L, const T* st, const T* u0v, const T* f0v, T* r0v, int g0, int gs) {
  const long long NP = L.NP;
  for (long long ib = g0; ib < L.nn * L.nb; ib += gs) {
    const long long b = ib / L.nn, i = ib - b * L.nn, vo = b * 3 * NP;
    const T* u = u0v + vo;
    const T* f = f0v + vo;
    T* r = r0v + vo;
    const long long n = bot_node(L, i);
    T acc[3] = {0, 0, 0};
    if (L.vclass[n] & NC_ACTIVE) stencil_apply<T>(L, st, u, n, false, acc);
    r[n] = f[n] - acc[0]; r[n + NP] = f[n + NP] - acc[1]; r[n + 2 * NP] = f[n + 2 * NP] - acc[2];
  }
}

// FC: the coarsening factor when known at compile time (its loops unrolled,
// so a thread's loads are all in flight at once), 0 to read it from C
template <typename T, int FC = 0>
__device__ void bot_restrict(const Level& Fl, const Level& C, const T* rf0, T* fc0, int g0, int gs) {
  const int F = FC > 0 ? FC : C.factor;
  for (long long ib = g0; ib < C.nn * C.nb; ib += gs) {
    const long long b = ib / C.nn, i = ib - b * C.nn;
    const T* rf = rf0 + b * 3 * Fl.NP;
    T* fc = fc0 + b * 3 * C.NP;
    const int X = (int)(i % C.nx), Y = (int)((i / C.nx) % C.ny), Z = (int)(i / ((long long)C.nx * C.ny));
    const long long nC = C.nidx(X, Y, Z);
    T s0 = 0, s1 = 0, s2 = 0;
    if (C.vclass[nC] & NC_ACTIVE) {
#pragma unroll
      for (int dz = -F + 1; dz < F; dz++) {
        const int z = F * Z + dz;
        if (z < 0 || z >= Fl.nz) continue;
#pragma unroll
        for (int dy = -F + 1; dy < F; dy++) {
          const int y = F * Y + dy;
          if (y < 0 || y >= Fl.ny) continue;
          const T wyz = (T)(F - abs(dy)) / (T)F * ((T)(F - abs(dz)) / (T)F);
#pragma unroll
          for (int dx = -F + 1; dx < F; dx++) {
            const int x = F * X + dx;
            if (x < 0 || x >= Fl.nx) continue;
            const long long n = Fl.nidx(x, y, z);
            const T w = wyz * ((T)(F - abs(dx)) / (T)F);
            s0 += w * rf[n]; s1 += w * rf[n + Fl.NP]; s2 += w * rf[n + 2 * Fl.NP];
          }
        }
      }
    }
    fc[nC] = s0; fc[nC + C.NP] = s1; fc[nC + 2 * C.NP] = s2;
  }
}

// the restriction with one thread per (coarse node, component) and the
// factor known at compile time: a thread's (2F - 1)^3 loads are independent
// and unrolled (the same sums in the same order as bot_restrict)
template <typename T, int F>
__device__ void bot_restrict3(const Level& Fl, const Level& C, const T* rf0, T* fc0, int g0, int gs) {
  // the levels of the persistent kernel are below 2^31 nodes (checked by its
  // launcher): 32-bit index arithmetic
  const unsigned nn = (unsigned)C.nn, nx = (unsigned)C.nx, ny = (unsigned)C.ny;
  for (unsigned it = g0; it < 3u * nn * (unsigned)C.nb; it += gs) {
    const unsigned ib = it / 3u, c = it - 3u * ib;
    const unsigned b = ib / nn, i = ib - b * nn;
    const T* rf = rf0 + (long long)b * 3 * Fl.NP + c * Fl.NP;
    T* fc = fc0 + (long long)b * 3 * C.NP + c * C.NP;
    const unsigned iy = i / nx, Z = iy / ny;
    const int X = (int)(i - iy * nx), Y = (int)(iy - Z * ny);
    const long long nC = C.nidx(X, Y, Z);
    T sum = 0;
    if (C.vclass[nC] & NC_ACTIVE) {
#pragma unroll
      for (int dz = -F + 1; dz < F; dz++) {
        const int z = F * Z + dz;
        if (z < 0 || z >= Fl.nz) continue;
#pragma unroll
        for (int dy = -F + 1; dy < F; dy++) {
          const int y = F * Y + dy;
          if (y < 0 || y >= Fl.ny) continue;
          const T wyz = (T)(F - abs(dy)) / (T)F * ((T)(F - abs(dz)) / (T)F);
#pragma unroll
          for (int dx = -F + 1; dx < F; dx++) {
            const int x = F * X + dx;
            if (x < 0 || x >= Fl.nx) continue;
            const T w = wyz * ((T)(F - abs(dx)) / (T)F);
            sum += w * rf[Fl.nidx(x, y, z)];
          }
        }
      }
    }
    fc[nC] = sum;
  }
}

template <typename T>
__device__ void bot_prolong(const Level& Fl, const Level& C, const T* uc0, T* uf0, int g0, int gs) {
  const int F = C.factor;
  for (long long ib = g0; ib < Fl.nn * Fl.nb; ib += gs) {
    const long long b = ib / Fl.nn, i = ib - b * Fl.nn;
    const T* uc = uc0 + b * 3 * C.NP;
    T* uf = uf0 + b * 3 * Fl.NP;
    const int x = (int)(i % Fl.nx), y = (int)((i / Fl.nx) % Fl.ny), z = (int)(i / ((long long)Fl.nx * Fl.ny));
    const long long n = Fl.nidx(x, y, z);
    const uint8_t cls = Fl.vclass[n];
    if (!(cls & NC_ACTIVE) || (cls & NC_SUPPORT)) continue;
    const int X0 = x / F, Y0 = y / F, Z0 = z / F;
    const int ox = x - F * X0, oy = y - F * Y0, oz = z - F * Z0;
    T s0 = 0, s1 = 0, s2 = 0;
    for (int A = 0; A < 8; A++) {
      const int ax = A & 1, ay = (A >> 1) & 1, az = A >> 2;
      const T w = (ax ? (T)ox : (T)(F - ox)) / (T)F * ((ay ? (T)oy : (T)(F - oy)) / (T)F) *
                  ((az ? (T)oz : (T)(F - oz)) / (T)F);
      const long long nC = C.nidx(X0 + ax, Y0 + ay, Z0 + az);
      s0 += w * uc[nC]; s1 += w * uc[nC + C.NP]; s2 += w * uc[nC + 2 * C.NP];
    }
    uf[n] += s0; uf[n + Fl.NP] += s1; uf[n + 2 * Fl.NP] += s2;
  }
}

// the prolongation with one thread per (fine node, component): the same
// sums in the same order as bot_prolong, a third of the loads per thread
template <typename T>
__device__ void bot_prolong3(const Level& Fl, const Level& C, const T* uc0, T* uf0, int g0, int gs) {
  const int F = C.factor;
  // 32-bit index arithmetic, as in bot_restrict3
  const unsigned nn = (unsigned)Fl.nn, nx = (unsigned)Fl.nx, ny = (unsigned)Fl.ny;
  for (unsigned it = g0; it < 3u * nn * (unsigned)Fl.nb; it += gs) {
    const unsigned ib = it / 3u, c = it - 3u * ib;
    const unsigned b = ib / nn, i = ib - b * nn;
    const T* uc = uc0 + (long long)b * 3 * C.NP + c * C.NP;
    T* uf = uf0 + (long long)b * 3 * Fl.NP + c * Fl.NP;
    const unsigned iy = i / nx, zz = iy / ny;
    const int x = (int)(i - iy * nx), y = (int)(iy - zz * ny), z = (int)zz;
    const long long n = Fl.nidx(x, y, z);
    const uint8_t cls = Fl.vclass[n];
    if (!(cls & NC_ACTIVE) || (cls & NC_SUPPORT)) continue;
    const int X0 = x / F, Y0 = y / F, Z0 = z / F;
    const int ox = x - F * X0, oy = y - F * Y0, oz = z - F * Z0;
    T sum = 0;
#pragma unroll
    for (int A = 0; A < 8; A++) {
      const int ax = A & 1, ay = (A >> 1) & 1, az = A >> 2;
      const T w = (ax ? (T)ox : (T)(F - ox)) / (T)F * ((ay ? (T)oy : (T)(F - oy)) / (T)F) *
                  ((az ? (T)oz : (T)(F - oz)) / (T)F);
      sum += w * uc[C.nidx(X0 + ax, Y0 + ay, Z0 + az)];
    }
    uf[n] += sum;
  }
}

template <typename T>
__device__ void bot_copy(const Level& L, const T* a, T* b, int g0, int gs) {
  for (long long i = g0; i < 3 * L.NP * L.nb; i += gs) b[i] = a[i];
}

template <typename T>
__global__ void __cluster_dims__(BOT_CTAS, 1, 1) __launch_bounds__(BOT_THREADS, 1)
    k_bottom(const __grid_constant__ BottomArgs<T> A) {
  cg::cluster_group cl = cg::this_cluster();
  const int g0 = (int)cl.block_rank() * BOT_THREADS + threadIdx.x, gs = BOT_CTAS * BOT_THREADS;
  // the smoothers rotate each level's u, t and r; ucur[li] is the one that
  // holds the level's iterate between the down- and the up-sweep
  T* ucur[BOT_MAX_LEVELS];
  // down: pre-smoothing from a zero iterate, residual, restriction
  for (int li = A.lb; li < A.nl - 1; li++) {
    const Level& L = A.L[li];
    const T* st = bv_st<T>(L);
    T* u = bv_u<T>(L);
    T *cur = u, *oth = bv_t<T>(L), *prv = bv_r<T>(L);
    for (int s = 0; s < A.pre; s++) {
      bot_jacobi<T>(L, st, cur, bv_f<T>(L), oth, A.om[li][s], s == 0, s <= 1 ? (const T*)nullptr : prv, A.c1[li][s],
                    g0, gs);
      cl.sync();
      T* w = prv; prv = cur; cur = oth; oth = w;
    }
    if (A.pre == 0) {
      for (long long i = g0; i < 3 * L.NP * L.nb; i += gs) u[i] = T(0);
      cl.sync();
    }
    ucur[li] = cur;
    // the residual goes to a vector the iterate is not in
    bot_residual<T>(L, st, cur, bv_f<T>(L), oth, g0, gs);
    cl.sync();
    bot_restrict<T>(L, A.L[li + 1], oth, bv_f<T>(A.L[li + 1]), g0, gs);
    cl.sync();
  }
  // coarsest: u = Kinv f at the listed nodes, zero elsewhere; one warp per row
  {
    const Level& C = A.L[A.nl - 1];
    T* u = bv_u<T>(C);
    const T* f = bv_f<T>(C);
    const long long VS = 3 * C.NP;
    const int N = 3 * A.nc;
    for (long long i = g0; i < VS * C.nb; i += gs) u[i] = T(0);
    for (long long ib = g0; ib < (long long)A.nc * C.nb; ib += gs) {
      const long long b = ib / A.nc, i = ib - b * A.nc;
      const long long n = A.cnodes[i] + b * VS;
      double* cf = A.cf + b * N;
      cf[3 * i + 0] = (double)f[n];
      cf[3 * i + 1] = (double)f[n + C.NP];
      cf[3 * i + 2] = (double)f[n + 2 * C.NP];
    }
    cl.sync();
    const int lane = threadIdx.x & 31, warp = g0 >> 5, nwarps = gs >> 5;
    for (long long rb = warp; rb < (long long)N * C.nb; rb += nwarps) {
      const long long b = rb / N;
      const int row = (int)(rb - b * N);
      const double* cf = A.cf + b * N;
      const double* k = A.kinv + (long long)row * N;
      double s = 0;
      for (int j = lane; j < N; j += 32) s += k[j] * cf[j];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      if (lane == 0) u[b * VS + A.cnodes[row / 3] + (row % 3) * C.NP] = (T)s;
    }
    ucur[A.nl - 1] = u;
    cl.sync();
  }
  // up: prolongation and post-smoothing; the top level ends in its u
  for (int li = A.nl - 2; li >= A.lb; li--) {
    const Level& L = A.L[li];
    const T* st = bv_st<T>(L);
    T* u = bv_u<T>(L);
    T *cur = ucur[li], *oth, *prv;
    T* bufs[3] = {u, bv_t<T>(L), bv_r<T>(L)};
    {
      int k = 0;
      T* rest[2];
      for (int q = 0; q < 3; q++)
        if (bufs[q] != cur) rest[k++] = bufs[q];
      oth = rest[0];
      prv = rest[1];
    }
    bot_prolong<T>(L, A.L[li + 1], ucur[li + 1], cur, g0, gs);
    cl.sync();
    for (int s = 0; s < A.post; s++) {
      bot_jacobi<T>(L, st, cur, bv_f<T>(L), oth, A.om[li][s], false, s == 0 ? (const T*)nullptr : prv, A.c1[li][s],
                    g0, gs);
      cl.sync();
      T* w = prv; prv = cur; cur = oth; oth = w;
    }
    ucur[li] = cur;
    if (li == A.lb && cur != u) {
      bot_copy<T>(L, cur, u, g0, gs);
      cl.sync();
    }
  }
}

// The same bottom of the V-cycle as one persistent kernel over the whole GPU:
// a cooperative launch (every CTA resident at once) whose phases are
// separated by a grid-wide barrier.  The sweeps and residuals run as the
// row-split per-level kernel does (tiles of 32 x CTY nodes, three threads per
// node, the same arithmetic: bit-identical sweeps), the transfers and the
// coarsest solve as in k_bottom.
// a barrier wait gives up after this many SM clock cycles (about 2 s)
constexpr long long kGbarCycles = 4000000000LL;

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// grid-wide barrier on bar = {arrivals, generation, gave-up flag}: one arrival
// per CTA; the last resets the count and advances the generation.  gen (thread
// 0's copy of the generation) moves on with it.  Returns false on every
// thread of every CTA once some wait has given up (bar[2] set): the kernel
// then returns, and the host reports it after the solve.
// (target, limit: the arrivals that complete the barrier and the wait's bound
// in clock cycles; the self-test sets them, the bottom kernel keeps the grid
// size and kGbarCycles)
__device__ bool gbar_sync(unsigned* bar, unsigned& gen, int tid, unsigned target = 0, long long limit = kGbarCycles) {
  __shared__ int s_ok;
  if (target == 0) target = gridDim.x;
  __syncthreads();
  if (tid == 0) {
    int ok = *reinterpret_cast<volatile unsigned*>(bar + 2) == 0u;
    if (ok) {
      const unsigned g = gen;
      __threadfence();
      if (atomicAdd(bar, 1u) == target - 1) {
        atomicExch(bar, 0u);
        __threadfence();
        atomicExch(bar + 1, g + 1);
      } else {
        const long long t0 = clock64();
        while (ld_acquire_gpu(bar + 1) == g) {
          if (*reinterpret_cast<volatile unsigned*>(bar + 2) != 0u) { ok = 0; break; }
          if (clock64() - t0 > limit) {
            atomicExch(bar + 2, 1u);
            ok = 0;
            break;
          }
          __nanosleep(64);
        }
      }
      __threadfence();
      gen = g + 1;
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// one row-split sweep (MODE 2) or residual (MODE 0) of a level, tile by tile
template <typename T, int MODE, bool ZERO>
__device__ void gb_sweep_rows(const Level& L, const T* st, const T* u, const T* f, T* out, T omega, const T* uprev,
                              T c1, T (*sres)[CTY][32]) {
  const int tx = (L.nx + 31) / 32, ty = (L.ny + CTY - 1) / CTY;
  const long long nt = (long long)tx * ty * L.nz * L.nb;
  for (long long t = blockIdx.x; t < nt; t += gridDim.x) {
    const int bx = (int)(t % tx);
    const long long q = t / tx;
    const int by = (int)(q % ty);
    const long long zb = q / ty;
    const int bsys = (int)(zb / L.nz), z = (int)(zb - (long long)bsys * L.nz);
    coarse_r_node<T, MODE, ZERO>(L, st, u, f, out, omega, uprev, c1, bx * 32 + threadIdx.x, by * CTY + threadIdx.y,
                                 z, bsys, sres);
    __syncthreads();  // sres is reused by the next tile
  }
}

// FP32: the sweeps of the persistent kernel on groups of four consecutive
// padded nodes, nine threads per group, one per neighbour row (plane dz, row
// dy): a thread loads its row's u (a 16-byte vector and two scalars per
// component) and the 27 stencil vectors of its three neighbours, 36 loads
// where a row-split thread makes 162, so a small level's sweep is a few load
// latencies long.  The nine partial sums meet in shared memory in a fixed
// order; four of the group's threads then finish one node each as k_coarse4
// does (residual, or damped block Jacobi / Chebyshev step; halo rows
// unwritten).
constexpr int G9 = 32;  // node groups per tile (9 G9 threads)
template <int MODE, bool ZERO>
__device__ void gb_sweep4(const Level& L, const float* __restrict__ st, const float* u0v, const float* f0v,
                          float* out0v, float omega, const float* up0v, float c1, float (*red)[12][G9]) {
  const int tg = threadIdx.x % G9, q = threadIdx.x / G9;  // q = 3 (dz + 1) + (dy + 1)
  const int pz = q / 3, py = q - 3 * pz;
  const long long NP = L.NP, px = L.px, pxy = (long long)L.px * L.py;
  const long long ng = NP / 4, ngt = ng * L.nb;
  const long long ntile = (ngt + G9 - 1) / G9;
  for (long long t = blockIdx.x; t < ntile; t += gridDim.x) {
    const long long gg = t * G9 + tg;
    const long long bsys = gg < ngt ? (long long)((unsigned)gg / (unsigned)ng) : 0, g = gg - bsys * ng;
    const long long vo = bsys * 3 * NP;
    const float* u = u0v + vo;
    const long long p0 = 4 * g;
    bool work = gg < ngt;
    int xp = 0;
    bool act[4] = {false, false, false, false};
    if (work) {
      // the levels of this kernel are small (NP < 2^31): 32-bit divisions
      const unsigned p0u = (unsigned)p0, pxyu = (unsigned)pxy, pxu = (unsigned)px;
      const int zp = (int)(p0u / pxyu);
      const unsigned rem = p0u - (unsigned)zp * pxyu;
      const int yp = (int)(rem / pxu);
      xp = (int)(rem - (unsigned)yp * pxu);
      work = !(zp < 1 || zp > L.nz || yp < 1 || yp > L.ny);  // halo row: stays zero
    }
    bool any = false;
    if (work) {
      const uchar4 cl4 = *reinterpret_cast<const uchar4*>(L.vclass + p0);
      const uint8_t cls[4] = {cl4.x, cl4.y, cl4.z, cl4.w};
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int x = xp + k - 1;
        act[k] = x >= 0 && x < L.nx && (cls[k] & NC_ACTIVE);
        any = any || act[k];
      }
    }
    float acc[3][4];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int k = 0; k < 4; k++) acc[r][k] = 0.f;
    if (any && !ZERO) {
      const long long nb = p0 + (long long)(pz - 1) * pxy + (long long)(py - 1) * px;
      float w[3][6];  // u at x offsets -1 .. 4 of the group's row in this neighbour row
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const float* uc = u + nb + c * NP;
        const float4 m = *reinterpret_cast<const float4*>(uc);
        // at xp = 0 the left neighbour is outside the row (the group's first
        // node is halo, its result discarded); likewise the right one at the end
        w[c][0] = xp > 0 ? uc[-1] : 0.f;
        w[c][1] = m.x; w[c][2] = m.y; w[c][3] = m.z; w[c][4] = m.w;
        w[c][5] = xp + 4 < px ? uc[4] : 0.f;
      }
#pragma unroll
      for (int dx = 0; dx < 3; dx++) {
        const int d = q * 3 + dx;
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
          for (int c = 0; c < 3; c++) {
            const float4 sv = *reinterpret_cast<const float4*>(st + st_at<float>(NP, d * 9 + r * 3 + c, p0));
            acc[r][0] = fmaf(sv.x, w[c][dx + 0], acc[r][0]);
            acc[r][1] = fmaf(sv.y, w[c][dx + 1], acc[r][1]);
            acc[r][2] = fmaf(sv.z, w[c][dx + 2], acc[r][2]);
            acc[r][3] = fmaf(sv.w, w[c][dx + 3], acc[r][3]);
          }
      }
    }
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int k = 0; k < 4; k++) red[q][r * 4 + k][tg] = acc[r][k];
    __syncthreads();
    if (q < 4 && work) {
      // thread q finishes node k = q of the group: its rows' nine partial
      // sums in the order dz, dy = (-1, -1) .. (1, 1)
      const int k = q;
      const long long n = p0 + k;
      float a[3];
#pragma unroll
      for (int r = 0; r < 3; r++) {
        float sum = red[0][r * 4 + k][tg];
#pragma unroll
        for (int sl = 1; sl < 9; sl++) sum += red[sl][r * 4 + k][tg];
        a[r] = sum;
      }
      const float* f = f0v + vo;
      float* out = out0v + vo;
      float res[3];
#pragma unroll
      for (int r = 0; r < 3; r++) res[r] = f[n + r * NP] - (act[k] ? a[r] : 0.f);
      if (MODE == 0) {
#pragma unroll
        for (int r = 0; r < 3; r++) out[n + r * NP] = res[r];
      } else if (!act[k]) {
#pragma unroll
        for (int r = 0; r < 3; r++) out[n + r * NP] = 0.f;
      } else {
        float Sk[9];
#pragma unroll
        for (int i = 0; i < 9; i++) Sk[i] = st[st_at<float>(NP, 13 * 9 + i, n)];
        float uo[3], up[3];
#pragma unroll
        for (int r = 0; r < 3; r++) {
          uo[r] = ZERO ? 0.f : u[n + r * NP];
          up[r] = up0v ? up0v[vo + n + r * NP] : 0.f;
        }
        const float r0 = res[0], r1 = res[1], r2 = res[2];
        const float A = Sk[4] * Sk[8] - Sk[5] * Sk[7], B = -(Sk[3] * Sk[8] - Sk[5] * Sk[6]),
                    C = Sk[3] * Sk[7] - Sk[4] * Sk[6];
        const float det = Sk[0] * A + Sk[1] * B + Sk[2] * C;
        const float id = omega / det;
        const float i01 = -(Sk[1] * Sk[8] - Sk[2] * Sk[7]), i02 = Sk[1] * Sk[5] - Sk[2] * Sk[4];
        const float i11 = Sk[0] * Sk[8] - Sk[2] * Sk[6], i12 = -(Sk[0] * Sk[5] - Sk[2] * Sk[3]);
        const float i21 = -(Sk[0] * Sk[7] - Sk[1] * Sk[6]), i22 = Sk[0] * Sk[4] - Sk[1] * Sk[3];
        out[n] = uo[0] + c1 * (uo[0] - up[0]) + id * (A * r0 + i01 * r1 + i02 * r2);
        out[n + NP] = uo[1] + c1 * (uo[1] - up[1]) + id * (B * r0 + i11 * r1 + i12 * r2);
        out[n + 2 * NP] = uo[2] + c1 * (uo[2] - up[2]) + id * (C * r0 + i21 * r1 + i22 * r2);
      }
    }
    __syncthreads();  // red is reused by the next tile
  }
}

// threads of a CTA of the persistent kernel: nine per group of G9 four-node
// groups (FP32), 32 x CTY x 3 for the row-split sweeps (FP64)
template <typename T>
constexpr int gb_threads() { return sizeof(T) == 4 ? 9 * G9 : 32 * CTY * 3; }
// shared exchange of a sweep: [9][12][G9] floats (FP32), [3][CTY][32] T (FP64)
template <typename T>
constexpr int gb_smem() { return sizeof(T) == 4 ? 9 * 12 * G9 * 4 : 3 * CTY * 32 * (int)sizeof(T); }

template <typename T, int MODE, bool ZERO>
__device__ __forceinline__ void gb_sweep(const Level& L, const T* st, const T* u, const T* f, T* out, T omega,
                                         const T* uprev, T c1, unsigned char* sm) {
  if constexpr (sizeof(T) == 4)
    gb_sweep4<MODE, ZERO>(L, st, u, f, out, omega, uprev, c1, reinterpret_cast<float (*)[12][G9]>(sm));
  else
    gb_sweep_rows<T, MODE, ZERO>(L, st, u, f, out, omega, uprev, c1, reinterpret_cast<T (*)[CTY][32]>(sm));
}

template <typename T>
__global__ void __launch_bounds__(gb_threads<T>(), sizeof(T) == 4 ? 2 : 1) k_bottom_grid(const __grid_constant__ BottomArgs<T> A,
                                                                 unsigned* bar) {
  __shared__ __align__(16) unsigned char sres[gb_smem<T>()];
  constexpr int NT = gb_threads<T>();
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int g0 = blockIdx.x * NT + tid, gs = gridDim.x * NT;
  unsigned gen = 0;
  if (tid == 0) gen = ld_acquire_gpu(bar + 1);
#define GB_SYNC() \
  if (!gbar_sync(bar, gen, tid)) return
  T* ucur[BOT_MAX_LEVELS];
  // down: pre-smoothing from a zero iterate, residual, restriction
  for (int li = A.lb; li < A.nl - 1; li++) {
    const Level& L = A.L[li];
    const T* st = bv_st<T>(L);
    T* u = bv_u<T>(L);
    T *cur = u, *oth = bv_t<T>(L), *prv = bv_r<T>(L);
    for (int s = 0; s < A.pre; s++) {
      if (s == 0)
        gb_sweep<T, 2, true>(L, st, cur, bv_f<T>(L), oth, A.om[li][s], (const T*)nullptr, A.c1[li][s], sres);
      else
        gb_sweep<T, 2, false>(L, st, cur, bv_f<T>(L), oth, A.om[li][s], s <= 1 ? (const T*)nullptr : prv,
                              A.c1[li][s], sres);
      GB_SYNC();
      T* w = prv; prv = cur; cur = oth; oth = w;
    }
    if (A.pre == 0) {
      for (long long i = g0; i < 3 * L.NP * L.nb; i += gs) u[i] = T(0);
      GB_SYNC();
    }
    ucur[li] = cur;
    gb_sweep<T, 0, false>(L, st, cur, bv_f<T>(L), oth, T(0), (const T*)nullptr, T(0), sres);
    GB_SYNC();
    if (A.L[li + 1].factor == 2)
      bot_restrict3<T, 2>(L, A.L[li + 1], oth, bv_f<T>(A.L[li + 1]), g0, gs);
    else
      bot_restrict<T>(L, A.L[li + 1], oth, bv_f<T>(A.L[li + 1]), g0, gs);
    if (li + 1 == A.nl - 1) {  // the coarsest iterate is zero outside the listed nodes
      const Level& C = A.L[li + 1];
      T* uc = bv_u<T>(C);
      for (long long i = g0; i < 3 * C.NP * C.nb; i += gs) uc[i] = T(0);
    }
    GB_SYNC();
  }
  // coarsest: u = Kinv f at the listed nodes (zeroed elsewhere above); one
  // warp per row, f read through the node list
  {
    const Level& C = A.L[A.nl - 1];
    T* u = bv_u<T>(C);
    const T* f = bv_f<T>(C);
    const long long VS = 3 * C.NP;
    const int N = 3 * A.nc;
    const int lane = tid & 31, warp = g0 >> 5, nwarps = gs >> 5;
    for (long long rb = warp; rb < (long long)N * C.nb; rb += nwarps) {
      const long long b = rb / N;
      const int row = (int)(rb - b * N);
      const T* fb = f + b * VS;
      const double* k = A.kinv + (long long)row * N;
      double sum = 0;
#pragma unroll 4
      for (int j = lane; j < N; j += 32) sum += k[j] * (double)fb[A.cnodes[j / 3] + (j % 3) * C.NP];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
      if (lane == 0) u[b * VS + A.cnodes[row / 3] + (row % 3) * C.NP] = (T)sum;
    }
    ucur[A.nl - 1] = u;
    GB_SYNC();
  }
  // up: prolongation and post-smoothing; the top level ends in its u
  for (int li = A.nl - 2; li >= A.lb; li--) {
    const Level& L = A.L[li];
    const T* st = bv_st<T>(L);
    T* u = bv_u<T>(L);
    T *cur = ucur[li], *oth, *prv;
    T* bufs[3] = {u, bv_t<T>(L), bv_r<T>(L)};
    {
      int k = 0;
      T* rest[2];
      for (int q = 0; q < 3; q++)
        if (bufs[q] != cur) rest[k++] = bufs[q];
      oth = rest[0];
      prv = rest[1];
    }
    bot_prolong3<T>(L, A.L[li + 1], ucur[li + 1], cur, g0, gs);
    GB_SYNC();
    for (int s = 0; s < A.post; s++) {
      gb_sweep<T, 2, false>(L, st, cur, bv_f<T>(L), oth, A.om[li][s], s == 0 ? (const T*)nullptr : prv,
                            A.c1[li][s], sres);
      GB_SYNC();
      T* w = prv; prv = cur; cur = oth; oth = w;
    }
    ucur[li] = cur;
    if (li == A.lb && cur != u) {
      bot_copy<T>(L, cur, u, g0, gs);
      GB_SYNC();
    }
  }
#undef GB_SYNC
}

// ---------------------------------------------------------------- host wrappers
// grids over the nodes of a level for every system it carries
static inline dim3 node_grid(const Level& l) { return dim3(cdiv(l.nx, 32), cdiv(l.ny, 8), l.nz * l.nb); }
static inline dim3 chunk_grid(const Level& l, int kb) { return dim3(cdiv(l.nx, 32), cdiv(l.ny, 8), l.nz * cdiv(l.nb, kb)); }
// levels above this many nodes use the per-node stencil kernel
static const long long kRowSplitMaxNodes = 100000;

template <typename T>
static const T* stencil_of(const Level& l);
template <>
const double* stencil_of<double>(const Level& l) { return l.st64; }
template <>
const float* stencil_of<float>(const Level& l) { return l.st32; }

// kernel variant of a coarse level: 0 one thread per node (large levels), 1
// one per (node, row) (the rest), 2 nine per node (k_coarse_r9: only when
// rso_autotune finds it faster; on cubes from 32^3 to 256^3 it measured
// slower than 1 on every level), unless rso_autotune measured the level
static int coarse_variant(const rso_handle* h, int level) {
  const int t = level < 16 ? h->tune.rowsplit[level] : -1;
  if (t >= 0 && t <= 2) return t;
  return h->L[level].nn > kRowSplitMaxNodes ? 0 : 1;
}
static bool node_per_thread(const rso_handle* h, int level) { return coarse_variant(h, level) == 0; }
int coarse_variant_of(const rso_handle* h, int level) { return coarse_variant(h, level); }

// profiling class of a coarse sweep: the streamed FP32 kernel has its own
static int coarse_class(const rso_handle* h, int level, int elem_size) {
  if (elem_size == 8) return PC_COARSE64;
  return node_per_thread(h, level) && h->L[level].nb == 1 ? PC_COARSE32_STREAM : PC_COARSE32;
}

template <typename T>
rso_status coarse_residual(rso_handle* h, int level, const T* u, const T* f, T* r) {
  const Level& l = h->L[level];
  const int cls = coarse_class(h, level, sizeof(T));
  if (h->prof_on) prof_begin(h, cls, (double)l.nn);
  if (node_per_thread(h, level)) {
    if (l.nb == 1 && sizeof(T) == 4 && l.NP < (1LL << 31)) {
      k_coarse4<0><<<cdiv(l.NP / 4, C4G), dim3(C4G, 3), 0, h->stream>>>(l, (const float*)stencil_of<T>(l), (const float*)u,
                                                               (const float*)f, (float*)r, 0.f, nullptr, 0.f);
    } else if (l.nb == 1) {
      k_coarse<T, 0, 1><<<chunk_grid(l, 1), dim3(32, 8), 0, h->stream>>>(l, stencil_of<T>(l), u, f, r, T(0), (const T*)nullptr, T(0));
    } else {
      k_coarse<T, 0, 4><<<chunk_grid(l, 4), dim3(32, 8), 0, h->stream>>>(l, stencil_of<T>(l), u, f, r, T(0), (const T*)nullptr, T(0));
    }
    rso::note_launch();
  } else if (coarse_variant(h, level) == 2) {
    k_coarse_r9<T, 0><<<dim3(cdiv(l.nx, 32), cdiv(l.ny, CTY9), l.nz * l.nb), dim3(32, CTY9, 9), 0, h->stream>>>(l, stencil_of<T>(l), u, f, r, T(0), (const T*)nullptr, T(0)); rso::note_launch();
  } else {
    k_coarse_r<T, 0><<<dim3(cdiv(l.nx, 32), cdiv(l.ny, CTY), l.nz * l.nb), dim3(32, CTY, 3), 0, h->stream>>>(l, stencil_of<T>(l), u, f, r, T(0), (const T*)nullptr, T(0)); rso::note_launch();
  }
  if (h->prof_on) prof_end(h, cls);
  return launch_check(h, "coarse_residual");
}
template <typename T>
rso_status coarse_jacobi(rso_handle* h, int level, const T* u_in, const T* f, T* u_out, double omega,
                         const T* u_prev, double c1) {
  const Level& l = h->L[level];
  const int cls = coarse_class(h, level, sizeof(T));
  if (h->prof_on) prof_begin(h, cls, (double)l.nn);
  if (node_per_thread(h, level)) {
    if (l.nb == 1 && sizeof(T) == 4 && l.NP < (1LL << 31)) {
      k_coarse4<2><<<cdiv(l.NP / 4, C4G), dim3(C4G, 3), 0, h->stream>>>(l, (const float*)stencil_of<T>(l), (const float*)u_in,
                                                               (const float*)f, (float*)u_out, (float)omega,
                                                               (const float*)u_prev, (float)c1);
    } else if (l.nb == 1) {
      k_coarse<T, 2, 1><<<chunk_grid(l, 1), dim3(32, 8), 0, h->stream>>>(l, stencil_of<T>(l), u_in, f, u_out, (T)omega, u_prev, (T)c1);
    } else {
      k_coarse<T, 2, 4><<<chunk_grid(l, 4), dim3(32, 8), 0, h->stream>>>(l, stencil_of<T>(l), u_in, f, u_out, (T)omega, u_prev, (T)c1);
    }
    rso::note_launch();
  } else if (coarse_variant(h, level) == 2) {
    k_coarse_r9<T, 2><<<dim3(cdiv(l.nx, 32), cdiv(l.ny, CTY9), l.nz * l.nb), dim3(32, CTY9, 9), 0, h->stream>>>(l, stencil_of<T>(l), u_in, f, u_out, (T)omega, u_prev, (T)c1); rso::note_launch();
  } else {
    k_coarse_r<T, 2><<<dim3(cdiv(l.nx, 32), cdiv(l.ny, CTY), l.nz * l.nb), dim3(32, CTY, 3), 0, h->stream>>>(l, stencil_of<T>(l), u_in, f, u_out, (T)omega, u_prev, (T)c1); rso::note_launch();
  }
  if (h->prof_on) prof_end(h, cls);
  return launch_check(h, "coarse_jacobi");
}
template <typename T>
rso_status coarse_gs(rso_handle* h, int level, T* u, const T* f, int colour, int reverse) {
  const Level& l = h->L[level];
  int cx = colour & 1, cy = (colour >> 1) & 1, cz = colour >> 2;
  dim3 g(cdiv((l.nx - cx + 1) / 2, 32), cdiv((l.ny - cy + 1) / 2, 8), (l.nz - cz + 1) / 2);
  if (g.x == 0 || g.y == 0 || g.z == 0) return RSO_OK;
  if (h->prof_on) prof_begin(h, (sizeof(T) == 4 ? PC_COARSE32 : PC_COARSE64), (double)l.nn / 8);
  k_coarse_gs<T><<<g, dim3(32, 8), 0, h->stream>>>(l, stencil_of<T>(l), u, f, cx, cy, cz, reverse); rso::note_launch();
  if (h->prof_on) prof_end(h, (sizeof(T) == 4 ? PC_COARSE32 : PC_COARSE64));
  return launch_check(h, "coarse_gs");
}
template <typename T>
rso_status restrict_(rso_handle* h, int cl, const T* rf, T* fc) {
  const Level& c = h->L[cl];
  const Level& f = h->L[cl - 1];
  if ((size_t)3 * f.nx * f.ny * c.nz * c.nb > h->xfer_n) {
    h->err = "restriction scratch smaller than the level pair needs";
    return RSO_ERR_STATE;
  }
  T* t = reinterpret_cast<T*>(h->xfer);
  const dim3 gz(cdiv(f.nx, 32), cdiv(f.ny, 8), c.nz * c.nb);
  // FP32, one system: the z pass on 16-byte vectors into padded planes (the
  // scratch holds 2 xfer_n floats, 3 px py nz_coarse of them here)
  if (sizeof(T) == 4 && c.nb == 1 && (c.factor == 4 || c.factor == 2) &&
      (size_t)3 * f.px * f.py * c.nz <= 2 * h->xfer_n) {
    const dim3 g4((unsigned)cdiv((long long)f.px * f.py / 4, 256), c.nz);
    float* t4 = reinterpret_cast<float*>(h->xfer);
    // the y-filtered planes after t when the scratch holds both
    const size_t tn = (size_t)3 * f.px * f.py * c.nz, tyn = (size_t)3 * c.nz * c.ny * f.px;
    float* ty = tn + tyn <= 2 * h->xfer_n ? t4 + tn : nullptr;
    const dim3 gy((unsigned)cdiv((long long)(f.px / 4) * c.ny, 256), c.nz);
    const dim3 gx(cdiv(c.nx, 32), cdiv(c.ny, 8), c.nz);
    if (c.factor == 4) {
      k_restrict_z_v4<4><<<g4, 256, 0, h->stream>>>(f, c.nz, (const float*)rf, t4); rso::note_launch();
      if (ty) {
        k_restrict_y_v4<4><<<gy, 256, 0, h->stream>>>(f, c, t4, ty); rso::note_launch();
        k_restrict_x<4><<<gx, dim3(32, 8), 0, h->stream>>>(f, c, ty, (float*)fc); rso::note_launch();
      } else {
        k_restrict_xy<float, 4, true><<<node_grid(c), dim3(32, 8), 0, h->stream>>>(f, c, t4, (float*)fc); rso::note_launch();
      }
    } else {
      k_restrict_z_v4<2><<<g4, 256, 0, h->stream>>>(f, c.nz, (const float*)rf, t4); rso::note_launch();
      if (ty) {
        k_restrict_y_v4<2><<<gy, 256, 0, h->stream>>>(f, c, t4, ty); rso::note_launch();
        k_restrict_x<2><<<gx, dim3(32, 8), 0, h->stream>>>(f, c, ty, (float*)fc); rso::note_launch();
      } else {
        k_restrict_xy<float, 2, true><<<node_grid(c), dim3(32, 8), 0, h->stream>>>(f, c, t4, (float*)fc); rso::note_launch();
      }
    }
    return launch_check(h, "restrict");
  }
  if (c.factor == 4) {
    k_restrict_z<T, 4><<<gz, dim3(32, 8), 0, h->stream>>>(f, c.nz, rf, t); rso::note_launch();
    k_restrict_xy<T, 4><<<node_grid(c), dim3(32, 8), 0, h->stream>>>(f, c, t, fc); rso::note_launch();
  } else if (c.factor == 2) {
    k_restrict_z<T, 2><<<gz, dim3(32, 8), 0, h->stream>>>(f, c.nz, rf, t); rso::note_launch();
    k_restrict_xy<T, 2><<<node_grid(c), dim3(32, 8), 0, h->stream>>>(f, c, t, fc); rso::note_launch();
  } else {
    h->err = "coarsening factor must be 2 or 4";
    return RSO_ERR_UNSUPPORTED;
  }
  return launch_check(h, "restrict");
}
template <typename T>
rso_status prolong(rso_handle* h, int cl, const T* uc, T* uf) {
  const Level& f = h->L[cl - 1];
  const Level& c = h->L[cl];
  const size_t row_smem = sizeof(float) * PROW_WARPS * 3 * (c.nx + 1);
  if (sizeof(T) == 4 && f.nb == 1 && (c.factor == 4 || c.factor == 2) && row_smem <= 48 * 1024) {
    const dim3 g((unsigned)cdiv(f.ny, PROW_WARPS), f.nz);
    if (c.factor == 4)
      k_prolong_row<4><<<g, dim3(32, PROW_WARPS), row_smem, h->stream>>>(f, c, (const float*)uc, (float*)uf);
    else
      k_prolong_row<2><<<g, dim3(32, PROW_WARPS), row_smem, h->stream>>>(f, c, (const float*)uc, (float*)uf);
    rso::note_launch();
  } else if (sizeof(T) == 4 && f.nb == 1 && (c.factor == 4 || c.factor == 2)) {
    const unsigned nblk = (unsigned)cdiv(f.NP / 4, 256);
    if (c.factor == 4)
      k_prolong_v4<4><<<nblk, 256, 0, h->stream>>>(f, c, (const float*)uc, (float*)uf);
    else
      k_prolong_v4<2><<<nblk, 256, 0, h->stream>>>(f, c, (const float*)uc, (float*)uf);
    rso::note_launch();
  } else if (c.factor == 4) {
    k_prolong<T, 4><<<node_grid(f), dim3(32, 8), 0, h->stream>>>(f, c, uc, uf); rso::note_launch();
  } else if (c.factor == 2) {
    k_prolong<T, 2><<<node_grid(f), dim3(32, 8), 0, h->stream>>>(f, c, uc, uf); rso::note_launch();
  } else {
    h->err = "coarsening factor must be 2 or 4";
    return RSO_ERR_UNSUPPORTED;
  }
  return launch_check(h, "prolong");
}
template <typename T>
rso_status coarsest_solve(rso_handle* h, const T* f, T* u) {
  const Level& c = h->L.back();
  if (h->nc == 0) return RSO_OK;
  const int N = 3 * h->nc;
  for (int b = 0; b < c.nb; b++) {  // one system after the other through the shared right-hand side buffer
    const long long vo = (long long)b * 3 * c.NP;
    k_gather_coarse<T><<<cdiv(h->nc, 128), 128, 0, h->stream>>>(c, f + vo, h->c_nodes, h->nc, h->c_f); rso::note_launch();
    k_gemv_scatter<T><<<cdiv(N, 8), 256, 0, h->stream>>>(c, h->c_K + (size_t)N * N, h->c_f, h->nc, h->c_nodes, u + vo);
    rso::note_launch();
  }
  return launch_check(h, "coarsest_solve");
}

// index of the first level handled by the bottom kernel (-1: none).  It needs
// damped Jacobi or Chebyshev and at least one smoothed level above the
// coarsest; the level is rso_autotune's choice or the built-in rule's.
int bottom_level(const rso_handle* h, bool fp32) {
  const int nl = (int)h->L.size();
  if (h->cfg.smoother == RSO_SMOOTH_GS || nl < 3 || nl > BOT_MAX_LEVELS || h->nc == 0) return -1;
  if (h->cfg.pre > BOT_MAX_SWEEPS || h->cfg.post > BOT_MAX_SWEEPS) return -1;
  // a level chosen by rso_autotune: any level from 1 to nl - 2, or none
  if (h->tune.bottom == -1) return -1;
  if (h->tune.bottom >= 1 && h->tune.bottom <= nl - 2) return h->tune.bottom;
  // built-in rule, for the FP32 V-cycle of mixed precision (the FP64 one keeps
  // its per-level launches): the persistent grid-wide kernel from the first
  // level of at most kBottomMaxNodes nodes, whose sweeps are latency-bound
  // (256^3: from 33^3, 35.2 -> 33.6 ms per solve; 64^3: from 17^3, 5.6 ->
  // 4.2 ms); the cluster kernel only when rso_autotune finds it faster
  if (!fp32 || h->cfg.precision != RSO_MIXED || h->tune.bottom_kind != 1) return -1;
  for (int li = 1; li <= nl - 2; li++)
    if (h->L[li].nn <= kBottomMaxNodes) return li;
  return -1;
}

template <typename T>
rso_status bottom_vcycle(rso_handle* h, int lb, int pre, int post) {
  BottomArgs<T> A;
  const int nl = (int)h->L.size();
  for (int li = 0; li < nl; li++) {
    A.L[li] = h->L[li];
    double om[BOT_MAX_SWEEPS], c1[BOT_MAX_SWEEPS];
    smoother_steps(h, h->L[li].lam, BOT_MAX_SWEEPS, om, c1);
    for (int k = 0; k < BOT_MAX_SWEEPS; k++) {
      A.om[li][k] = (T)om[k];
      A.c1[li][k] = (T)c1[k];
    }
  }
  A.lb = lb; A.nl = nl; A.pre = pre; A.post = post;
  const int N = 3 * h->nc;
  A.kinv = h->c_K + (size_t)N * N;
  A.cnodes = h->c_nodes;
  A.nc = h->nc;
  A.cf = h->L[0].nb > 1 ? h->c_fb : h->c_f;
  double bnodes = 0;
  for (int li = lb; li < nl; li++) bnodes += (double)h->L[li].nn * h->L[li].nb;
  if (h->tune.bottom_kind == 0) {
    if (h->prof_on) prof_begin(h, PC_BOTTOM, bnodes);
    k_bottom<T><<<BOT_CTAS, BOT_THREADS, 0, h->stream>>>(A); rso::note_launch();
    if (h->prof_on) prof_end(h, PC_BOTTOM);
    return launch_check(h, "bottom_vcycle");
  }
  for (int li = lb; li < nl; li++)
    if (h->L[li].NP * h->L[li].nb >= (1LL << 31)) {
      h->err = "the persistent bottom kernel takes levels below 2^31 padded nodes";
      return RSO_ERR_UNSUPPORTED;
    }
  // the persistent kernel: as many CTAs as the largest level has tiles, at
  // most as many as are resident at once (a cooperative launch refuses more)
  static std::atomic<int> occ_cache[2][64];
  const int ti = sizeof(T) == 4 ? 0 : 1;
  const int dev = h->device >= 0 && h->device < 64 ? h->device : 0;
  int occ = occ_cache[ti][dev].load(std::memory_order_relaxed);
  if (occ <= 0) {
    RSO_CHECK_CUDA(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_bottom_grid<T>, gb_threads<T>(), 0));
    occ_cache[ti][dev].store(occ, std::memory_order_relaxed);
  }
  int sms = 0;
  RSO_CHECK_CUDA(h, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  long long need = 1;
  for (int li = lb; li < nl; li++) {
    const Level& l = h->L[li];
    need = std::max(need, sizeof(T) == 4 ? (long long)cdiv(l.NP / 4 * l.nb, G9)
                                         : (long long)cdiv(l.nx, 32) * cdiv(l.ny, CTY) * l.nz * l.nb);
  }
  const int grid = (int)std::max<long long>(1, std::min<long long>(need, (long long)occ * sms));
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(grid);
  lc.blockDim = sizeof(T) == 4 ? dim3(gb_threads<T>()) : dim3(32, CTY, 3);
  lc.dynamicSmemBytes = 0;
  lc.stream = h->stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  if (h->prof_on) prof_begin(h, PC_BOTTOM, bnodes);
  RSO_CHECK_CUDA(h, cudaLaunchKernelEx(&lc, k_bottom_grid<T>, A, h->gbar));
  rso::note_launch();
  if (h->prof_on) prof_end(h, PC_BOTTOM);
  return launch_check(h, "bottom_vcycle (grid)");
}
// Self-test of the bounded barrier wait: a cooperative launch of a few CTAs
// passes `rounds` barriers whose arrival target is the grid size plus
// short_by; with short_by > 0 no barrier completes, so every CTA's wait gives
// up after limit cycles, sets the flag and returns (no fault, no hang).
__global__ void k_gbar_selftest(unsigned* bar, int rounds, unsigned short_by, long long limit) {
  unsigned gen = 0;
  if (threadIdx.x == 0) gen = ld_acquire_gpu(bar + 1);
  for (int r = 0; r < rounds; r++)
    if (!gbar_sync(bar, gen, threadIdx.x, gridDim.x + short_by, limit)) return;
}

template rso_status bottom_vcycle<double>(rso_handle*, int, int, int);
template rso_status bottom_vcycle<float>(rso_handle*, int, int, int);

// once per handle: the support mask of every fine element, the list of
// coarse elements that have support-touching children, and the cuBLAS handle
rso_status galerkin_setup(rso_handle* h) {
  if (h->L.size() < 2) return RSO_OK;
  const Level& f = h->L[0];
  const Level& c = h->L[1];
  const int F = c.factor, F3 = F * F * F;
  RSO_CHECK_CUDA(h, cudaMalloc(&h->efix, f.NQ));
  RSO_CHECK_CUDA(h, cudaMemsetAsync(h->efix, 0, f.NQ, h->stream));
  k_elem_fixmask<<<cdiv(f.ne, 256), 256, 0, h->stream>>>(f, h->efix); rso::note_launch();
  RSO_TRY(launch_check(h, "element support mask"));
  std::vector<uint8_t> ef(f.NQ);
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(ef.data(), h->efix, f.NQ, cudaMemcpyDeviceToHost, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  std::vector<uint8_t> mark(c.ne, 0);
  for (int z = 0; z < f.ez; z++)
    for (int y = 0; y < f.ey; y++)
      for (int x = 0; x < f.ex; x++)
        if (ef[f.eidx(x, y, z)]) mark[x / F + (long long)c.ex * (y / F + (long long)c.ey * (z / F))] = 1;
  std::vector<int> list;
  for (long long E = 0; E < c.ne; E++)
    if (mark[E]) list.push_back((int)E);
  h->n_gfix = (int)list.size();
  if (h->n_gfix) {
    RSO_CHECK_CUDA(h, cudaMalloc(&h->gfix, sizeof(int) * list.size()));
    RSO_CHECK_CUDA(h, cudaMemcpy(h->gfix, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice));
  }
  (void)F3;
  return RSO_OK;
}

rso_status galerkin(rso_handle* h) {
  for (size_t li = 1; li < h->L.size(); li++) {
    Level& c = h->L[li];
    const Level& f = h->L[li - 1];
    if (li == 1)
    {
      const int F = c.factor;
      const unsigned nblk = (unsigned)cdiv(c.ne, GE);
      if (F == 4) k_galerkin_first<4><<<nblk, 256, 0, h->stream>>>(f, c, h->rp64, h->efix, h->T1, c.KE);
      else k_galerkin_first<2><<<nblk, 256, 0, h->stream>>>(f, c, h->rp64, h->efix, h->T1, c.KE);
      rso::note_launch();
      RSO_TRY(launch_check(h, "galerkin first level"));
      if (h->n_gfix > 0) {
        k_galerkin_fix<<<h->n_gfix, 288, 0, h->stream>>>(f, c, F, h->rp64, h->K0_dev, h->efix, h->gfix, c.KE);
      }
    }
    else
      k_galerkin_next<<<(unsigned)c.ne, 288, 0, h->stream>>>(f, c, f.KE, c.KE);
    rso::note_launch();
    RSO_TRY(launch_check(h, "galerkin"));
    k_assemble<<<cdiv(27 * c.nn, 256), 256, 0, h->stream>>>(c, c.KE, c.st64, c.st32); rso::note_launch();
    RSO_TRY(launch_check(h, "assemble"));
  }
  return RSO_OK;
}

rso_status coarsest_factor(rso_handle* h) {
  if (h->L.size() < 2 || h->nc == 0) return RSO_OK;
  const Level& c = h->L.back();
  const int N = 3 * h->nc;
  RSO_CHECK_CUDA(h, cudaMemsetAsync(h->c_K, 0, sizeof(double) * (size_t)N * N, h->stream));
  RSO_CHECK_CUDA(h, cudaMemsetAsync(h->c_flag, 0, sizeof(int), h->stream));
  // crow map lives right after the c_nodes list (see capi set-up)
  k_coarse_dense<<<cdiv((long long)h->nc * 243, 256), 256, 0, h->stream>>>(c, c.st64, h->c_nodes,
                                                                           h->c_nodes + h->nc, h->nc, h->c_K); rso::note_launch();
  RSO_TRY(launch_check(h, "coarsest assembly"));
  // support-free problems: K is singular on the rigid motions R of the
  // coarsest nodes; the pseudo-inverse (the reference's BDCSVD solve,
  // grid/Grid.cpp:4123-4185) is (K + a R R^T)^-1 - R R^T / a, a the mean diagonal
  double a_rig = 0;
  if (!h->has_support && h->c_R) {
    RSO_TRY(dense_trace(h, h->c_K, N, h->c_f));
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(&a_rig, h->c_f, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
    a_rig /= N;
    if (!(a_rig > 0)) { h->err = "coarsest operator has no positive diagonal"; return RSO_ERR_STATE; }
    RSO_TRY(dense_rank_update(h, h->c_K, N, h->c_R, 6, a_rig));
  }
  RSO_TRY(dense_spd_inverse(h, h->c_K, h->c_K + (size_t)N * N, h->c_K + 2 * (size_t)N * N, N, h->c_flag));
  if (a_rig > 0) RSO_TRY(dense_rank_update(h, h->c_K + (size_t)N * N, N, h->c_R, 6, -1.0 / a_rig));
  int flag = 0;
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(&flag, h->c_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  if (flag) {
    h->err = h->has_support ? "coarsest operator is not positive definite (no support node reaches it?)"
                            : "coarsest operator is singular beyond the rigid motions (disconnected parts?)";
    return RSO_ERR_UNSUPPORTED;
  }
  return RSO_OK;
}

// lambda_max(D^-1 K) per level: power iteration on the Jacobi operator
// random start vector, zero at inactive nodes, halo and (fine level) support nodes
__global__ void k_seed_vec(const Level L, float* v, uint64_t seed, int zero_support) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= L.NP) return;
  const uint8_t c = L.vclass[i];
  const bool z = !(c & NC_ACTIVE) || (zero_support && (c & NC_SUPPORT));
#pragma unroll
  for (int k = 0; k < 3; k++) v[i + k * L.NP] = z ? 0.f : (float)rso_urand(seed, (uint64_t)(i + k * L.NP));
}

// lambda_max(D^-1 K) of every smoothed level: 12 power iterations in FP32
// (the estimate only sets the smoother's step sizes and gets a 5 % margin)
rso_status estimate_lambda(rso_handle* h) {
  const int iters = 12;
  for (size_t li = 0; li + 1 < h->L.size() || (li == 0 && h->L.size() == 1); li++) {
    Level& l = h->L[li];
    const long long n3 = 3 * l.NP;
    k_seed_vec<<<cdiv(l.NP, 256), 256, 0, h->stream>>>(l, l.u32, 777 + li, li == 0); rso::note_launch();
    RSO_CHECK_CUDA(h, cudaMemsetAsync(l.f32, 0, sizeof(float) * n3, h->stream));
    double lam = 1.0;
    for (int it = 0; it < iters; it++) {
      // t = u - D^-1 K u, r = D^-1 K u
      if (li == 0) RSO_TRY(fine_jacobi<float>(h, l.u32, l.f32, l.t32, h->rp32, 1.0));
      else RSO_TRY(coarse_jacobi<float>(h, (int)li, l.u32, l.f32, l.t32, 1.0));
      double uu = 0, rr = 0;
      RSO_TRY(pow_step(h, n3, l.u32, l.t32, l.r32, &uu, &rr));
      if (!(uu > 0)) break;
      lam = std::sqrt(rr / uu);
      std::swap(l.u32, l.r32);
    }
    l.lam = 1.05 * lam;
    if (h->L.size() == 1) break;
  }
  return fine_stage_check(h);
}

template rso_status coarse_residual<double>(rso_handle*, int, const double*, const double*, double*);
template rso_status coarse_residual<float>(rso_handle*, int, const float*, const float*, float*);
template rso_status coarse_jacobi<double>(rso_handle*, int, const double*, const double*, double*, double,
                                          const double*, double);
template rso_status coarse_jacobi<float>(rso_handle*, int, const float*, const float*, float*, double, const float*,
                                         double);
template rso_status coarse_gs<double>(rso_handle*, int, double*, const double*, int, int);
template rso_status coarse_gs<float>(rso_handle*, int, float*, const float*, int, int);
template rso_status restrict_<double>(rso_handle*, int, const double*, double*);
template rso_status restrict_<float>(rso_handle*, int, const float*, float*);
template rso_status prolong<double>(rso_handle*, int, const double*, double*);
template rso_status prolong<float>(rso_handle*, int, const float*, float*);
template rso_status coarsest_solve<double>(rso_handle*, const double*, double*);
template rso_status coarsest_solve<float>(rso_handle*, const float*, float*);

}  // namespace rso

using namespace rso;

extern "C" rso_status rso_grid_barrier_selftest(rso_handle* h, int short_by, double limit_ms, int* gave_up) {
  if (!h || !gave_up || short_by < 0 || short_by > 1 || !(limit_ms > 0) || limit_ms > 1000) return RSO_ERR_INVALID_ARG;
  if (!h->gbar) {
    h->err = "grid barrier state not allocated";
    return RSO_ERR_STATE;
  }
  const int dev = h->device >= 0 ? h->device : 0;
  int khz = 0;
  RSO_CHECK_CUDA(h, cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, dev));
  const long long limit = (long long)(limit_ms * (khz > 0 ? khz : 2000000));
  RSO_CHECK_CUDA(h, cudaMemsetAsync(h->gbar, 0, sizeof(unsigned) * 4, h->stream));
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(4);
  lc.blockDim = dim3(128);
  lc.stream = h->stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  RSO_CHECK_CUDA(h, cudaLaunchKernelEx(&lc, k_gbar_selftest, h->gbar, 8, (unsigned)short_by, limit));
  note_launch();
  unsigned flag = 0;
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(&flag, h->gbar + 2, sizeof(flag), cudaMemcpyDeviceToHost, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  RSO_CHECK_CUDA(h, cudaMemsetAsync(h->gbar, 0, sizeof(unsigned) * 4, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  *gave_up = flag != 0;
  return RSO_OK;
}
