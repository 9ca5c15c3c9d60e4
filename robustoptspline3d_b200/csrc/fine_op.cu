// Matrix-free SIMP elasticity operator on the finest level.
//
// r_i = f_i - sum_{e incident to i} rho_e^p sum_{j in e} K0[vi, vj] u_j
// (update_residual_OTFA_WS_kernel grid/Grid.cu:2320-2376, applyK_OTFA_kernel
// grid/Grid.cu:4358-4436, gs_relax_OTFA_WS_kernel grid/Grid.cu:1742-1885).
//
// The residual / apply / damped-Jacobi kernel (k_fine_w) evaluates every
// element product K0 u_e in the sum/difference ("Walsh") basis of the
// element's nodes, where K0 is block diagonal (8 blocks of 3x3, 45 non-zero
// entries), and shares the face transforms between the two elements on
// either side of a node plane, so a fine node costs about 200 additions and
// multiplications instead of 576 multiply-adds.  Support DOFs hold zero by
// construction, so neighbours need no Dirichlet test; support rows are
// handled from the node-class byte.  The point Gauss-Seidel colour sweep and
// the first Jacobi sweep from a zero iterate use K0 directly.
#include "rso_internal.cuh"
#include <cmath>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_pipeline.h>
#include <atomic>
#include <mutex>

namespace rso {

__constant__ double cK0d[576];
__constant__ float cK0f[576];

template <typename T>
__device__ __forceinline__ T k0(int i);
template <>
__device__ __forceinline__ double k0<double>(int i) { return cK0d[i]; }
template <>
__device__ __forceinline__ float k0<float>(int i) { return cK0f[i]; }

rso_status upload_walsh(rso_handle* h);

rso_status upload_K0(rso_handle* h) {
  RSO_TRY(upload_walsh(h));
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

// ---------------------------------------------------------------- Walsh-basis element operator
//
// Along each axis the two nodes of an element are combined into a sum and a
// difference (H = [[1, 1], [-1, 1]]); over the 8 nodes this is W = H (x) H (x) H,
// with W^T W = 8 I.  The reflections of the cube commute with K0, so in this
// basis K0 splits into 8 symmetric 3x3 blocks: block c couples the entries
// (mode c ^ (1 << j), component j), j = 0..2, and
//   K0 u = W^T B W u,  B = (W K0 W^T) / 64  (45 non-zeros instead of 576).
// Structural zeros (exact for the isotropic cube; checked on the host):
// for one-bit c the translation row/column (c >> i & 1), for two-bit c the
// entries coupling the axis outside c with the two inside it.
__constant__ double cBd[72];  // [c][i][j]
__constant__ float cBf[72];
__constant__ double cD0d[9];  // diagonal 3x3 block of local node 0
__constant__ float cD0f[9];
// The packed FP32 kernel uses the blocks' finer structure (the isotropic
// material and the cube's rotations; checked on the host): with
//   A0, B0, A7, B7 the diagonal and off-diagonal entries of blocks 0 and 7
//   (full 3 x 3, a I + b (J - I)), P, Q those of the one-bit blocks
//   ([[P, Q], [Q, P]] on the two axes outside c), R, S those of the two-bit
//   blocks (R on the 2 x 2 block of the two axes in c, all four entries; S
//   on the axis outside c)
// and the node-0 diagonal block D0 = [[Da, Db, Db], [Db, Da, Db], [Db, Db, Da]],
// cWp holds, duplicated into both lanes: A0 - B0, B0, A7 - B7, B7, P, Q, R, S, Da, Db.
__constant__ float2 cWp[10];
enum { W_A0 = 0, W_B0, W_A7, W_B7, W_P, W_Q, W_R, W_S, W_DA, W_DB };

template <typename T>
__device__ __forceinline__ T bw(int i);
template <>
__device__ __forceinline__ double bw<double>(int i) { return cBd[i]; }
template <>
__device__ __forceinline__ float bw<float>(int i) { return cBf[i]; }
template <typename T>
__device__ __forceinline__ T d0(int i);
template <>
__device__ __forceinline__ double d0<double>(int i) { return cD0d[i]; }
template <>
__device__ __forceinline__ float d0<float>(int i) { return cD0f[i]; }

__host__ __device__ constexpr bool b_zero(int c, int i, int j) {
  const int pc = (c & 1) + ((c >> 1) & 1) + ((c >> 2) & 1);
  if (pc == 1) return ((c >> i) & 1) || ((c >> j) & 1);
  if (pc == 2) {
    const int out = ~c & 7;
    return (((out >> i) & 1) != 0) != (((out >> j) & 1) != 0);
  }
  return false;
}

rso_status upload_walsh(rso_handle* h) {
  const double* K = h->K0;
  // W[m][a] = prod_axis H[m_axis][a_axis]
  auto Hh = [](int m, int b) { return m == 0 ? 1.0 : (b ? 1.0 : -1.0); };
  double W[8][8];
  for (int m = 0; m < 8; m++)
    for (int a = 0; a < 8; a++) W[m][a] = Hh(m & 1, a & 1) * Hh((m >> 1) & 1, (a >> 1) & 1) * Hh(m >> 2, a >> 2);
  double B[72], kmax = 0;
  for (int i = 0; i < 576; i++) kmax = std::fmax(kmax, std::fabs(K[i]));
  for (int c = 0; c < 8; c++)
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        const int mi = c ^ (1 << i), mj = c ^ (1 << j);
        double s = 0;
        for (int a = 0; a < 8; a++)
          for (int b = 0; b < 8; b++) s += W[mi][a] * K[(a * 3 + i) * 24 + b * 3 + j] * W[mj][b];
        s /= 64.0;
        if (b_zero(c, i, j)) {
          if (std::fabs(s) > 1e-12 * kmax) {
            h->err = "element matrix lacks the reflection symmetry of the cube";
            return RSO_ERR_INVALID_ARG;
          }
          s = 0;
        }
        B[c * 9 + i * 3 + j] = s;
      }
  // diagonal blocks: K0[a][a](i, j) = D0(i, j) * sigma_i(a) * sigma_j(a), sigma = 1 - 2 bit
  double D0[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) D0[i * 3 + j] = K[i * 24 + j];
  for (int a = 0; a < 8; a++)
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        const double si = ((a >> i) & 1) ? -1.0 : 1.0, sj = ((a >> j) & 1) ? -1.0 : 1.0;
        if (std::fabs(K[(a * 3 + i) * 24 + a * 3 + j] - D0[i * 3 + j] * si * sj) > 1e-12 * kmax) {
          h->err = "element matrix diagonal blocks lack the reflection symmetry of the cube";
          return RSO_ERR_INVALID_ARG;
        }
      }
  float Bf[72], Df[9];
  for (int i = 0; i < 72; i++) Bf[i] = (float)B[i];
  for (int i = 0; i < 9; i++) Df[i] = (float)D0[i];
  RSO_CHECK_CUDA(h, cudaMemcpyToSymbolAsync(cBd, B, sizeof(B), 0, cudaMemcpyHostToDevice, h->stream));
  RSO_CHECK_CUDA(h, cudaMemcpyToSymbolAsync(cBf, Bf, sizeof(Bf), 0, cudaMemcpyHostToDevice, h->stream));
  RSO_CHECK_CUDA(h, cudaMemcpyToSymbolAsync(cD0d, D0, sizeof(D0), 0, cudaMemcpyHostToDevice, h->stream));
  RSO_CHECK_CUDA(h, cudaMemcpyToSymbolAsync(cD0f, Df, sizeof(Df), 0, cudaMemcpyHostToDevice, h->stream));
  // the finer structure the packed kernel relies on (see cWp)
  auto Bv = [&](int c, int i, int j) { return B[c * 9 + i * 3 + j]; };
  const double A0 = Bv(0, 0, 0), B0 = Bv(0, 0, 1), A7 = Bv(7, 0, 0), B7 = Bv(7, 0, 1);
  const double Pv = Bv(1, 1, 1), Qv = Bv(1, 1, 2), Rv = Bv(3, 0, 0), Sv = Bv(3, 2, 2);
  const double Da = D0[0], Db = D0[1];
  double worst = 0;
  for (int c = 0; c < 8; c++)
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        const int pc = (c & 1) + ((c >> 1) & 1) + ((c >> 2) & 1);
        double e = 0;
        if (b_zero(c, i, j)) e = 0;
        else if (pc == 0) e = i == j ? A0 : B0;
        else if (pc == 3) e = i == j ? A7 : B7;
        else if (pc == 1) e = i == j ? Pv : Qv;
        else e = ((~c >> i) & 1) ? Sv : Rv;  // the axis outside c: S, else R
        worst = std::fmax(worst, std::fabs(Bv(c, i, j) - e));
      }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) worst = std::fmax(worst, std::fabs(D0[i * 3 + j] - (i == j ? Da : Db)));
  if (worst > 1e-12 * kmax) {
    h->err = "element matrix lacks the symmetry of an isotropic cube";
    return RSO_ERR_INVALID_ARG;
  }
  const double Wv[10] = {A0 - B0, B0, A7 - B7, B7, Pv, Qv, Rv, Sv, Da, Db};
  float2 Wp[10];
  for (int i = 0; i < 10; i++) Wp[i] = make_float2((float)Wv[i], (float)Wv[i]);
  RSO_CHECK_CUDA(h, cudaMemcpyToSymbolAsync(cWp, Wp, sizeof(Wp), 0, cudaMemcpyHostToDevice, h->stream));
  // the host copies are stack arrays: finish the copies before returning
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

// Residual / apply / damped-Jacobi kernel.  A CTA of 32 x TY threads marches
// along z through FZC node planes.  Thread (tx, ty) owns the element column
// (ex, ey) = (x0 - 1 + tx, y0 - 1 + ty) and the node (ex + 1, ey + 1), so a
// CTA computes 32 x TY element columns and writes the 31 x (TY - 1) nodes
// whose four surrounding columns it holds.  Per element layer z (between node
// planes z and z+1) a thread
//   1. forms the xy sum/difference modes of the 4 nodes of its top face
//      (plane z+1) from the staged plane, the bottom face coming from the
//      previous layer,
//   2. combines them along z, applies the 8 blocks of B and scales by rho^p,
//   3. splits the result into its bottom- and top-face parts, adds the bottom
//      part to the top part of layer z-1 (both act on plane z), and
//   4. transforms that face back to its 4 corner nodes; the node sums the
//      corners of its 4 columns through shared memory.
// Node planes of u (3 components, 33 x (TY+1)) and element layers of rho^p are
// staged with cp.async WPD stages ahead in WNSLOT slots.
constexpr int WTX = 32, FZC = 32, WPD = 2, WNSLOT = 4;
static_assert((WNSLOT & (WNSLOT - 1)) == 0, "slot indices are masks of the stage number");

template <typename T, int TY>
constexpr int walsh_smem_bytes() {
  return (int)sizeof(T) * (WNSLOT * (3 * 36 * (TY + 1) + 36 * TY) + 2 * 9 * WTX * TY);
}

// MODE 0: out = f - K u;  MODE 1: out = K u (support rows pass u);
// MODE 2: out = u + c1 (u - uprev) + omega D^-1 (f - K u), D = 3x3 diagonal
//         block: damped block Jacobi for c1 = 0, a Chebyshev step otherwise
//         (uprev NULL reads as zero)
// RR (MODE 0 only): also write an FP32 copy of r (out32) and sum r . r into
// per-CTA partials (dotp); a separate instantiation so the plain residual
// carries none of it
template <typename T, int MODE, int TY, bool RR = false>
__global__ void __launch_bounds__(WTX* TY, sizeof(T) == 8 ? 2 : 3)
    k_fine_w(const Level L, const T* __restrict__ u, const T* __restrict__ f, T* __restrict__ out,
             const T* __restrict__ rp, T omega, double* __restrict__ dotp, const T* __restrict__ uprev,
             T c1, float* __restrict__ out32) {
  // Staged rows are 16-byte aligned windows of RX entries starting at the
  // tile's first padded x index rounded down to a multiple of 4 (ox = offset
  // of the tile inside the window), copied in 16-byte chunks.
  constexpr int RX = 36, NPL = RX * (TY + 1), NE = WTX * TY, SLOT = 3 * NPL + RX * TY;
  constexpr int EPC = 16 / (int)sizeof(T), CPR = RX / EPC;  // entries per chunk, chunks per row
  constexpr int NCH = (3 * (TY + 1) + TY) * CPR, KC = (NCH + NE - 1) / NE;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ss = reinterpret_cast<T*>(smem_raw);  // [WNSLOT][SLOT]: u plane (3 comps x (TY+1) rows) + rho layer (TY rows)
  T* sx = ss + WNSLOT * SLOT;              // [2][9][NE]: corners (0,0), (1,0), (0,1), by plane parity
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * WTX + tx;
  const int x0 = blockIdx.x * (WTX - 1), y0 = blockIdx.y * (TY - 1);
  // blockIdx.z = z chunk + (number of chunks) * system; systems share rho^p
  const int nzc = (L.nz + FZC - 1) / FZC, bsys = blockIdx.z / nzc;
  const int z0 = (blockIdx.z - bsys * nzc) * FZC, z1 = min(z0 + FZC, L.nz);
  {
    const long long off = (long long)bsys * 3 * L.NP;
    u += off;
    f += off;
    out += off;
    if (uprev != nullptr) uprev += off;
  }
  const int ex = x0 - 1 + tx, ey = y0 - 1 + ty;
  const long long NP = L.NP;
  const int xs = x0 & ~3, ox = x0 - xs;

  // this thread's chunks: in-plane global offset (-1: zero fill), shared
  // offset, and whether the chunk belongs to the rho layer
  int goff[KC], soff[KC];
  bool isr[KC];
#pragma unroll
  for (int kk = 0; kk < KC; kk++) {
    const int k = tid + kk * NE;
    const int row = k / CPR, j = k - row * CPR, xg = xs + j * EPC;
    goff[kk] = -1;
    soff[kk] = -1;
    isr[kk] = false;
    if (k < NCH) {
      if (row < 3 * (TY + 1)) {
        const int c = row / (TY + 1), yr = row - c * (TY + 1), gyp = y0 + yr;  // padded y index
        soff[kk] = c * NPL + yr * RX + j * EPC;
        if (gyp <= L.py - 1 && xg + EPC <= L.px) goff[kk] = (int)(c * NP + (long long)gyp * L.px + xg);
      } else {
        const int yr = row - 3 * (TY + 1), gyp = y0 + yr;
        isr[kk] = true;
        soff[kk] = 3 * NPL + yr * RX + j * EPC;
        if (gyp <= L.qy - 1 && xg + EPC <= L.qx) goff[kk] = (int)((long long)gyp * L.qx + xg);
      }
    }
  }
  const long long pxy = (long long)L.px * L.py, qxy = (long long)L.qx * L.qy;
  // stage s: node plane s of u and element layer s of rho^p (zero outside)
  auto issue = [&](int s) {
    T* dst = ss + ((s + WNSLOT) & (WNSLOT - 1)) * SLOT;
    const long long po = pxy * (s + 1), qo = qxy * (s + 1);
#pragma unroll
    for (int kk = 0; kk < KC; kk++) {
      if (soff[kk] < 0) continue;
      const bool ok = goff[kk] >= 0 && (isr[kk] ? s <= L.ez : s <= L.nz);
      if (ok)
        __pipeline_memcpy_async(dst + soff[kk], isr[kk] ? rp + qo + goff[kk] : u + po + goff[kk], 16);
      else
        *reinterpret_cast<float4*>(dst + soff[kk]) = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __pipeline_commit();
  };
  // xy modes of the 4 face nodes of this column on a staged plane; also the
  // own node (corner (1,1)) values
  auto face = [&](const T* pl, T (&F)[4][3], T (&own)[3]) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const T* p = pl + c * NPL + ty * RX + tx + ox;
      const T a00 = p[0], a10 = p[1], a01 = p[RX], a11 = p[RX + 1];
      const T s0 = a00 + a10, d0 = a10 - a00, s1 = a01 + a11, d1 = a11 - a01;
      F[0][c] = s0 + s1;  // (mx, my) = (0, 0)
      F[1][c] = d0 + d1;  // (1, 0)
      F[2][c] = s1 - s0;  // (0, 1)
      F[3][c] = d1 - d0;  // (1, 1)
      own[c] = a11;
    }
  };

  for (int s = z0 - 1; s <= z0 - 1 + WPD; s++) issue(s);
  __pipeline_wait_prior(WPD);
  __syncthreads();
  const bool writer = tx < WTX - 1 && ty < TY - 1 && ex + 1 < L.nx && ey + 1 < L.ny;
  // per-plane registers: F face modes of plane z; Gt top-face part of layer
  // z-1; uc/uo u at the own node on planes z / z-1; own corner, f and class
  // of the plane being emitted; ra/rb rho^p of the 4 columns in the two
  // layers around it
  T F[4][3], Gt[4][3], uc[3], uo[3], own[3], fo[3], po[3], ra[4], rb[4];
  uint8_t clo = 0;
  double pq = 0;  // with dotp: MODE 1 this thread's share of u . (K u), MODE 0 of r . r
  face(ss + ((z0 - 1 + WNSLOT) & (WNSLOT - 1)) * SLOT, F, uc);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    Gt[q][0] = Gt[q][1] = Gt[q][2] = T(0);
    ra[q] = rb[q] = T(0);
  }
#pragma unroll
  for (int c = 0; c < 3; c++) uo[c] = own[c] = fo[c] = po[c] = T(0);

  // node plane zo from the corners its 4 columns left in exchange buffer xb
  auto emit = [&](int zo, const T* xb) {
    if (!writer) return;
    T acc[3];
#pragma unroll
    for (int c = 0; c < 3; c++)
      acc[c] = own[c] + xb[(2 * 3 + c) * NE + tid + 1] + xb[(1 * 3 + c) * NE + tid + WTX] +
               xb[(0 * 3 + c) * NE + tid + WTX + 1];
    const long long n = L.nidx(ex + 1, ey + 1, zo);
    const bool work = (clo & NC_ACTIVE) && !(clo & NC_SUPPORT);
    if (MODE == 0) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const T r = fo[c] - (work ? acc[c] : T(0));
        out[n + c * NP] = r;
        if constexpr (RR) {  // an FP32 copy of r and r . r from the same pass
          out32[n + c * NP] = (float)r;
          pq += (double)r * (double)r;
        }
      }
    } else if (MODE == 1) {
      const bool pass = (clo & NC_SUPPORT) != 0;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const T q = pass ? uo[c] : (work ? acc[c] : T(0));
        out[n + c * NP] = q;
        pq += (double)uo[c] * (double)q;
      }
    } else {
      if (!work) {
#pragma unroll
        for (int c = 0; c < 3; c++) out[n + c * NP] = T(0);
      } else {
        // D = sum_e rho_e K0[a_e][a_e]; node bits in column (ex + a, ey + b), layer zo - 1 + l
        // are (1 - a, 1 - b, 1 - l), so sigma = (2a - 1, 2b - 1, 2l - 1); ra: l = 0, rb: l = 1
        const T R = (ra[0] + ra[1] + ra[2] + ra[3]) + (rb[0] + rb[1] + rb[2] + rb[3]);
        const T pxy_ = (ra[0] + ra[3] - ra[1] - ra[2]) + (rb[0] + rb[3] - rb[1] - rb[2]);
        const T xlo = ra[1] + ra[3] - ra[0] - ra[2], xhi = rb[1] + rb[3] - rb[0] - rb[2];
        const T ylo = ra[2] + ra[3] - ra[0] - ra[1], yhi = rb[2] + rb[3] - rb[0] - rb[1];
        const T pxz = xhi - xlo, pyz = yhi - ylo;
        const T a = d0<T>(0) * R, b = d0<T>(1) * pxy_, cc = d0<T>(2) * pxz;
        const T d = d0<T>(4) * R, e = d0<T>(5) * pyz, g = d0<T>(8) * R;
        const T r0 = fo[0] - acc[0], r1 = fo[1] - acc[1], r2 = fo[2] - acc[2];
        const T A = d * g - e * e, B = cc * e - b * g, C = b * e - cc * d;
        const T det = a * A + b * B + cc * C;
        const T id = omega / det;
        const T E = a * g - cc * cc, Fm = b * cc - a * e, I = a * d - b * b;
        out[n] = uo[0] + c1 * (uo[0] - po[0]) + id * (A * r0 + B * r1 + C * r2);
        out[n + NP] = uo[1] + c1 * (uo[1] - po[1]) + id * (B * r0 + E * r1 + Fm * r2);
        out[n + 2 * NP] = uo[2] + c1 * (uo[2] - po[2]) + id * (C * r0 + Fm * r1 + I * r2);
      }
    }
  };

  for (int z = z0 - 1; z < z1; z++) {
    // one barrier per layer: stage z+1 is staged, the corners of plane z-1
    // are visible, and the slot of stage z-1 is free for refilling
    __pipeline_wait_prior(WPD - 1);
    __syncthreads();
    issue(z + 1 + WPD);
    if (z - 1 >= z0) emit(z - 1, sx + ((z - 1) & 1) * 9 * NE);
    if (writer && z >= z0) {
      // operands of plane z, used when it is emitted in the next step
      const long long n = L.nidx(ex + 1, ey + 1, z);
      clo = L.vclass[n];
      if (MODE != 1) {
#pragma unroll
        for (int c = 0; c < 3; c++) fo[c] = f[n + c * NP];
        if (MODE == 2 && uprev != nullptr) {
#pragma unroll
          for (int c = 0; c < 3; c++) po[c] = uprev[n + c * NP];
        }
      }
    }
    const T* su = ss + ((z + 1 + WNSLOT) & (WNSLOT - 1)) * SLOT;
    const T* sr = ss + ((z + WNSLOT) & (WNSLOT - 1)) * SLOT + 3 * NPL;
    T v[8][3], un[3];
    {
      T Fn[4][3];
      face(su, Fn, un);
#pragma unroll
      for (int q = 0; q < 4; q++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          v[q][c] = F[q][c] + Fn[q][c];
          v[q + 4][c] = Fn[q][c] - F[q][c];
          F[q][c] = Fn[q][c];
        }
    }
    // blocks of B, in place (block c maps its three entries onto themselves), times rho^p
    const int ri = ty * RX + tx + ox;
    const T re = sr[ri];
#pragma unroll
    for (int c = 0; c < 8; c++) {
      T in[3], o[3];
#pragma unroll
      for (int j = 0; j < 3; j++) in[j] = v[c ^ (1 << j)][j];
#pragma unroll
      for (int i = 0; i < 3; i++) {
        T s = T(0);
#pragma unroll
        for (int j = 0; j < 3; j++)
          if (!b_zero(c, i, j)) s = fma(bw<T>(c * 9 + i * 3 + j), in[j], s);
        o[i] = s * re;
      }
#pragma unroll
      for (int i = 0; i < 3; i++) v[c ^ (1 << i)][i] = o[i];
    }
    if (MODE == 2) {
#pragma unroll
      for (int q = 0; q < 4; q++) ra[q] = rb[q];
      rb[0] = re;
      rb[1] = writer ? sr[ri + 1] : T(0);
      rb[2] = writer ? sr[ri + RX] : T(0);
      rb[3] = writer ? sr[ri + RX + 1] : T(0);
    }
    // bottom face (plane z) = S - D, top face (plane z+1) = S + D
    T tot[4][3];
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int c = 0; c < 3; c++) {
        tot[q][c] = Gt[q][c] + (v[q][c] - v[q + 4][c]);
        Gt[q][c] = v[q][c] + v[q + 4][c];
      }
    if (z >= z0) {
      // back to the 4 corners of plane z: corner (bx, by); (1,1) stays here
      T* xb = sx + (z & 1) * 9 * NE;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const T e0 = tot[0][c] - tot[1][c], e1 = tot[0][c] + tot[1][c];  // my = 0: bx = 0, 1
        const T g0 = tot[2][c] - tot[3][c], g1 = tot[2][c] + tot[3][c];  // my = 1
        xb[(0 * 3 + c) * NE + tid] = e0 - g0;  // (0, 0)
        xb[(1 * 3 + c) * NE + tid] = e1 - g1;  // (1, 0)
        xb[(2 * 3 + c) * NE + tid] = e0 + g0;  // (0, 1)
        own[c] = e1 + g1;                      // (1, 1)
      }
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      uo[c] = uc[c];
      uc[c] = un[c];
    }
  }
  __syncthreads();
  emit(z1 - 1, sx + ((z1 - 1) & 1) * 9 * NE);
  if ((MODE == 1 || RR) && dotp != nullptr) {
    // per-CTA partial of u . (K u) or r . r, summed by a second pass
    __shared__ double sred[TY];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pq += __shfl_down_sync(0xffffffffu, pq, o);
    if (tx == 0) sred[ty] = pq;
    __syncthreads();
    if (tid == 0) {
      double t = 0;
#pragma unroll
      for (int w = 0; w < TY; w++) t += sred[w];
      dotp[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * (blockIdx.z - bsys * nzc)) +
           (long long)bsys * gridDim.x * gridDim.y * nzc] = t;
    }
  }
  __pipeline_wait_prior(0);
}

// ---------------------------------------------------------------- FP32 kernel on packed pairs
//
// The same operator as k_fine_w for FP32, with two element columns per
// thread: column A = (ex, ey) and column B = (ex, ey + 1).  Every addition and
// multiplication of the two columns is the same, so they run as one packed
// FP32x2 instruction on B200 (add/sub/mul/fma .f32x2), which halves the
// issue slots of the arithmetic; the staging, indexing and loop overhead is
// shared by both columns.  A thread emits the nodes (ex + 1, ey + 1) and
// (ex + 1, ey + 2).
__device__ __forceinline__ float2 p_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 p_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 p_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 p_sub(float2 a, float2 b) {
  unsigned long long r;
  const unsigned long long x = *reinterpret_cast<const unsigned long long*>(&a);
  const unsigned long long y = *reinterpret_cast<const unsigned long long*>(&b);
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(x), "l"(y));
  return *reinterpret_cast<const float2*>(&r);
}

constexpr int kPairMinBlocksRes = 4, kPairMinBlocksJac = 4;

// Bulk-tensor staging (TMA): one thread issues the copies of a stage, their
// completion is tracked by an mbarrier per slot.  Every wait is bounded: after
// kStageTries polls it gives up, counts the event in g_stage_timeouts (read and
// reported as an error by the host after the solve) and lets the kernel run
// on, all of its accesses staying in bounds.
__device__ unsigned int g_stage_timeouts;
constexpr int kStageTries = 1 << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity) {
  for (int i = 0; i < kStageTries; i++)
    if (mbar_test(b, parity)) return true;
  atomicAdd(&g_stage_timeouts, 1u);
  return false;
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* m, int x, int y, int z, int w, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(m)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* m, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(m)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Slot layout of the packed kernel (floats): the u plane (3 comps x (2 TYP + 1)
// rows of 36) at 0, the rho^p layer (2 TYP rows of 36) at pair_rho_off, each
// part starting on 128 bytes as bulk-tensor copies require.
template <int TYP>
constexpr int pair_rho_off() { return (3 * 36 * (2 * TYP + 1) + 31) / 32 * 32; }
template <int TYP>
constexpr int pair_slot() { return pair_rho_off<TYP>() + (36 * 2 * TYP + 31) / 32 * 32; }
// staging slots of the packed kernel: the Jacobi / Chebyshev step keeps two
// more stages resident, so that it reads rho^p of the layers around the
// emitted plane and u at the emitted nodes from shared memory, not registers;
// it takes 8 slots rather than 6 so that slot indices and phases are a mask
// and a shift of the stage number, not a division by 6
constexpr int pair_slots(int mode, bool tma) { return mode == 2 && tma ? 2 * WNSLOT : WNSLOT; }
template <int TYP>
constexpr int pair_smem_bytes(int nslot) {
  // slots + corner exchange [2][4 values][3 comps][32 TYP] + 128 bytes to
  // round the base up to a 128-byte boundary
  return 4 * (nslot * pair_slot<TYP>() + 2 * 12 * 32 * TYP) + 128;
}

// resident CTAs per SM (for 4 thread rows) the register budget is cut for:
// the residual and the Jacobi / Chebyshev step fit 128 registers without
// spills, K u (MODE 1, which carries u at the emitted nodes) 168
constexpr int pair_min_blocks(int mode, int typ) {
  return ((mode == 0 ? kPairMinBlocksRes : mode == 2 ? kPairMinBlocksJac : 3) * 4 + typ - 1) / typ;
}

// TMA: stage u planes and rho^p layers with bulk-tensor copies (tmu: 4-D map
// (px, py, pz, 3 nb) of u, box 36 x (2 TYP + 1) x 1 x 3; tmr: 3-D map
// (qx, qy, qz) of rho^p, box 36 x 2 TYP x 1; out-of-range boxes read zero);
// otherwise every thread stages 16-byte chunks with cp.async.
// DOT (MODE 2 only): also sum f . out into per-CTA partials (dotp); a
// separate instantiation so the plain step carries none of it
template <int MODE, int TYP, bool TMA, bool DOT = false>
__global__ void __launch_bounds__(32 * TYP, pair_min_blocks(MODE, TYP))
    k_fine_p(const Level L, const float* __restrict__ u, const float* __restrict__ f, float* __restrict__ out,
             const float* __restrict__ rp, float omega, double* __restrict__ dotp, const float* __restrict__ uprev,
             float c1, int fzc, const __grid_constant__ CUtensorMap tmu, const __grid_constant__ CUtensorMap tmr) {
  constexpr int RX = 36, ROWS = 2 * TYP, NPL = RX * (ROWS + 1), NT = WTX * TYP;
  constexpr int NS = pair_slots(MODE, TMA);
  static_assert((NS & (NS - 1)) == 0, "slot indices are masks of the stage number");
  constexpr bool LEAN = MODE == 2 && TMA;  // operands of the emitted plane re-read from the slots
  constexpr int RHO = pair_rho_off<TYP>(), SLOT = pair_slot<TYP>();
  constexpr uint32_t STAGE_BYTES = sizeof(float) * (3 * NPL + RX * ROWS);  // both boxes of a stage
  constexpr int CPR = RX / 4;  // 16-byte chunks per staged row
  constexpr int NCH = (3 * (ROWS + 1) + ROWS) * CPR, KC = (NCH + NT - 1) / NT;
  extern __shared__ __align__(128) unsigned char smem_pair[];
  // slots start on a 128-byte shared-memory address whatever the base
  float* ss = reinterpret_cast<float*>(smem_pair + ((128u - (smem_u32(smem_pair) & 127u)) & 127u));  // [NS][SLOT]
  float* sx = ss + NS * SLOT;                  // [2][4][3][NT] corner exchange, by plane parity
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * WTX + tx;
  const int x0 = blockIdx.x * (WTX - 1), y0 = blockIdx.y * (ROWS - 1);
  // blockIdx.z = z chunk of fzc node planes + (number of chunks) * system
  const int nzc = (L.nz + fzc - 1) / fzc, bsys = blockIdx.z / nzc;
  const int z0 = (blockIdx.z - bsys * nzc) * fzc, z1 = min(z0 + fzc, L.nz);
  {
    const long long off = (long long)bsys * 3 * L.NP;
    u += off;
    f += off;
    out += off;
    if (uprev != nullptr) uprev += off;
  }
  const int ex = x0 - 1 + tx, ey = y0 - 1 + 2 * ty;
  const int NP = (int)L.NP, px = L.px;  // 3 NP < 2^31 (checked by the launcher)
  const int nb0 = (ex + 2) + px * (ey + 2), pxy32 = px * L.py;  // node (ex + 1, ey + 1, z) at nb0 + pxy32 (z + 1)
  const int xs = x0 & ~3, ox = x0 - xs;

  int goff[TMA ? 1 : KC], soff[TMA ? 1 : KC];
  bool isr[TMA ? 1 : KC];
#pragma unroll
  for (int kk = 0; kk < (TMA ? 0 : KC); kk++) {
    const int k = tid + kk * NT;
    const int row = k / CPR, j = k - row * CPR, xg = xs + j * 4;
    goff[kk] = -1;
    soff[kk] = -1;
    isr[kk] = false;
    if (k < NCH) {
      if (row < 3 * (ROWS + 1)) {
        const int c = row / (ROWS + 1), yr = row - c * (ROWS + 1), gyp = y0 + yr;
        soff[kk] = c * NPL + yr * RX + j * 4;
        if (gyp <= L.py - 1 && xg + 4 <= L.px) goff[kk] = c * NP + gyp * L.px + xg;
      } else {
        const int yr = row - 3 * (ROWS + 1), gyp = y0 + yr;
        isr[kk] = true;
        soff[kk] = RHO + yr * RX + j * 4;
        if (gyp <= L.qy - 1 && xg + 4 <= L.qx) goff[kk] = gyp * L.qx + xg;
      }
    }
  }
  const long long pxy = (long long)L.px * L.py, qxy = (long long)L.qx * L.qy;
  __shared__ __align__(8) uint64_t bars[NS];
  bool gave_up = false;
  // stage s (node plane s, element layer s) into slot (s + NS) mod NS (NS a power of two, s >= -1)
  auto issue = [&](int s) {
    float* dst = ss + ((s + NS) & (NS - 1)) * SLOT;
    if constexpr (TMA) {
      // thread 0 only; stages past z1 are never read and not issued
      if (s > z1) return;
      uint64_t* bar = &bars[(s + NS) & (NS - 1)];
      mbar_expect_tx(bar, STAGE_BYTES);
      tma_load_4d(dst, &tmu, xs, y0, s + 1, 3 * bsys, bar);
      tma_load_3d(dst + RHO, &tmr, xs, y0, s + 1, bar);
    } else {
      const long long po = pxy * (s + 1), qo = qxy * (s + 1);
#pragma unroll
      for (int kk = 0; kk < KC; kk++) {
        if (soff[kk] < 0) continue;
        const bool ok = goff[kk] >= 0 && (isr[kk] ? s <= L.ez : s <= L.nz);
        if (ok)
          __pipeline_memcpy_async(dst + soff[kk], isr[kk] ? rp + qo + goff[kk] : u + po + goff[kk], 16);
        else
          *reinterpret_cast<float4*>(dst + soff[kk]) = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      __pipeline_commit();
    }
  };
  // TMA: wait until stage s has landed (the k-th use of a slot completes phase k)
  auto wait_stage = [&](int s) {
    const uint32_t parity = ((uint32_t)(s - (z0 - 1)) / NS) & 1u;  // s >= z0 - 1
    if (!mbar_wait(&bars[(s + NS) & (NS - 1)], parity)) gave_up = true;
  };
  // xy modes of the face nodes of both columns on a staged plane (lane 0:
  // column A, lane 1: column B), and u at the two emitted nodes
  auto face = [&](const float* pl, float2 (&F)[4][3], float2 (&own)[3]) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float* p = pl + c * NPL + 2 * ty * RX + tx + ox;
      const float2 q00 = make_float2(p[0], p[RX]), q10 = make_float2(p[1], p[RX + 1]);
      const float2 q01 = make_float2(p[RX], p[2 * RX]), q11 = make_float2(p[RX + 1], p[2 * RX + 1]);
      const float2 s0 = p_add(q00, q10), d0 = p_sub(q10, q00), s1 = p_add(q01, q11), d1 = p_sub(q11, q01);
      F[0][c] = p_add(s0, s1);
      F[1][c] = p_add(d0, d1);
      F[2][c] = p_sub(s1, s0);
      F[3][c] = p_sub(d1, d0);
      own[c] = q11;
    }
  };

  if constexpr (TMA) {
    if (tid == 0) {
#pragma unroll
      for (int k = 0; k < NS; k++) mbar_init(&bars[k], 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0)
      for (int s = z0 - 1; s <= z0 - 1 + WPD; s++) issue(s);
    wait_stage(z0 - 1);
  } else {
    for (int s = z0 - 1; s <= z0 - 1 + WPD; s++) issue(s);
    __pipeline_wait_prior(WPD);
    __syncthreads();
  }
  const bool wA = tx < WTX - 1 && ex + 1 < L.nx && ey + 1 < L.ny;
  const bool wB = wA && ty < TYP - 1 && ey + 2 < L.ny;
  const float2 zero2 = make_float2(0.f, 0.f);
  float2 F[4][3], Gt[4][3], uc[3], uo[3], own[3], fo[3], po[3], ra[4], rb[4];
  uint8_t clA = 0, clB = 0;
  double pq = 0;  // with dotp: MODE 1 u . (K u); with DOT (MODE 2) f . out
  float2 zq = make_float2(0.f, 0.f);  // DOT: f . out of the two columns along the march
  face(ss + ((z0 - 1 + NS) & (NS - 1)) * SLOT, F, uc);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    Gt[q][0] = Gt[q][1] = Gt[q][2] = zero2;
    ra[q] = rb[q] = zero2;
  }
#pragma unroll
  for (int c = 0; c < 3; c++) uo[c] = own[c] = fo[c] = po[c] = zero2;

  auto emit = [&](int zo, const float* xb) {
    if (!wA) return;
    float2 acc[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      acc[c] = p_add(own[c], make_float2(xb[(0 * 3 + c) * NT + tid + 1], xb[(1 * 3 + c) * NT + tid + 1]));
      if (wB) acc[c].y += xb[(2 * 3 + c) * NT + tid + WTX] + xb[(3 * 3 + c) * NT + tid + WTX + 1];
    }
    const int n = nb0 + pxy32 * (zo + 1);  // L.nidx(ex + 1, ey + 1, zo) in 32 bits
    const bool workA = (clA & NC_ACTIVE) && !(clA & NC_SUPPORT);
    const bool workB = (clB & NC_ACTIVE) && !(clB & NC_SUPPORT);
    float2 res[3];
    if (MODE == 0) {
#pragma unroll
      for (int c = 0; c < 3; c++)
        res[c] = make_float2(fo[c].x - (workA ? acc[c].x : 0.f), fo[c].y - (workB ? acc[c].y : 0.f));
    } else if (MODE == 1) {
      const bool passA = (clA & NC_SUPPORT) != 0, passB = (clB & NC_SUPPORT) != 0;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        res[c] = make_float2(passA ? uo[c].x : (workA ? acc[c].x : 0.f), passB ? uo[c].y : (workB ? acc[c].y : 0.f));
        pq += (double)uo[c].x * (double)res[c].x;
        if (wB) pq += (double)uo[c].y * (double)res[c].y;
      }
    } else {
      // diagonal block from rho^p of the 4 columns around each node in the
      // layers below (ra) and above (rb), as in k_fine_w
      if constexpr (LEAN) {
        // u at the two nodes from plane zo, rho^p from layers zo - 1 and zo
        // (stages zo - 1 and zo stay resident until stage zo + NS is issued)
        const int base = 2 * ty * RX + tx + ox;
        const float* pu = ss + ((zo + NS) & (NS - 1)) * SLOT + base;
        const float* pa = ss + ((zo - 1 + NS) & (NS - 1)) * SLOT + RHO + base;
        const float* pb = ss + ((zo + NS) & (NS - 1)) * SLOT + RHO + base;
#pragma unroll
        for (int c = 0; c < 3; c++) uo[c] = make_float2(pu[c * NPL + RX + 1], pu[c * NPL + 2 * RX + 1]);
        ra[0] = make_float2(pa[0], pa[RX]);
        ra[1] = make_float2(pa[1], pa[RX + 1]);
        ra[2] = make_float2(pa[RX], wB ? pa[2 * RX] : 0.f);
        ra[3] = make_float2(pa[RX + 1], wB ? pa[2 * RX + 1] : 0.f);
        rb[0] = make_float2(pb[0], pb[RX]);
        rb[1] = make_float2(pb[1], pb[RX + 1]);
        rb[2] = make_float2(pb[RX], wB ? pb[2 * RX] : 0.f);
        rb[3] = make_float2(pb[RX + 1], wB ? pb[2 * RX + 1] : 0.f);
      }
      const float2 R = p_add(p_add(p_add(ra[0], ra[1]), p_add(ra[2], ra[3])), p_add(p_add(rb[0], rb[1]), p_add(rb[2], rb[3])));
      const float2 pxy_ = p_add(p_sub(p_add(ra[0], ra[3]), p_add(ra[1], ra[2])), p_sub(p_add(rb[0], rb[3]), p_add(rb[1], rb[2])));
      const float2 xlo = p_sub(p_add(ra[1], ra[3]), p_add(ra[0], ra[2])), xhi = p_sub(p_add(rb[1], rb[3]), p_add(rb[0], rb[2]));
      const float2 ylo = p_sub(p_add(ra[2], ra[3]), p_add(ra[0], ra[1])), yhi = p_sub(p_add(rb[2], rb[3]), p_add(rb[0], rb[1]));
      const float2 pxz = p_sub(xhi, xlo), pyz = p_sub(yhi, ylo);
      // D0 = [[Da, Db, Db], [Db, Da, Db], [Db, Db, Da]]: the three diagonal entries coincide
      const float2 a = p_mul(cWp[W_DA], R), b = p_mul(cWp[W_DB], pxy_), cc = p_mul(cWp[W_DB], pxz);
      const float2 d = a, e = p_mul(cWp[W_DB], pyz), g = a;
      const float2 r0 = p_sub(fo[0], acc[0]), r1 = p_sub(fo[1], acc[1]), r2 = p_sub(fo[2], acc[2]);
      const float2 A = p_sub(p_mul(d, g), p_mul(e, e)), B = p_sub(p_mul(cc, e), p_mul(b, g));
      const float2 C = p_sub(p_mul(b, e), p_mul(cc, d));
      const float2 det = p_fma(a, A, p_fma(b, B, p_mul(cc, C)));
      const float2 id = make_float2(__fdividef(omega, det.x), __fdividef(omega, det.y));
      const float2 E = p_sub(p_mul(a, g), p_mul(cc, cc)), Fm = p_sub(p_mul(b, cc), p_mul(a, e));
      const float2 I = p_sub(p_mul(a, d), p_mul(b, b));
      const float2 cc1 = make_float2(c1, c1);
      float2 dl[3];
      dl[0] = p_fma(A, r0, p_fma(B, r1, p_mul(C, r2)));
      dl[1] = p_fma(B, r0, p_fma(E, r1, p_mul(Fm, r2)));
      dl[2] = p_fma(C, r0, p_fma(Fm, r1, p_mul(I, r2)));
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const float2 v = p_fma(id, dl[c], p_fma(cc1, p_sub(uo[c], po[c]), uo[c]));
        res[c] = make_float2(workA ? v.x : 0.f, workB ? v.y : 0.f);
      }
      // DOT: this thread's share of f . out (the CG step's r . z when this
      // is the V-cycle's last sweep), summed in FP32 along the march (one
      // packed fma per component) and in FP64 across threads
      if constexpr (DOT) {
#pragma unroll
        for (int c = 0; c < 3; c++) zq = p_fma(fo[c], res[c], zq);
      }
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      out[n + c * NP] = res[c].x;
      if (wB) out[n + px + c * NP] = res[c].y;
    }
  };

  for (int z = z0 - 1; z < z1; z++) {
    // stage z + 1 has landed, the corners of plane z - 1 are visible and the
    // slot of stage z - 1 is free for refilling
    if constexpr (TMA) {
      wait_stage(z + 1);
      __syncthreads();
      if (tid == 0) issue(z + 1 + WPD);
    } else {
      __pipeline_wait_prior(WPD - 1);
      __syncthreads();
      issue(z + 1 + WPD);
    }
    if (z - 1 >= z0) emit(z - 1, sx + ((z - 1) & 1) * 12 * NT);
    if (wA && z >= z0) {
      const int n = nb0 + pxy32 * (z + 1);
      clA = L.vclass[n];
      if (wB) clB = L.vclass[n + px];
      if (MODE != 1) {
#pragma unroll
        for (int c = 0; c < 3; c++) fo[c] = make_float2(f[n + c * NP], wB ? f[n + px + c * NP] : 0.f);
        if (MODE == 2 && uprev != nullptr) {
#pragma unroll
          for (int c = 0; c < 3; c++) po[c] = make_float2(uprev[n + c * NP], wB ? uprev[n + px + c * NP] : 0.f);
        }
      }
    }
    const float* su = ss + ((z + 1 + NS) & (NS - 1)) * SLOT;
    const float* sr = ss + ((z + NS) & (NS - 1)) * SLOT + RHO;
    float2 v[8][3], un[3];
    {
      float2 Fn[4][3];
      face(su, Fn, un);
#pragma unroll
      for (int q = 0; q < 4; q++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          v[q][c] = p_add(F[q][c], Fn[q][c]);
          v[q + 4][c] = p_sub(Fn[q][c], F[q][c]);
          F[q][c] = Fn[q][c];
        }
    }
    const int ri = 2 * ty * RX + tx + ox;
    const float2 re = make_float2(sr[ri], sr[ri + RX]);
    // rho^p B: block c maps v[c ^ (1 << j)][j] to v[c ^ (1 << i)][i] (each
    // entry of v belongs to exactly one block), in the structure of cWp; the
    // constants enter each block directly, so that nothing stays live across
    // blocks
    {
      // blocks 0 and 7: o_i = rho ((A - B) in_i + B (in_0 + in_1 + in_2))
      {
        const float2 a = v[1][0], b = v[2][1], c = v[4][2];
        const float2 w = p_mul(cWp[W_B0], p_add(p_add(a, b), c));
        v[1][0] = p_mul(re, p_fma(cWp[W_A0], a, w));
        v[2][1] = p_mul(re, p_fma(cWp[W_A0], b, w));
        v[4][2] = p_mul(re, p_fma(cWp[W_A0], c, w));
      }
      {
        const float2 a = v[6][0], b = v[5][1], c = v[3][2];
        const float2 w = p_mul(cWp[W_B7], p_add(p_add(a, b), c));
        v[6][0] = p_mul(re, p_fma(cWp[W_A7], a, w));
        v[5][1] = p_mul(re, p_fma(cWp[W_A7], b, w));
        v[3][2] = p_mul(re, p_fma(cWp[W_A7], c, w));
      }
      // one-bit blocks 1, 2, 4: rho [[P, Q], [Q, P]] on the two axes outside
      // c; the output of the axis in c is zero
      {
        const float2 a = v[3][1], b = v[5][2];  // c = 1: axes 1, 2
        v[3][1] = p_mul(re, p_fma(cWp[W_Q], b, p_mul(cWp[W_P], a)));
        v[5][2] = p_mul(re, p_fma(cWp[W_Q], a, p_mul(cWp[W_P], b)));
        v[0][0] = zero2;
      }
      {
        const float2 a = v[3][0], b = v[6][2];  // c = 2: axes 0, 2
        v[3][0] = p_mul(re, p_fma(cWp[W_Q], b, p_mul(cWp[W_P], a)));
        v[6][2] = p_mul(re, p_fma(cWp[W_Q], a, p_mul(cWp[W_P], b)));
        v[0][1] = zero2;
      }
      {
        const float2 a = v[5][0], b = v[6][1];  // c = 4: axes 0, 1
        v[5][0] = p_mul(re, p_fma(cWp[W_Q], b, p_mul(cWp[W_P], a)));
        v[6][1] = p_mul(re, p_fma(cWp[W_Q], a, p_mul(cWp[W_P], b)));
        v[0][2] = zero2;
      }
      // two-bit blocks 3, 5, 6: rho R (in_a + in_b) on both axes in c, rho S on the other
      {
        const float2 w = p_mul(re, p_mul(cWp[W_R], p_add(v[2][0], v[1][1])));  // c = 3: axes 0, 1
        v[2][0] = w; v[1][1] = w; v[7][2] = p_mul(re, p_mul(cWp[W_S], v[7][2]));
      }
      {
        const float2 w = p_mul(re, p_mul(cWp[W_R], p_add(v[4][0], v[1][2])));  // c = 5: axes 0, 2
        v[4][0] = w; v[1][2] = w; v[7][1] = p_mul(re, p_mul(cWp[W_S], v[7][1]));
      }
      {
        const float2 w = p_mul(re, p_mul(cWp[W_R], p_add(v[4][1], v[2][2])));  // c = 6: axes 1, 2
        v[4][1] = w; v[2][2] = w; v[7][0] = p_mul(re, p_mul(cWp[W_S], v[7][0]));
      }
    }
    if (MODE == 2 && !LEAN) {
#pragma unroll
      for (int q = 0; q < 4; q++) ra[q] = rb[q];
      rb[0] = re;
      // lane 1 reads row 2 ty + 2, which exists for ty < TYP - 1 only
      rb[1] = make_float2(sr[ri + 1], sr[ri + RX + 1]);
      rb[2] = make_float2(sr[ri + RX], wB ? sr[ri + 2 * RX] : 0.f);
      rb[3] = make_float2(sr[ri + RX + 1], wB ? sr[ri + 2 * RX + 1] : 0.f);
    }
    float2 tot[4][3];
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int c = 0; c < 3; c++) {
        tot[q][c] = p_add(Gt[q][c], p_sub(v[q][c], v[q + 4][c]));
        Gt[q][c] = p_add(v[q][c], v[q + 4][c]);
      }
    if (z >= z0) {
      float* xb = sx + (z & 1) * 12 * NT;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const float2 e0 = p_sub(tot[0][c], tot[1][c]), e1 = p_add(tot[0][c], tot[1][c]);
        const float2 g0 = p_sub(tot[2][c], tot[3][c]), g1 = p_add(tot[2][c], tot[3][c]);
        const float2 c00 = p_sub(e0, g0), c10 = p_sub(e1, g1), c01 = p_add(e0, g0), c11 = p_add(e1, g1);
        xb[(0 * 3 + c) * NT + tid] = c01.x + c00.y;  // A (0,1) + B (0,0): node (ex, ey + 1)
        xb[(1 * 3 + c) * NT + tid] = c01.y;          // B (0,1): node (ex, ey + 2)
        xb[(2 * 3 + c) * NT + tid] = c10.x;          // A (1,0): node (ex + 1, ey)
        xb[(3 * 3 + c) * NT + tid] = c00.x;          // A (0,0): node (ex, ey)
        own[c] = make_float2(c11.x + c10.y, c11.y);  // nodes (ex + 1, ey + 1), (ex + 1, ey + 2)
      }
    }
    if constexpr (!LEAN) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        uo[c] = uc[c];
        uc[c] = un[c];
      }
    }
  }
  __syncthreads();
  emit(z1 - 1, sx + ((z1 - 1) & 1) * 12 * NT);
  if constexpr (DOT) pq = (double)zq.x + (wB ? (double)zq.y : 0.0);
  if ((MODE == 1 || DOT) && dotp != nullptr) {
    __shared__ double sred[TYP];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pq += __shfl_down_sync(0xffffffffu, pq, o);
    if (tx == 0) sred[ty] = pq;
    __syncthreads();
    if (tid == 0) {
      double t = 0;
#pragma unroll
      for (int w = 0; w < TYP; w++) t += sred[w];
      dotp[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * (blockIdx.z - bsys * nzc)) +
           (long long)bsys * gridDim.x * gridDim.y * nzc] = t;
    }
  }
  if constexpr (TMA) {
    // every issued stage was waited for; after a wait that gave up, wait
    // (bounded) once more for the copies of the last stages still in flight
    if (gave_up)
      for (int s = max(z0 - 1, z1 - NS + 1); s <= z1; s++) wait_stage(s);
  } else {
    __pipeline_wait_prior(0);
  }
}

// damped Jacobi from a zero iterate: out = omega D^-1 f (no neighbour reads)
template <typename T>
__global__ void __launch_bounds__(256) k_fine_jacobi0(const Level L, const T* __restrict__ f, T* __restrict__ out,
                                                      const T* __restrict__ rp, T omega) {
  const int bsys = blockIdx.z / L.nz;
  const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z - bsys * L.nz;
  if (x >= L.nx || y >= L.ny) return;
  const long long NP = L.NP, qx = L.qx, qxy = (long long)L.qx * L.qy;
  f += (long long)bsys * 3 * NP;
  out += (long long)bsys * 3 * NP;
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

// FP32 first Jacobi step from zero with four consecutive padded nodes per
// thread (px is a multiple of 4): f, out and the node classes move as 16-byte
// vectors, and the 20 rho^p values of the group's elements (5 per row of
// elements) as one 16-byte and one scalar load per row.  Same arithmetic, in
// the same order, as k_fine_jacobi0<float>.  Halo rows are skipped; the halo
// nodes of a group are written as zero.
__global__ void __launch_bounds__(256) k_fine_jacobi0_v4(const Level L, const float* __restrict__ f,
                                                         float* __restrict__ out, const float* __restrict__ rp,
                                                         float omega) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long NP = L.NP, px = L.px, pxy = (long long)L.px * L.py;
  const long long p0 = 4 * g;
  if (p0 >= NP) return;
  // NP < 2^31 (checked by the launcher): 32-bit divisions
  const unsigned p0u = (unsigned)p0, pxyu = (unsigned)pxy, pxu = (unsigned)px;
  const int zp = (int)(p0u / pxyu);
  const unsigned rem = p0u - (unsigned)zp * pxyu;
  const int yp = (int)(rem / pxu), xp = (int)(rem - (unsigned)yp * pxu);
  if (zp < 1 || zp > L.nz || yp < 1 || yp > L.ny) return;
  const uchar4 cl4 = *reinterpret_cast<const uchar4*>(L.vclass + p0);
  const uint8_t cls[4] = {cl4.x, cl4.y, cl4.z, cl4.w};
  bool work[4];
  bool any = false;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int x = xp + k - 1;
    work[k] = x >= 0 && x < L.nx && (cls[k] & NC_ACTIVE) && !(cls[k] & NC_SUPPORT);
    any = any || work[k];
  }
  float o[3][4];
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int k = 0; k < 4; k++) o[c][k] = 0.f;
  if (any) {
    // element rows (y-1+b, z-1+c) of the nodes' 8 elements; element x of node
    // x + a - 1 ... padded element index xp + j - 1 for j = 0..4
    const long long qx = L.qx, qxy = (long long)L.qx * L.qy;
    float rr[4][5];
#pragma unroll
    for (int row = 0; row < 4; row++) {
      const long long e = (long long)(yp - 1 + (row & 1)) * qx + (long long)(zp - 1 + (row >> 1)) * qxy;
      // padded element x index xp - 1 + j: elements x - 1 + a of node x = xp - 1 + k
      const float* rowp = rp + e + xp;
      rr[row][0] = xp > 0 ? rowp[-1] : 0.f;
      if (xp + 4 <= L.qx) {
        const float4 m = *reinterpret_cast<const float4*>(rowp);
        rr[row][1] = m.x; rr[row][2] = m.y; rr[row][3] = m.z; rr[row][4] = m.w;
      } else {
#pragma unroll
        for (int j = 1; j < 5; j++) rr[row][j] = (xp + j - 1 < L.qx) ? rowp[j - 1] : 0.f;
      }
    }
    float fv[3][4];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float4 m = *reinterpret_cast<const float4*>(f + p0 + c * NP);
      fv[c][0] = m.x; fv[c][1] = m.y; fv[c][2] = m.z; fv[c][3] = m.w;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      if (!work[k]) continue;
      float D[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int q = 0; q < 8; q++) {
        // element q of the node: (a, b, c) = (q & 1, q >> 1 & 1, q >> 2)
        const float r = rr[((q >> 1) & 1) + 2 * (q >> 2)][k + (q & 1)];
        const int vi = 7 - q;
        D[0] += r * k0<float>((vi * 3 + 0) * 24 + vi * 3 + 0);
        D[1] += r * k0<float>((vi * 3 + 0) * 24 + vi * 3 + 1);
        D[2] += r * k0<float>((vi * 3 + 0) * 24 + vi * 3 + 2);
        D[3] += r * k0<float>((vi * 3 + 1) * 24 + vi * 3 + 1);
        D[4] += r * k0<float>((vi * 3 + 1) * 24 + vi * 3 + 2);
        D[5] += r * k0<float>((vi * 3 + 2) * 24 + vi * 3 + 2);
      }
      const float r0 = fv[0][k], r1 = fv[1][k], r2 = fv[2][k];
      const float a = D[0], b = D[1], c = D[2], d = D[3], e = D[4], gg = D[5];
      const float A = d * gg - e * e, B = c * e - b * gg, C = b * e - c * d;
      const float det = a * A + b * B + c * C;
      const float id = omega / det;
      const float E = a * gg - c * c, F = b * c - a * e, I = a * d - b * b;
      o[0][k] = id * (A * r0 + B * r1 + C * r2);
      o[1][k] = id * (B * r0 + E * r1 + F * r2);
      o[2][k] = id * (C * r0 + F * r1 + I * r2);
    }
  }
#pragma unroll
  for (int c = 0; c < 3; c++)
    *reinterpret_cast<float4*>(out + p0 + c * NP) = make_float4(o[c][0], o[c][1], o[c][2], o[c][3]);
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

static inline dim3 plane_grid(const Level& l) { return dim3(cdiv(l.nx, 32), cdiv(l.ny, 8), l.nz * l.nb); }
constexpr int WTY = 8;
static inline dim3 march_grid(const Level& l) {
  return dim3(cdiv(l.nx, WTX - 1), cdiv(l.ny, WTY - 1), cdiv(l.nz, FZC) * l.nb);
}
constexpr bool kPairTMA = true;  // packed kernel stages with TMA (else cp.async)
// thread rows pty of the packed FP32 kernel (2 pty element rows; rso_autotune picks 2 or 4)
// and its z chunk of fzc node planes
static inline dim3 pair_grid(const Level& l, int pty, int fzc) {
  return dim3(cdiv(l.nx, WTX - 1), cdiv(l.ny, 2 * pty - 1), cdiv(l.nz, fzc) * l.nb);
}

template <typename T>
static inline int pcls(int c32, int c64) { return sizeof(T) == 4 ? c32 : c64; }
// thread rows of the packed kernel's CTA (2, 4 or 8; 4 unless tuned)
static inline int fine_pty(const rso_handle* h) {
  return h->tune.fine_rows == 2 || h->tune.fine_rows == 8 ? h->tune.fine_rows : 4;
}
// z chunk of the packed kernel: the tuned value, else the largest of 32, 16,
// 8, 4 planes that gives the grid at least 4 CTAs per SM (a CTA marches its
// chunk plane by plane, so small levels need short chunks to fill the GPU;
// each chunk re-reads one plane below it)
int fine_zc(const rso_handle* h) {
  const int t = h->tune.fine_zc;
  if (t == 4 || t == 8 || t == 16 || t == 32) return t;
  const Level& l = h->L[0];
  const int pty = fine_pty(h);
  int zc = kFineZcMax;
  while (zc > kFineZcMin) {
    const dim3 g = pair_grid(l, pty, zc);
    if ((long long)g.x * g.y * g.z >= 4LL * 148) break;
    zc /= 2;
  }
  return zc;
}

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// tensor maps of the packed kernel's staged arrays: u as (px, py, pz, 3 nb)
// with a 36 x (rows + 1) x 1 x 3 box, rho^p as (qx, qy, qz) with 36 x rows x 1
static rso_status pair_tensor_maps(rso_handle* h, const Level& l, const float* u, const float* rp, int rows,
                                   CUtensorMap* mu, CUtensorMap* mr) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) {
    h->err = "cuTensorMapEncodeTiled is not available from the driver";
    return RSO_ERR_CUDA;
  }
  const cuuint64_t F = sizeof(float);
  const cuuint64_t du[4] = {(cuuint64_t)l.px, (cuuint64_t)l.py, (cuuint64_t)l.pz, (cuuint64_t)(3 * l.nb)};
  const cuuint64_t su[3] = {F * l.px, F * l.px * l.py, F * (cuuint64_t)l.NP};
  const cuuint32_t bu[4] = {36, (cuuint32_t)rows + 1, 1, 3}, e4[4] = {1, 1, 1, 1};
  const cuuint64_t dr[3] = {(cuuint64_t)l.qx, (cuuint64_t)l.qy, (cuuint64_t)l.qz};
  const cuuint64_t sr[2] = {F * l.qx, F * l.qx * l.qy};
  const cuuint32_t br[3] = {36, (cuuint32_t)rows, 1};
  CUresult r1 = enc(mu, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(u), du, su, bu, e4,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  CUresult r2 = enc(mr, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(rp), dr, sr, br, e4,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r1 != CUDA_SUCCESS || r2 != CUDA_SUCCESS) {
    h->err = "tensor map encoding of the fine-level arrays failed";
    return RSO_ERR_CUDA;
  }
  return RSO_OK;
}

// fails if a staged-copy wait of the fine kernels gave up since the last call
// (never in a healthy run); resets the device-wide count
rso_status fine_stage_check(rso_handle* h) {
  unsigned int n = 0, zero = 0, gb = 0;
  RSO_CHECK_CUDA(h, cudaMemcpyFromSymbolAsync(&n, g_stage_timeouts, sizeof(n), 0, cudaMemcpyDeviceToHost, h->stream));
  if (h->gbar) RSO_CHECK_CUDA(h, cudaMemcpyAsync(&gb, h->gbar + 2, sizeof(gb), cudaMemcpyDeviceToHost, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  if (gb != 0) {
    // nothing runs on the stream now: the barrier starts afresh
    RSO_CHECK_CUDA(h, cudaMemsetAsync(h->gbar, 0, sizeof(unsigned) * 4, h->stream));
    RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
    h->err = "a grid-barrier wait of the persistent bottom kernel timed out";
    return RSO_ERR_CUDA;
  }
  if (n != 0) {
    RSO_CHECK_CUDA(h, cudaMemcpyToSymbolAsync(g_stage_timeouts, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, h->stream));
    RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
    h->err = "a staged-copy wait of the fine operator timed out";
    return RSO_ERR_CUDA;
  }
  return RSO_OK;
}

template <typename T, int MODE>
static rso_status launch_fine(rso_handle* h, const T* u, const T* f, T* out, const T* rp, double omega, int cls,
                              const char* what, double* dotp = nullptr, const T* uprev = nullptr, double c1 = 0.0,
                              float* out32 = nullptr) {
  const Level& l = h->L[0];
  if (3 * l.NP >= (1LL << 31)) {
    h->err = "fine level too large for 32-bit in-plane offsets";
    return RSO_ERR_UNSUPPORTED;
  }
  // the kernel stages 16-byte chunks: both arrays must start on 16 bytes
  if ((reinterpret_cast<uintptr_t>(u) | reinterpret_cast<uintptr_t>(rp)) & 15) {
    h->err = "fine operator inputs must be 16-byte aligned";
    return RSO_ERR_INVALID_ARG;
  }
  // FP32: two columns per thread on packed pairs, staged by TMA; FP64: one
  // column per thread, staged by cp.async
  constexpr bool packed = sizeof(T) == 4;
  const int pty = fine_pty(h);
  const int smem = packed ? (pty == 2   ? pair_smem_bytes<2>(pair_slots(MODE, kPairTMA))
                             : pty == 8 ? pair_smem_bytes<8>(pair_slots(MODE, kPairTMA))
                                        : pair_smem_bytes<4>(pair_slots(MODE, kPairTMA)))
                          : walsh_smem_bytes<T, WTY>();
  // MODE 2 with dotp: the instantiation that also sums f . out
  const bool jdot = MODE == 2 && dotp != nullptr;
  const void* kern;
  if constexpr (packed) {
    if (jdot)
      kern = pty == 2   ? reinterpret_cast<const void*>(k_fine_p<MODE, 2, kPairTMA, true>)
             : pty == 8 ? reinterpret_cast<const void*>(k_fine_p<MODE, 8, kPairTMA, true>)
                        : reinterpret_cast<const void*>(k_fine_p<MODE, 4, kPairTMA, true>);
    else
      kern = pty == 2   ? reinterpret_cast<const void*>(k_fine_p<MODE, 2, kPairTMA>)
             : pty == 8 ? reinterpret_cast<const void*>(k_fine_p<MODE, 8, kPairTMA>)
                        : reinterpret_cast<const void*>(k_fine_p<MODE, 4, kPairTMA>);
  } else if (MODE == 0 && out32 != nullptr) {
    kern = reinterpret_cast<const void*>(k_fine_w<T, MODE, WTY, true>);
  } else {
    kern = reinterpret_cast<const void*>(k_fine_w<T, MODE, WTY>);
  }
  // the shared-memory opt-in is per device and kernel; setting it twice from
  // racing threads is harmless, so an atomic flag per device suffices
  static std::atomic<bool> attr[3][2][64];
  const int ti = pty == 2 ? 0 : pty == 4 ? 1 : 2;
  const bool second = jdot || (MODE == 0 && out32 != nullptr);  // the instantiation with the extra outputs
  std::atomic<bool>* done = (h->device >= 0 && h->device < 64) ? &attr[ti][second ? 1 : 0][h->device] : nullptr;
  if (!done || !done->load(std::memory_order_acquire)) {
    RSO_CHECK_CUDA(h, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    if (done) done->store(true, std::memory_order_release);
  }
  if constexpr (packed) {
    const int fzc = fine_zc(h);
    CUtensorMap mu{}, mr{};
    if (kPairTMA) RSO_TRY(pair_tensor_maps(h, l, u, rp, 2 * pty, &mu, &mr));
    if (h->prof_on) prof_begin(h, cls, (double)l.nn);
    if (jdot) {
      if (pty == 2)
        k_fine_p<MODE, 2, kPairTMA, true><<<pair_grid(l, 2, fzc), dim3(WTX, 2), smem, h->stream>>>(
            l, u, f, out, rp, (float)omega, dotp, uprev, (float)c1, fzc, mu, mr);
      else if (pty == 8)
        k_fine_p<MODE, 8, kPairTMA, true><<<pair_grid(l, 8, fzc), dim3(WTX, 8), smem, h->stream>>>(
            l, u, f, out, rp, (float)omega, dotp, uprev, (float)c1, fzc, mu, mr);
      else
        k_fine_p<MODE, 4, kPairTMA, true><<<pair_grid(l, 4, fzc), dim3(WTX, 4), smem, h->stream>>>(
            l, u, f, out, rp, (float)omega, dotp, uprev, (float)c1, fzc, mu, mr);
    } else if (pty == 2)
      k_fine_p<MODE, 2, kPairTMA><<<pair_grid(l, 2, fzc), dim3(WTX, 2), smem, h->stream>>>(
          l, u, f, out, rp, (float)omega, MODE == 2 ? nullptr : dotp, uprev, (float)c1, fzc, mu, mr);
    else if (pty == 8)
      k_fine_p<MODE, 8, kPairTMA><<<pair_grid(l, 8, fzc), dim3(WTX, 8), smem, h->stream>>>(
          l, u, f, out, rp, (float)omega, MODE == 2 ? nullptr : dotp, uprev, (float)c1, fzc, mu, mr);
    else
      k_fine_p<MODE, 4, kPairTMA><<<pair_grid(l, 4, fzc), dim3(WTX, 4), smem, h->stream>>>(
          l, u, f, out, rp, (float)omega, MODE == 2 ? nullptr : dotp, uprev, (float)c1, fzc, mu, mr);
  } else {
    if (h->prof_on) prof_begin(h, cls, (double)l.nn);
    if (MODE == 0 && out32 != nullptr)
      k_fine_w<T, MODE, WTY, true><<<march_grid(l), dim3(WTX, WTY), smem, h->stream>>>(l, u, f, out, rp, (T)omega,
                                                                                       dotp, uprev, (T)c1, out32);
    else
      k_fine_w<T, MODE, WTY><<<march_grid(l), dim3(WTX, WTY), smem, h->stream>>>(
          l, u, f, out, rp, (T)omega, MODE == 0 ? nullptr : dotp, uprev, (T)c1, nullptr);
  }
  rso::note_launch();
  if (h->prof_on) prof_end(h, cls);
  return launch_check(h, what);
}

template <typename T>
rso_status fine_residual(rso_handle* h, const T* u, const T* f, T* r, const T* rp) {
  return launch_fine<T, 0>(h, u, f, r, rp, 0.0, pcls<T>(PC_FINE_RES32, PC_FINE_RES64), "fine_residual");
}
// the FP64 residual with its FP32 copy r32 and r . r (dot_dev) from the same
// pass (single system; the entries the operator does not write are left as they are)
rso_status fine_residual64_rr(rso_handle* h, const double* u, const double* f, double* r, float* r32,
                              double* dot_dev) {
  const Level& l0 = h->L[0];
  const dim3 g = march_grid(l0);
  const long long nb = (long long)g.x * g.y * g.z;
  if (l0.nb != 1 || nb > h->fpart_n) {
    h->err = "fine partial-sum buffer smaller than the grid";
    return RSO_ERR_STATE;
  }
  const rso_status st = launch_fine<double, 0>(h, u, f, r, h->rp64, 0.0, PC_FINE_RES64, "fine_residual64_rr",
                                               h->fpart, nullptr, 0.0, r32);
  if (st != RSO_OK) return st;
  return reduce_partials(h, h->fpart, (int)nb, dot_dev);
}
template <typename T>
rso_status fine_applyK(rso_handle* h, const T* u, T* f, const T* rp) {
  return launch_fine<T, 1>(h, u, u, f, rp, 0.0, pcls<T>(PC_FINE_RES32, PC_FINE_APPLYK64), "fine_applyK");
}
// f = K u and dot_dev = u . f in one pass (the CG step's p . q)
rso_status fine_applyK_dot(rso_handle* h, const double* u, double* f, const double* rp, double* dot_dev, int stride) {
  const dim3 g = march_grid(h->L[0]);
  const long long nb = (long long)g.x * g.y * g.z;  // all systems
  if (nb > h->fpart_n) {
    h->err = "fine partial-sum buffer smaller than the grid";
    return RSO_ERR_STATE;
  }
  const rso_status st = launch_fine<double, 1>(h, u, u, f, rp, 0.0, PC_FINE_APPLYK64, "fine_applyK_dot", h->fpart);
  if (st != RSO_OK) return st;
  // one sum per system: dot_dev[b] over the b-th block of partials
  return reduce_partials_batch(h, h->fpart, (int)(nb / h->L[0].nb), h->L[0].nb, dot_dev, stride);
}
// the same in FP32 on the packed kernel (the reliable-update PCG's K p);
// dot_dev[b * stride] per system of a batch
rso_status fine_applyK_dot32(rso_handle* h, const float* u, float* f, double* dot_dev, int stride) {
  const Level& l0 = h->L[0];
  const dim3 g = pair_grid(l0, fine_pty(h), fine_zc(h));
  const long long nb = (long long)g.x * g.y * g.z;  // all systems
  if (nb > h->fpart_n) {
    h->err = "fine partial-sum buffer smaller than the grid";
    return RSO_ERR_STATE;
  }
  const rso_status st = launch_fine<float, 1>(h, u, u, f, h->rp32, 0.0, PC_FINE_RES32, "fine_applyK_dot32", h->fpart);
  if (st != RSO_OK) return st;
  return reduce_partials_batch(h, h->fpart, (int)(nb / l0.nb), l0.nb, dot_dev, stride);
}
template <typename T>
rso_status fine_jacobi(rso_handle* h, const T* u_in, const T* f, T* u_out, const T* rp, double omega,
                       const T* u_prev, double c1) {
  return launch_fine<T, 2>(h, u_in, f, u_out, rp, omega, pcls<T>(PC_FINE_JAC32, PC_FINE_JAC64), "fine_jacobi", nullptr,
                           u_prev, c1);
}
// the FP32 step with dot_dev = f . u_out in the same pass; with several
// systems, system b's sum goes to dot_dev[b * stride]
rso_status fine_jacobi_dot32(rso_handle* h, const float* u_in, const float* f, float* u_out, double omega,
                             const float* u_prev, double c1, double* dot_dev, int stride) {
  const Level& l0 = h->L[0];
  const dim3 g = pair_grid(l0, fine_pty(h), fine_zc(h));
  const long long nb = (long long)g.x * g.y * g.z;  // all systems
  if (nb > h->fpart_n) {
    h->err = "fine partial-sum buffer smaller than the grid";
    return RSO_ERR_STATE;
  }
  const rso_status st = launch_fine<float, 2>(h, u_in, f, u_out, h->rp32, omega, PC_FINE_JAC32, "fine_jacobi_dot32",
                                              h->fpart, u_prev, c1);
  if (st != RSO_OK) return st;
  if (l0.nb == 1) return reduce_partials(h, h->fpart, (int)nb, dot_dev);
  return reduce_partials_batch(h, h->fpart, (int)(nb / l0.nb), l0.nb, dot_dev, stride);
}
template <typename T>
rso_status fine_jacobi0(rso_handle* h, const T* f, T* u_out, const T* rp, double omega) {
  const Level& l = h->L[0];
  if (sizeof(T) == 4 && l.nb == 1 && l.NP < (1LL << 31)) {
    k_fine_jacobi0_v4<<<cdiv(l.NP / 4, 256), 256, 0, h->stream>>>(l, (const float*)f, (float*)u_out,
                                                                 (const float*)rp, (float)omega);
    rso::note_launch();
    return launch_check(h, "fine_jacobi0");
  }
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
template rso_status fine_jacobi<double>(rso_handle*, const double*, const double*, double*, const double*, double,
                                        const double*, double);
template rso_status fine_jacobi<float>(rso_handle*, const float*, const float*, float*, const float*, double,
                                       const float*, double);
template rso_status fine_jacobi0<double>(rso_handle*, const double*, double*, const double*, double);
template rso_status fine_jacobi0<float>(rso_handle*, const float*, float*, const float*, double);
template rso_status fine_gs<double>(rso_handle*, double*, const double*, const double*, int, int);
template rso_status fine_gs<float>(rso_handle*, float*, const float*, const float*, int, int);

}  // namespace rso
