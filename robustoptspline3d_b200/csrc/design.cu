// Design-variable maps and their adjoints on the element grid:
// compliance sensitivity, Heaviside projection, sensitivity/density filter,
// B-spline density map (forward and race-free adjoint) and the self-support
// constraint with its analytic coefficient gradient.
//
// The B-spline maps are separable.  Element centres lie on the element grid,
// so the basis values depend on one coordinate each; they are tabulated per
// axis (span index, order values and first derivatives) and the adjoint
// dC/dc_ijk = sum_e g_e Nx_i(x_e) Ny_j(y_e) Nz_k(z_e) is evaluated as three
// successive one-axis contractions (a gather per output, no atomics), instead
// of the reference's racy per-element scatter (grid/Grid.cu:3797, 3908, 8220).
#include "rso_internal.cuh"
#include <cmath>
#include <algorithm>

namespace rso {

// ---------------------------------------------------------------- sensitivity
// s_e = -p rho^(p-1) u_e^T K0 u_e (energy=0) or rho^p u_e^T K0 u_e (energy=1)
__global__ void __launch_bounds__(256) k_sensitivity(const Level L, const double* __restrict__ u,
                                                     const float* __restrict__ rho, const double* __restrict__ K0g,
                                                     double p, int energy, float* __restrict__ out) {
  __shared__ double K0[576];
  for (int i = threadIdx.x; i < 576; i += blockDim.x) K0[i] = K0g[i];
  __syncthreads();
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= L.ne) return;
  const int x = t % L.ex, y = (t / L.ex) % L.ey, z = t / ((long long)L.ex * L.ey);
  const long long e = L.eidx(x, y, z);
  if (!L.emask[e]) { out[e] = 0.f; return; }
  double ue[24];
#pragma unroll
  for (int a = 0; a < 8; a++) {
    const long long n = L.nidx(x + (a & 1), y + ((a >> 1) & 1), z + (a >> 2));
    ue[3 * a] = u[n]; ue[3 * a + 1] = u[n + L.NP]; ue[3 * a + 2] = u[n + 2 * L.NP];
  }
  double q = 0;
  for (int i = 0; i < 24; i++) {
    double s = 0;
#pragma unroll
    for (int j = 0; j < 24; j++) s += K0[i * 24 + j] * ue[j];
    q += ue[i] * s;
  }
  const double r = (double)rho[e];
  out[e] = energy ? (float)(pow(r, p) * q) : (float)(-p * pow(r, p - 1) * q);
}

rso_status sensitivity(rso_handle* h, const double* u_pad, float* sens_pad, int energy) {
  const Level& l = h->L[0];
  k_sensitivity<<<cdiv(l.ne, 256), 256, 0, h->stream>>>(l, u_pad, h->rho, h->K0_dev, h->cfg.penal, energy, sens_pad); rso::note_launch();
  return launch_check(h, "sensitivity");
}

// ---------------------------------------------------------------- Heaviside
__global__ void k_heaviside(const Level L, const float* __restrict__ in, double beta, double rmin,
                            const uint8_t* __restrict__ shell, int chain, const float* __restrict__ gin,
                            float* __restrict__ out) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= L.NQ) return;
  if (!L.emask[e]) { out[e] = 0.f; return; }
  const double eta = 0.5, den = tanh(beta * eta) + tanh(beta * (1 - eta));
  const double r = (double)in[e];
  if (chain) {
    const double t = tanh(beta * (r - eta));
    out[e] = (float)((double)gin[e] * beta * (1 - t * t) / den);
  } else {
    double v = (tanh(beta * eta) + tanh(beta * (r - eta))) / den;
    v = fmin(fmax(v, rmin), 1.0);
    if (shell && shell[e]) v = 1.0;
    out[e] = (float)v;
  }
}

rso_status heaviside(rso_handle* h, const float* in_pad, double beta, const uint8_t* shell_pad, float* out_pad) {
  const Level& l = h->L[0];
  k_heaviside<<<cdiv(l.NQ, 256), 256, 0, h->stream>>>(l, in_pad, beta, h->cfg.rho_min, shell_pad, 0, nullptr, out_pad); rso::note_launch();
  return launch_check(h, "heaviside");
}

rso_status heaviside_chain(rso_handle* h, const float* rho_pad, double beta, const float* gin, float* gout) {
  const Level& l = h->L[0];
  k_heaviside<<<cdiv(l.NQ, 256), 256, 0, h->stream>>>(l, rho_pad, beta, 0.0, nullptr, 1, gin, gout); rso::note_launch();
  return launch_check(h, "heaviside_chain");
}

// ---------------------------------------------------------------- filter
// weights w(r) = 1 - 6r^2 + 8r^3 - 3r^4, r = |d|/R, |d|^2 <= R^2, reach int(R+0.5)
struct FOff { int dx, dy, dz; double w; };

__global__ void k_filter(const Level L, const FOff* __restrict__ off, int noff, const float* __restrict__ in,
                         float* __restrict__ out, int mode, const float* __restrict__ wsum) {
  // mode 0: out = sum w in / sum w;  1: out = sum w (weight sums);  2: out = sum w in/W_n (adjoint)
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= L.ne) return;
  const int x = t % L.ex, y = (t / L.ex) % L.ey, z = t / ((long long)L.ex * L.ey);
  const long long e = L.eidx(x, y, z);
  if (!L.emask[e]) { out[e] = 0.f; return; }
  double gs = 0, ws = 0;
  for (int k = 0; k < noff; k++) {
    const int xx = x + off[k].dx, yy = y + off[k].dy, zz = z + off[k].dz;
    if (xx < 0 || yy < 0 || zz < 0 || xx >= L.ex || yy >= L.ey || zz >= L.ez) continue;
    const long long n = L.eidx(xx, yy, zz);
    if (!L.emask[n]) continue;
    const double w = off[k].w;
    ws += w;
    if (mode == 0) gs += w * (double)in[n];
    else if (mode == 2) gs += w * (double)in[n] / (double)wsum[n];
  }
  out[e] = (float)(mode == 0 ? gs / ws : (mode == 1 ? ws : gs));
}

rso_status filter(rso_handle* h, double R, const float* in_pad, float* out_pad, int adjoint) {
  const Level& l = h->L[0];
  std::vector<FOff> off;
  const int Ri = (int)(R + 0.5);
  const double R2 = R * R;
  for (int dx = -Ri; dx <= Ri; dx++)
    for (int dy = -Ri; dy <= Ri; dy++)
      for (int dz = -Ri; dz <= Ri; dz++) {
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 > R2) continue;
        const double r = std::sqrt(r2 / R2), rr = r * r;
        off.push_back({dx, dy, dz, 1 - 6 * rr + 8 * rr * r - 3 * rr * rr});
      }
  // the tap table is kept on the handle and rebuilt only when the radius changes
  if (!h->filt_taps || h->filt_radius != R) {
    if ((long long)off.size() > h->filt_cap) {
      if (h->filt_taps) RSO_CHECK_CUDA(h, cudaFree(h->filt_taps));
      h->filt_taps = nullptr;
      RSO_CHECK_CUDA(h, cudaMalloc(&h->filt_taps, sizeof(FOff) * off.size()));
      h->filt_cap = (long long)off.size();
    }
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(h->filt_taps, off.data(), sizeof(FOff) * off.size(), cudaMemcpyHostToDevice,
                                      h->stream));
    // the host table is a local vector: finish the copy before it goes away
    RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
    h->filt_radius = R;
  }
  const FOff* d_off = static_cast<const FOff*>(h->filt_taps);
  if (!adjoint) {
    k_filter<<<cdiv(l.ne, 256), 256, 0, h->stream>>>(l, d_off, (int)off.size(), in_pad, out_pad, 0, nullptr); rso::note_launch();
  } else {
    float* W = h->e_d;
    k_filter<<<cdiv(l.ne, 256), 256, 0, h->stream>>>(l, d_off, (int)off.size(), in_pad, W, 1, nullptr); rso::note_launch();
    k_filter<<<cdiv(l.ne, 256), 256, 0, h->stream>>>(l, d_off, (int)off.size(), in_pad, out_pad, 2, W); rso::note_launch();
  }
  return launch_check(h, "filter");
}

// ---------------------------------------------------------------- volume
rso_status volume(rso_handle* h, const float* rho_pad, double* vol) {
  const Level& l = h->L[0];
  RSO_TRY(sum_float(h, rho_pad, l.NQ, h->scal + 14));
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(h->h_scal + 14, h->scal + 14, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  // Grid::volumeRatio divides by the GS-padded element count (grid/Grid.cu:5642-5650)
  *vol = h->h_scal[14] / (double)h->n_gs_elements;
  return RSO_OK;
}

// ---------------------------------------------------------------- spline set-up
// first-knot index i = (int)((pos - bmin)/step) + order in float (the
// reference's span computation, grid/Grid.cu:3477-3479) and Cox-de Boor
// values / first derivatives in double (Piegl-Tiller A2.2/A2.3, the
// recursion of SplineBasisX/SplineBasisDeriX grid/Grid.cu:427-857).
__global__ void k_spline_axis(int n, int order, int nb, float bmin, float step, const float* __restrict__ knots,
                              int* __restrict__ idx, double* __restrict__ N, double* __restrict__ dN) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n) return;
  const float pos = (float)((double)((float)x * 1.0f) + 0.5);
  const int i = (int)__fdiv_rn(__fsub_rn(pos, bmin), step) + order;
  const bool inside = !(i < order || i > nb);
  idx[x] = inside ? i : -1;
  for (int j = 0; j < order; j++) { N[x * order + j] = 0; dN[x * order + j] = 0; }
  if (!inside) return;
  const int span = i - 1, p = order - 1;
  double ndu[6][6], left[6], right[6];
  ndu[0][0] = 1.0;
  const double u = (double)pos;
  for (int j = 1; j <= p; j++) {
    left[j] = u - (double)knots[span + 1 - j];
    right[j] = (double)knots[span + j] - u;
    double saved = 0.0;
    for (int r = 0; r < j; r++) {
      ndu[j][r] = right[r + 1] + left[j - r];
      const double temp = ndu[r][j - 1] / ndu[j][r];
      ndu[r][j] = saved + right[r + 1] * temp;
      saved = left[j - r] * temp;
    }
    ndu[j][j] = saved;
  }
  for (int j = 0; j <= p; j++) N[x * order + j] = ndu[j][p];
  for (int r = 0; r <= p; r++) {
    double d = 0;
    if (p >= 1) {
      if (r >= 1) d = ndu[r - 1][p - 1] / ndu[p][r - 1];
      if (r <= p - 1) d -= ndu[r][p - 1] / ndu[p][r];
      d *= p;
    }
    dN[x * order + r] = d;
  }
}

// de Boor value at an arbitrary coordinate (used by the orientation probe)
__device__ bool axis_basis(double u, int order, int nb, float bmin, float step, const float* knots, int* I,
                           double* N) {
  const float pf = (float)u;
  const int i = (int)__fdiv_rn(__fsub_rn(pf, bmin), step) + order;
  *I = i;
  if (i < order || i > nb) return false;
  const int span = i - 1, p = order - 1;
  double left[6], right[6];
  N[0] = 1.0;
  for (int j = 1; j <= p; j++) {
    left[j] = u - (double)knots[span + 1 - j];
    right[j] = (double)knots[span + j] - u;
    double saved = 0;
    for (int r = 0; r < j; r++) {
      const double temp = N[r] / (right[r + 1] + left[j - r]);
      N[r] = saved + right[r + 1] * temp;
      saved = left[j - r] * temp;
    }
    N[j] = saved;
  }
  return true;
}

struct SplineDev {
  int order, nb0, nb1, nb2;
  float bmin0, bmin1, bmin2, step0, step1, step2;
  const float *k0, *k1, *k2;
  const int *i0, *i1, *i2;
  const double *N0, *N1, *N2, *D0, *D1, *D2;
};

static SplineDev spline_dev(rso_handle* h, const float* knots_dev) {
  const Spline& s = h->sp;
  SplineDev d;
  d.order = s.order; d.nb0 = s.nb[0]; d.nb1 = s.nb[1]; d.nb2 = s.nb[2];
  d.bmin0 = s.bmin[0]; d.bmin1 = s.bmin[1]; d.bmin2 = s.bmin[2];
  d.step0 = s.step[0]; d.step1 = s.step[1]; d.step2 = s.step[2];
  d.k0 = knots_dev; d.k1 = knots_dev + s.knots[0].size(); d.k2 = d.k1 + s.knots[1].size();
  d.i0 = s.idx[0]; d.i1 = s.idx[1]; d.i2 = s.idx[2];
  d.N0 = s.N[0]; d.N1 = s.N[1]; d.N2 = s.N[2];
  d.D0 = s.dN[0]; d.D1 = s.dN[1]; d.D2 = s.dN[2];
  return d;
}

// ---------------------------------------------------------------- spline forward
__global__ void k_coeff2density(const Level L, SplineDev S, const double* __restrict__ c, double rmin,
                                const uint8_t* __restrict__ shell, float* __restrict__ out) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= L.ne) return;
  const int x = t % L.ex, y = (t / L.ex) % L.ey, z = t / ((long long)L.ex * L.ey);
  const long long e = L.eidx(x, y, z);
  if (!L.emask[e]) { out[e] = 0.f; return; }
  const int o = S.order;
  const int i = S.i0[x], j = S.i1[y], k = S.i2[z];
  double v;
  if (i < 0 || j < 0 || k < 0) {
    v = -0.2;
  } else {
    v = 0;
    const double* Nx = S.N0 + x * o;
    const double* Ny = S.N1 + y * o;
    const double* Nz = S.N2 + z * o;
    for (int cz = 0; cz < o; cz++)
      for (int cy = 0; cy < o; cy++) {
        const double wyz = Ny[cy] * Nz[cz];
        const double* row = c + (i - o) + (long long)(j - o + cy) * S.nb0 + (long long)(k - o + cz) * S.nb0 * S.nb1;
        for (int cx = 0; cx < o; cx++) v += row[cx] * Nx[cx] * wyz;
      }
  }
  v = fmin(fmax(v, rmin), 1.0);
  if (shell && shell[e]) v = 1.0;
  out[e] = (float)v;
}

rso_status coeff2density(rso_handle* h, const double* c, const uint8_t* shell_pad, float* out_pad) {
  const Level& l = h->L[0];
  if (!h->sp.order) { h->err = "spline not set up"; return RSO_ERR_STATE; }
  k_coeff2density<<<cdiv(l.ne, 256), 256, 0, h->stream>>>(l, spline_dev(h, h->sp.knots_dev), c, h->cfg.rho_min,
                                                           shell_pad, out_pad); rso::note_launch();
  return launch_check(h, "coeff2density");
}

// ---------------------------------------------------------------- separable adjoint
// stage 1: G1[a][y][z] = sum_x w(x,y,z) Bx(x)[a - i0(x) + o]   (a = basis index along x)
__global__ void k_sep1(const Level L, SplineDev S, const double* __restrict__ wpad, const float* __restrict__ wpadf,
                       int dx, const int* __restrict__ lo, const int* __restrict__ hi, double* __restrict__ G1) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long tot = (long long)S.nb0 * L.ey * L.ez;
  if (t >= tot) return;
  const int a = t % S.nb0;
  const long long yz = t / S.nb0;
  const int y = yz % L.ey, z = yz / L.ey;
  double s = 0;
  if (S.i1[y] >= 0 && S.i2[z] >= 0) {
    const int o = S.order;
    const double* B = dx ? S.D0 : S.N0;
    for (int x = lo[a]; x <= hi[a]; x++) {
      const long long e = L.eidx(x, y, z);
      const double w = wpad ? wpad[e] : (double)wpadf[e];
      if (w == 0) continue;
      s += w * B[x * o + a - S.i0[x] + o];
    }
  }
  G1[t] = s;
}
// stage 2: G2[a][b][z] = sum_y G1[a][y][z] By(y)[b - i1(y) + o]
__global__ void k_sep2(const Level L, SplineDev S, const double* __restrict__ G1, int dy, const int* __restrict__ lo,
                       const int* __restrict__ hi, double* __restrict__ G2) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long tot = (long long)S.nb0 * S.nb1 * L.ez;
  if (t >= tot) return;
  const int a = t % S.nb0, b = (t / S.nb0) % S.nb1, z = t / ((long long)S.nb0 * S.nb1);
  const int o = S.order;
  const double* B = dy ? S.D1 : S.N1;
  double s = 0;
  for (int y = lo[b]; y <= hi[b]; y++) s += G1[a + (long long)S.nb0 * (y + (long long)L.ey * z)] * B[y * o + b - S.i1[y] + o];
  G2[t] = s;
}
// stage 3: dc[a][b][c] += scale * sum_z G2[a][b][z] Bz(z)[c - i2(z) + o]
__global__ void k_sep3(const Level L, SplineDev S, const double* __restrict__ G2, int dz, const int* __restrict__ lo,
                       const int* __restrict__ hi, double scale, int accumulate, double* __restrict__ dc) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long tot = (long long)S.nb0 * S.nb1 * S.nb2;
  if (t >= tot) return;
  const int ab = t % ((long long)S.nb0 * S.nb1), c = t / ((long long)S.nb0 * S.nb1);
  const int o = S.order;
  const double* B = dz ? S.D2 : S.N2;
  double s = 0;
  for (int z = lo[c]; z <= hi[c]; z++) s += G2[ab + (long long)S.nb0 * S.nb1 * z] * B[z * o + c - S.i2[z] + o];
  dc[t] = (accumulate ? dc[t] : 0.0) + scale * s;
}


// dc (+)= scale * sum_e w_e Bx By Bz, w given as double (wd) or float (wf) padded element field
static rso_status separable_adjoint(rso_handle* h, const double* wd, const float* wf, int dx, int dy, int dz,
                                    double scale, int accumulate, double* dc) {
  const Level& l = h->L[0];
  SplineDev S = spline_dev(h, h->sp.knots_dev);
  double* G1 = h->sp.work[0];
  double* G2 = h->sp.work[1];
  const long long t1 = (long long)S.nb0 * l.ey * l.ez, t2 = (long long)S.nb0 * S.nb1 * l.ez,
                  t3 = (long long)S.nb0 * S.nb1 * S.nb2;
  int* r0 = h->sp.ranges[0];
  int* r1 = h->sp.ranges[1];
  int* r2 = h->sp.ranges[2];
  k_sep1<<<cdiv(t1, 256), 256, 0, h->stream>>>(l, S, wd, wf, dx, r0, r0 + S.nb0, G1); rso::note_launch();
  k_sep2<<<cdiv(t2, 256), 256, 0, h->stream>>>(l, S, G1, dy, r1, r1 + S.nb1, G2); rso::note_launch();
  k_sep3<<<cdiv(t3, 256), 256, 0, h->stream>>>(l, S, G2, dz, r2, r2 + S.nb2, scale, accumulate, dc); rso::note_launch();
  return launch_check(h, "separable_adjoint");
}

// element weights for the density adjoint: g on active, non-shell elements inside the spline domain
__global__ void k_mask_weights(const Level L, const float* __restrict__ g, const uint8_t* __restrict__ shell,
                               double* __restrict__ w) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= L.NQ) return;
  w[e] = (L.emask[e] && !(shell && shell[e])) ? (double)g[e] : 0.0;
}

rso_status density2coeff(rso_handle* h, const float* g_pad, const uint8_t* shell_pad, double* dc) {
  const Level& l = h->L[0];
  if (!h->sp.order) { h->err = "spline not set up"; return RSO_ERR_STATE; }
  double* w = h->sp.work[2];
  k_mask_weights<<<cdiv(l.NQ, 256), 256, 0, h->stream>>>(l, g_pad, shell_pad, w); rso::note_launch();
  return separable_adjoint(h, w, nullptr, 0, 0, 0, 1.0, 0, dc);
}

// ---------------------------------------------------------------- self-support
// Grid.cu:123-190 penalty pieces
__device__ __forceinline__ double d_H(double s, double beta) {
  const double eta = 0.5;
  return (tanh(beta * eta) + tanh(beta * (s - eta))) / (tanh(beta * eta) + tanh(beta * (1 - eta)));
}

struct SSPar {
  int mode;
  double beta, cosang, mid, sc, fpara, na, ia;
};

// pass 1: value, gradient and orientation probe per active element
__global__ void k_ss_eval(const Level L, SplineDev S, const double* __restrict__ c, SSPar P,
                          double* __restrict__ fv, double* __restrict__ gx, double* __restrict__ gy,
                          double* __restrict__ gz, float* __restrict__ dir) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= L.ne) return;
  const int x = t % L.ex, y = (t / L.ex) % L.ey, z = t / ((long long)L.ex * L.ey);
  const long long e = L.eidx(x, y, z);
  if (!L.emask[e]) { fv[e] = 0; gx[e] = gy[e] = gz[e] = 0; dir[e] = 0.f; return; }
  const int o = S.order;
  const int I = S.i0[x], J = S.i1[y], K = S.i2[z];
  const bool inside = I >= 0 && J >= 0 && K >= 0;
  double v = 0, g0 = 0, g1 = 0, g2 = 0;
  if (inside) {
    const double *N0 = S.N0 + x * o, *N1 = S.N1 + y * o, *N2 = S.N2 + z * o;
    const double *D0 = S.D0 + x * o, *D1 = S.D1 + y * o, *D2 = S.D2 + z * o;
    for (int q = 0; q < o; q++)
      for (int b = 0; b < o; b++) {
        const double* row = c + (I - o) + (long long)(J - o + b) * S.nb0 + (long long)(K - o + q) * S.nb0 * S.nb1;
        for (int a = 0; a < o; a++) {
          const double cc = row[a];
          v += cc * N0[a] * N1[b] * N2[q];
          g0 += cc * D0[a] * N1[b] * N2[q];
          g1 += cc * N0[a] * D1[b] * N2[q];
          g2 += cc * N0[a] * N1[b] * D2[q];
        }
      }
  }
  fv[e] = v; gx[e] = g0; gy[e] = g1; gz[e] = g2;
  // orientation probe 0.01 h along the gradient (grid/Grid.cu:7623-7714)
  const double pt[3] = {x + 0.5 + 0.01 * g0, y + 0.5 + 0.01 * g1, z + 0.5 + 0.01 * g2};
  int Ii[3];
  double Nb[3][6];
  bool ins = axis_basis(pt[0], o, S.nb0, S.bmin0, S.step0, S.k0, &Ii[0], Nb[0]);
  ins = ins && axis_basis(pt[1], o, S.nb1, S.bmin1, S.step1, S.k1, &Ii[1], Nb[1]);
  ins = ins && axis_basis(pt[2], o, S.nb2, S.bmin2, S.step2, S.k2, &Ii[2], Nb[2]);
  double vd = -0.1;
  if (ins) {
    vd = 0;
    for (int q = 0; q < o; q++)
      for (int b = 0; b < o; b++)
        for (int a = 0; a < o; a++)
          vd += c[(Ii[0] - o + a) + (long long)(Ii[1] - o + b) * S.nb0 + (long long)(Ii[2] - o + q) * S.nb0 * S.nb1] *
                Nb[0][a] * Nb[1][b] * Nb[2][q];
  }
  const double vv = inside ? v : -0.1;
  const double s = d_H(vv, P.beta) - d_H(vd, P.beta);
  dir[e] = s > 0 ? 1.f : -1.f;
}

// pass 2: per-element penalty, count, and the separable gradient weights
__global__ void k_ss_penalty(const Level L, SplineDev S, SSPar P, double flip, double direction,
                             const double* __restrict__ fv, const double* __restrict__ gx,
                             const double* __restrict__ gy, const double* __restrict__ gz, float* __restrict__ per,
                             double* __restrict__ wA, double* __restrict__ wZ, double* __restrict__ wX,
                             double* __restrict__ wY, float* __restrict__ down) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= L.ne) return;
  const int x = t % L.ex, y = (t / L.ex) % L.ey, z = t / ((long long)L.ex * L.ey);
  const long long e = L.eidx(x, y, z);
  wA[e] = wZ[e] = wX[e] = wY[e] = 0;
  if (!L.emask[e]) { if (per) per[e] = 0.f; down[e] = 0.f; return; }
  const double n0 = flip * gx[e], n1 = flip * gy[e], n2 = flip * gz[e];
  const double nn = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
  const double inner = n2 / nn / P.cosang;
  const bool dn = n2 < 0;
  down[e] = dn ? 1.f : 0.f;
  const double f = fv[e];
  const double nd = exp(-P.na * (f - 0.5) * (f - 0.5));
  const double dnd = -2 * P.na * (f - 0.5) * nd;
  const double ex_ = exp(-(inner - P.mid) / P.sc);
  const double ov = 2 / (1 + ex_), dov = 2 / (1 + ex_) / (1 + ex_) / P.sc * ex_;
  const double in_ = inner > 1 ? P.ia * (inner - 1) + 1 : 1, din = inner > 1 ? P.ia : 1;
  double val = 0, A = 0, B = 0;
  const int m = P.mode;
  const bool on = (m % 2 == 1) || dn;
  if (on) {
    if (m <= 1) { val = pow(inner, P.fpara); B = P.fpara * pow(inner, P.fpara - 1); }
    else if (m <= 3) { val = inner >= 1 ? P.fpara * (inner - 1) * (inner - 1) : 0; B = inner >= 1 ? 2 * P.fpara * (inner - 1) : 0; }
    else { val = nd * ov * in_; A = dnd * ov * in_; B = nd * dov * in_ + nd * ov * din; }
  }
  if (per) per[e] = (float)val;
  const bool inside = S.i0[x] >= 0 && S.i1[y] >= 0 && S.i2[z] >= 0;
  if (!inside) return;
  // dinner = al*(N N dN) + be*(dN N N) + ga*(N dN N)  (see compute_spline_bg_selfsupp_constraint_dcoeff)
  const double den = nn * nn * P.cosang;
  const double al = direction * (nn - n2 * n2 / nn) / den;
  const double be = -direction * n2 * n0 / nn / den;
  const double ga = -direction * n2 * n1 / nn / den;
  wA[e] = A;
  wZ[e] = B * al;
  wX[e] = B * be;
  wY[e] = B * ga;
}


rso_status selfsupport(rso_handle* h, const double* c, double beta, int mode, double opt_angle, double default_angle,
                       float* per_pad, double* dc, double* value, double* count, double* dirsum) {
  const Level& l = h->L[0];
  if (!h->sp.order) { h->err = "spline not set up"; return RSO_ERR_STATE; }
  SplineDev S = spline_dev(h, h->sp.knots_dev);
  SSPar P;
  P.mode = mode;
  P.beta = beta;
  P.cosang = std::cos(opt_angle);
  P.mid = std::cos(M_PI) / std::cos(default_angle);
  P.sc = (P.mid - 1) / std::log(1 / 0.004 - 1);
  P.fpara = mode <= 1 ? 8.0 : (mode <= 3 ? 10.0 : P.sc);  // p_norm, hfunction_c, adapt_sigmoid_c (grid/Grid.h:371-378)
  P.na = 200.0;
  P.ia = 15.0;
  double* fv = h->sp.work[3];
  double* gx = h->sp.work[4];
  double* gy = h->sp.work[5];
  double* gz = h->sp.work[6];
  float* dir = h->e_c;
  k_ss_eval<<<cdiv(l.ne, 256), 256, 0, h->stream>>>(l, S, c, P, fv, gx, gy, gz, dir); rso::note_launch();
  RSO_TRY(launch_check(h, "ss_eval"));
  RSO_TRY(sum_float(h, dir, l.NQ, h->scal + 13));
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(h->h_scal + 13, h->scal + 13, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  const double ds = h->h_scal[13];
  if (dirsum) *dirsum = ds;
  const double flip = ds < 0 ? -1.0 : 1.0;
  const double direction = ds > 0 ? 1.0 : -1.0;
  double* wA = h->sp.work[2];
  double* wZ = h->sp.work[7];
  double* wX = h->sp.work[8];
  double* wY = h->sp.work[9];
  float* down = h->e_d;
  float* per = per_pad ? per_pad : h->e_b;
  k_ss_penalty<<<cdiv(l.ne, 256), 256, 0, h->stream>>>(l, S, P, flip, direction, fv, gx, gy, gz, per, wA, wZ, wX, wY,
                                                        down); rso::note_launch();
  RSO_TRY(launch_check(h, "ss_penalty"));
  RSO_TRY(sum_float(h, per, l.NQ, h->scal + 12));
  RSO_TRY(sum_float(h, down, l.NQ, h->scal + 11));
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(h->h_scal + 11, h->scal + 11, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  const double sum = h->h_scal[12], ndown = h->h_scal[11];
  const double cnt = (mode % 2 == 0) ? ndown : (double)l.n_active_e;
  if (count) *count = cnt;
  double v = 0;
  if (cnt != 0) v = (mode <= 1) ? std::pow(sum / cnt, 1 / P.fpara) - 1 : sum / cnt;
  if (value) *value = v;
  if (dc) {
    const double scale = cnt == 0 ? 0.0 : 1.0 / cnt;
    RSO_TRY(separable_adjoint(h, wA, nullptr, 0, 0, 0, scale, 0, dc));
    RSO_TRY(separable_adjoint(h, wZ, nullptr, 0, 0, 1, scale, 1, dc));
    RSO_TRY(separable_adjoint(h, wX, nullptr, 1, 0, 0, scale, 1, dc));
    RSO_TRY(separable_adjoint(h, wY, nullptr, 0, 1, 0, scale, 1, dc));
  }
  return RSO_OK;
}

// knot series (grid/Grid.cpp:3307-3431, float arithmetic as the reference):
// the box [0, e] is enlarged by 2*e/(P+1) on both sides, step = (max-min)/(P+1),
// 'order' repeated end knots, n_basis = order + P.
rso_status spline_setup(rso_handle* h, int order, int px, int py, int pz) {
  if (order < 2 || order > 5 || px < 0 || py < 0 || pz < 0) return RSO_ERR_INVALID_ARG;
  Spline& s = h->sp;
  const Level& l = h->L[0];
  for (int a = 0; a < 3; a++) {
    cudaFree(s.idx[a]); cudaFree(s.N[a]); cudaFree(s.dN[a]); cudaFree(s.ranges[a]);
  }
  cudaFree(s.knots_dev);
  for (auto& p : s.work) { cudaFree(p); p = nullptr; }
  s.order = order;
  s.part[0] = px; s.part[1] = py; s.part[2] = pz;
  const int edim[3] = {l.ex, l.ey, l.ez};
  std::vector<float> allk;
  for (int a = 0; a < 3; a++) {
    const int P = s.part[a];
    s.nb[a] = order + P;
    float mn = 0.0f, mx = (float)edim[a];
    const float delta = mx - mn, scale_bound = 2.0f;
    mx += scale_bound * delta / (float)(P + 1);
    mn -= scale_bound * delta / (float)(P + 1);
    s.bmin[a] = mn; s.bmax[a] = mx;
    s.step[a] = (mx - mn) / (float)(P + 1);
    auto& K = s.knots[a];
    K.clear();
    float tmp = mn;
    for (int i = 0; i < order; i++) K.push_back(mn);
    for (int i = order; i < order + P; i++) { tmp += s.step[a]; K.push_back(tmp); }
    for (int i = order + P; i < 2 * order + P; i++) K.push_back(mx);
    allk.insert(allk.end(), K.begin(), K.end());
  }
  RSO_CHECK_CUDA(h, cudaMalloc(&s.knots_dev, sizeof(float) * allk.size()));
  RSO_CHECK_CUDA(h, cudaMemcpy(s.knots_dev, allk.data(), sizeof(float) * allk.size(), cudaMemcpyHostToDevice));
  size_t koff = 0;
  for (int a = 0; a < 3; a++) {
    const int n = edim[a];
    RSO_CHECK_CUDA(h, cudaMalloc(&s.idx[a], sizeof(int) * n));
    RSO_CHECK_CUDA(h, cudaMalloc(&s.N[a], sizeof(double) * n * order));
    RSO_CHECK_CUDA(h, cudaMalloc(&s.dN[a], sizeof(double) * n * order));
    k_spline_axis<<<cdiv(n, 128), 128, 0, h->stream>>>(n, order, s.nb[a], s.bmin[a], s.step[a], s.knots_dev + koff,
                                                        s.idx[a], s.N[a], s.dN[a]); rso::note_launch();
    RSO_TRY(launch_check(h, "spline_axis"));
    koff += s.knots[a].size();
    s.h_idx[a].resize(n);
    s.h_N[a].resize((size_t)n * order);
    s.h_dN[a].resize((size_t)n * order);
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(s.h_idx[a].data(), s.idx[a], sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream));
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(s.h_N[a].data(), s.N[a], sizeof(double) * n * order, cudaMemcpyDeviceToHost, h->stream));
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(s.h_dN[a].data(), s.dN[a], sizeof(double) * n * order, cudaMemcpyDeviceToHost, h->stream));
    RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
    // support ranges of every basis function along this axis
    std::vector<int> rg(2 * s.nb[a]);
    for (int b = 0; b < s.nb[a]; b++) { rg[b] = 0; rg[s.nb[a] + b] = -1; }
    std::vector<bool> seen(s.nb[a], false);
    for (int x = 0; x < n; x++) {
      const int i = s.h_idx[a][x];
      if (i < 0) continue;
      for (int b = i - order; b < i; b++) {
        if (!seen[b]) { rg[b] = x; seen[b] = true; }
        rg[s.nb[a] + b] = x;
      }
    }
    RSO_CHECK_CUDA(h, cudaMalloc(&s.ranges[a], sizeof(int) * rg.size()));
    RSO_CHECK_CUDA(h, cudaMemcpy(s.ranges[a], rg.data(), sizeof(int) * rg.size(), cudaMemcpyHostToDevice));
  }
  s.n_coeff = (long long)s.nb[0] * s.nb[1] * s.nb[2];
  RSO_CHECK_CUDA(h, cudaMalloc(&s.work[0], sizeof(double) * (size_t)s.nb[0] * l.ey * l.ez));
  RSO_CHECK_CUDA(h, cudaMalloc(&s.work[1], sizeof(double) * (size_t)s.nb[0] * s.nb[1] * l.ez));
  for (int i = 2; i < 10; i++) {
    RSO_CHECK_CUDA(h, cudaMalloc(&s.work[i], sizeof(double) * l.NQ));
    RSO_CHECK_CUDA(h, cudaMemset(s.work[i], 0, sizeof(double) * l.NQ));
  }
  cudaFree(h->coef_a); cudaFree(h->coef_b); cudaFree(h->coef_c);
  RSO_CHECK_CUDA(h, cudaMalloc(&h->coef_a, sizeof(double) * s.n_coeff));
  RSO_CHECK_CUDA(h, cudaMalloc(&h->coef_b, sizeof(double) * s.n_coeff));
  RSO_CHECK_CUDA(h, cudaMalloc(&h->coef_c, sizeof(double) * s.n_coeff));
  return RSO_OK;
}

}  // namespace rso
