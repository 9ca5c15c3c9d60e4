// C ABI of the design-variable maps (element fields are dense ex*ey*ez
// device arrays, coefficients dense n_coeff device arrays).
#include "rso_internal.cuh"
#include <cstring>

using namespace rso;

__global__ void k_pad_u8e(Level L, const uint8_t* __restrict__ dense, uint8_t* __restrict__ pad) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= L.ne) return;
  int x = i % L.ex, y = (i / L.ex) % L.ey, z = i / ((long long)L.ex * L.ey);
  pad[L.eidx(x, y, z)] = dense[i];
}
__global__ void k_f2d_n(const float* __restrict__ a, double* __restrict__ b, long long n) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (double)a[i];
}
__global__ void k_d2f_n(const double* __restrict__ a, float* __restrict__ b, long long n) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

// padded copy of an optional dense shell mask (NULL stays NULL), in a buffer
// the handle keeps: the first call with a mask allocates it, later calls reuse it
static rso_status pad_shell(rso_handle* h, const uint8_t* shell, uint8_t** out) {
  *out = nullptr;
  if (!shell) return RSO_OK;
  const Level& l = h->L[0];
  if (!h->shell_pad) RSO_CHECK_CUDA(h, cudaMalloc((void**)&h->shell_pad, l.NQ));
  RSO_CHECK_CUDA(h, cudaMemsetAsync(h->shell_pad, 0, l.NQ, h->stream));
  k_pad_u8e<<<cdiv(l.ne, 256), 256, 0, h->stream>>>(l, shell, h->shell_pad); rso::note_launch();
  *out = h->shell_pad;
  return launch_check(h, "pad_shell");
}

static rso_status finish(rso_handle* h, uint8_t* = nullptr) {
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_sensitivity(rso_handle* h, const double* u, float* sens) {
  if (!h || !u || !sens) return RSO_ERR_INVALID_ARG;
  RSO_TRY(pad_nodes(h, 0, u, h->L[0].u64));
  RSO_TRY(zero_support(h, h->L[0].u64));
  RSO_TRY(sensitivity(h, h->L[0].u64, h->e_a, 0));
  RSO_TRY(unpad_elems_f(h, h->e_a, sens));
  return finish(h);
}

extern "C" rso_status rso_element_energy(rso_handle* h, const double* u, float* en) {
  if (!h || !u || !en) return RSO_ERR_INVALID_ARG;
  RSO_TRY(pad_nodes(h, 0, u, h->L[0].u64));
  RSO_TRY(zero_support(h, h->L[0].u64));
  RSO_TRY(sensitivity(h, h->L[0].u64, h->e_a, 1));
  RSO_TRY(unpad_elems_f(h, h->e_a, en));
  return finish(h);
}

extern "C" rso_status rso_heaviside(rso_handle* h, const float* in, double beta, const uint8_t* shell, float* out) {
  if (!h || !in || !out) return RSO_ERR_INVALID_ARG;
  uint8_t* sh = nullptr;
  RSO_TRY(pad_shell(h, shell, &sh));
  RSO_TRY(pad_elems_f(h, in, h->e_a));
  RSO_TRY(heaviside(h, h->e_a, beta, sh, h->e_b));
  RSO_TRY(unpad_elems_f(h, h->e_b, out));
  return finish(h, sh);
}

extern "C" rso_status rso_heaviside_chain(rso_handle* h, const float* rho, double beta, const float* gin, float* gout) {
  if (!h || !rho || !gin || !gout) return RSO_ERR_INVALID_ARG;
  RSO_TRY(pad_elems_f(h, rho, h->e_a));
  RSO_TRY(pad_elems_f(h, gin, h->e_b));
  RSO_TRY(heaviside_chain(h, h->e_a, beta, h->e_b, h->e_c));
  RSO_TRY(unpad_elems_f(h, h->e_c, gout));
  return finish(h);
}

static rso_status filter_api(rso_handle* h, double R, const float* in, float* out, int adjoint) {
  if (!h || !in || !out || !(R > 0)) return RSO_ERR_INVALID_ARG;
  RSO_TRY(pad_elems_f(h, in, h->e_a));
  RSO_TRY(filter(h, R, h->e_a, h->e_b, adjoint));
  RSO_TRY(unpad_elems_f(h, h->e_b, out));
  return finish(h);
}

extern "C" rso_status rso_filter(rso_handle* h, double R, const float* in, float* out) {
  return filter_api(h, R, in, out, 0);
}
extern "C" rso_status rso_density_filter(rso_handle* h, double R, const float* in, float* out) {
  return filter_api(h, R, in, out, 0);
}
extern "C" rso_status rso_density_filter_adjoint(rso_handle* h, double R, const float* in, float* out) {
  return filter_api(h, R, in, out, 1);
}

extern "C" rso_status rso_volume(rso_handle* h, const float* rho, double* vol) {
  if (!h || !rho || !vol) return RSO_ERR_INVALID_ARG;
  RSO_TRY(pad_elems_f(h, rho, h->e_a));
  return volume(h, h->e_a, vol);
}

extern "C" rso_status rso_spline_setup(rso_handle* h, int order, int px, int py, int pz, int* n_coeff) {
  if (!h) return RSO_ERR_INVALID_ARG;
  RSO_TRY(spline_setup(h, order, px, py, pz));
  if (n_coeff) *n_coeff = (int)h->sp.n_coeff;
  return finish(h);
}

extern "C" rso_status rso_spline_axis(rso_handle* h, int axis, int* idx, double* N, double* dN) {
  if (!h || axis < 0 || axis > 2 || !h->sp.order) return RSO_ERR_INVALID_ARG;
  const Spline& s = h->sp;
  if (idx) std::memcpy(idx, s.h_idx[axis].data(), sizeof(int) * s.h_idx[axis].size());
  if (N) std::memcpy(N, s.h_N[axis].data(), sizeof(double) * s.h_N[axis].size());
  if (dN) std::memcpy(dN, s.h_dN[axis].data(), sizeof(double) * s.h_dN[axis].size());
  return RSO_OK;
}

extern "C" rso_status rso_coeff2density(rso_handle* h, const float* coeff, const uint8_t* shell, float* rho_hat) {
  if (!h || !coeff || !rho_hat) return RSO_ERR_INVALID_ARG;
  if (!h->sp.order) { h->err = "spline not set up"; return RSO_ERR_STATE; }
  uint8_t* sh = nullptr;
  RSO_TRY(pad_shell(h, shell, &sh));
  k_f2d_n<<<cdiv(h->sp.n_coeff, 256), 256, 0, h->stream>>>(coeff, h->coef_a, h->sp.n_coeff); rso::note_launch();
  RSO_TRY(coeff2density(h, h->coef_a, sh, h->e_a));
  RSO_TRY(unpad_elems_f(h, h->e_a, rho_hat));
  return finish(h, sh);
}

extern "C" rso_status rso_density2coeff_adjoint(rso_handle* h, const float* g, const uint8_t* shell, float* dc) {
  if (!h || !g || !dc) return RSO_ERR_INVALID_ARG;
  if (!h->sp.order) { h->err = "spline not set up"; return RSO_ERR_STATE; }
  uint8_t* sh = nullptr;
  RSO_TRY(pad_shell(h, shell, &sh));
  RSO_TRY(pad_elems_f(h, g, h->e_a));
  RSO_TRY(density2coeff(h, h->e_a, sh, h->coef_b));
  k_d2f_n<<<cdiv(h->sp.n_coeff, 256), 256, 0, h->stream>>>(h->coef_b, dc, h->sp.n_coeff); rso::note_launch();
  RSO_TRY(launch_check(h, "density2coeff"));
  return finish(h, sh);
}

extern "C" rso_status rso_selfsupport(rso_handle* h, const float* coeff, double beta, int mode, double opt_angle,
                                      double default_angle, float* per, float* dc, double* value, double* count,
                                      double* dirsum) {
  if (!h || !coeff || mode < 0 || mode > 5) return RSO_ERR_INVALID_ARG;
  if (!h->sp.order) { h->err = "spline not set up"; return RSO_ERR_STATE; }
  k_f2d_n<<<cdiv(h->sp.n_coeff, 256), 256, 0, h->stream>>>(coeff, h->coef_a, h->sp.n_coeff); rso::note_launch();
  RSO_TRY(selfsupport(h, h->coef_a, beta, mode, opt_angle, default_angle, h->e_a, dc ? h->coef_b : nullptr, value,
                      count, dirsum));
  if (per) RSO_TRY(unpad_elems_f(h, h->e_a, per));
  if (dc) { k_d2f_n<<<cdiv(h->sp.n_coeff, 256), 256, 0, h->stream>>>(h->coef_b, dc, h->sp.n_coeff); rso::note_launch(); }
  RSO_TRY(launch_check(h, "selfsupport"));
  return finish(h);
}
