// One robust spline design iteration (the loop body of optimization_ss,
// optimization/optimization.cpp:859-1075): coefficients -> density ->
// Heaviside -> Galerkin operators -> worst-case load (Lanczos, multigrid
// solves) -> self-support constraint -> adjoint chain (sensitivity,
// Heaviside, filter, spline adjoint) -> MMA update of the coefficients.
#include "rso_internal.cuh"
#include <chrono>
#include <cmath>

namespace rso {

__global__ void k_fill_active(const Level L, float v, float* out) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e < L.NQ) out[e] = L.emask[e] ? v : 0.f;
}
__global__ void k_scale_into(long long n, double a, const double* __restrict__ x, double* __restrict__ y) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) y[i] = a * x[i];
}

static double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Objective values and unscaled coefficient gradients at coefficients c:
// h->coef_a = d lambda / dc, h->coef_c = d volume / dc, h->coef_b = d ss / dc.
struct DesignEval {
  double lambda = 0, c_worst = 0, volume = 0, ss = 0;
  int iters = 0;
  double t_ops = 0, t_worst = 0, t_ss = 0, t_adj = 0;  // ms per phase
};

static rso_status evaluate_design(rso_handle* h, const double* c, const rso_iter_params* prm, DesignEval* ev) {
  const Level& l0 = h->L[0];
  if (!h->sp.order) { h->err = "spline not set up"; return RSO_ERR_STATE; }
  const long long n3 = 3 * l0.NP;
  const bool ss = prm->ss_mode >= 0;
  if (!h->fw) {
    RSO_CHECK_CUDA(h, cudaMalloc(&h->fw, sizeof(double) * n3));
    RSO_CHECK_CUDA(h, cudaMalloc(&h->uw, sizeof(double) * n3));
  }
  const double t0 = now_ms();
  // density: spline -> clamp -> Heaviside -> clamp (Grid.cu:3428-3435, optimization.cu:336-347)
  RSO_TRY(coeff2density(h, c, nullptr, h->e_rhohat));
  RSO_TRY(heaviside(h, h->e_rhohat, prm->beta, nullptr, h->rho));
  RSO_TRY(penalise(h));
  RSO_TRY(volume(h, h->rho, &ev->volume));
  // operators (update_stencil)
  RSO_TRY(galerkin(h));
  RSO_TRY(coarsest_factor(h));
  if (h->cfg.smoother != RSO_SMOOTH_GS) RSO_TRY(estimate_lambda(h));
  h->operators_ready = true;
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  const double t1 = now_ms();
  // worst case
  RSO_TRY(worst_case(h, prm->lanczos_steps, prm->constrain_direction, prm->solve_tol, prm->seed, h->fw, h->uw,
                     &ev->lambda, nullptr, &ev->iters));
  RSO_TRY(dot_host(h, h->fw, h->uw, n3, &ev->c_worst));
  const double t2 = now_ms();
  // self-support (deal_background_points, or deal_surface_points with surface points)
  ev->ss = 0;
  if (ss && prm->ss_points > 0) {
    float box[6];
    active_box(h, box);
    RSO_TRY(surface_points(h, c, prm->ss_mc_res > 0 ? prm->ss_mc_res : 64, prm->ss_points, box, nullptr));
    RSO_TRY(surface_selfsupport(h, c, prm->beta, prm->ss_mode, prm->opt_angle, prm->default_angle, nullptr, h->coef_b,
                                &ev->ss, nullptr, nullptr));
  } else if (ss) {
    RSO_TRY(selfsupport(h, c, prm->beta, prm->ss_mode, prm->opt_angle, prm->default_angle, nullptr, h->coef_b, &ev->ss,
                        nullptr, nullptr));
    RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  }
  const double t3 = now_ms();
  // adjoint chain (computeSensitivity2, optimization.cu:249-322)
  RSO_TRY(sensitivity(h, h->uw, h->e_a, 0));
  RSO_TRY(heaviside_chain(h, h->e_rhohat, prm->beta, h->e_a, h->e_b));
  k_fill_active<<<cdiv(l0.NQ, 256), 256, 0, h->stream>>>(l0, (float)(1.0 / (double)h->n_gs_elements), h->e_c); rso::note_launch();
  RSO_TRY(heaviside_chain(h, h->e_rhohat, prm->beta, h->e_c, h->e_d));
  float* gs = h->e_b;
  float* gv = h->e_d;
  if (prm->filter_mode == 0) {
    RSO_TRY(filter(h, prm->filter_radius, h->e_b, h->e_a, 0));
    RSO_TRY(filter(h, prm->filter_radius, h->e_d, h->e_c, 0));
    gs = h->e_a;
    gv = h->e_c;
  }
  RSO_TRY(density2coeff(h, gs, nullptr, h->coef_a));
  RSO_TRY(density2coeff(h, gv, nullptr, h->coef_c));
  RSO_TRY(launch_check(h, "adjoint chain"));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  const double t4 = now_ms();
  ev->t_ops = t1 - t0; ev->t_worst = t2 - t1; ev->t_ss = t3 - t2; ev->t_adj = t4 - t3;
  return RSO_OK;
}

rso_status design_iteration(rso_handle* h, rso_mma* mma, const rso_iter_params* prm, rso_iter_info* info) {
  if (!h->sp.order) { h->err = "spline not set up"; return RSO_ERR_STATE; }
  const long long nc = h->sp.n_coeff;
  if (mma_n(mma) != nc) { h->err = "MMA size differs from the number of spline coefficients"; return RSO_ERR_INVALID_ARG; }
  const int m = mma_m(mma);
  const bool ss = prm->ss_mode >= 0;
  if (m != (ss ? 2 : 1)) { h->err = "MMA needs 1 constraint (volume) or 2 (volume, self-support)"; return RSO_ERR_INVALID_ARG; }
  if (!h->coef_df) {
    RSO_CHECK_CUDA(h, cudaMalloc(&h->coef_df, sizeof(double) * nc));
    RSO_CHECK_CUDA(h, cudaMalloc(&h->coef_dg, sizeof(double) * nc * 2));
  }
  DesignEval ev;
  RSO_TRY(evaluate_design(h, mma_x(mma), prm, &ev));
  const double t4 = now_ms();
  // driver scalings (optimization.cpp:1008-1024) and the MMA inputs
  k_scale_into<<<cdiv(nc, 256), 256, 0, h->stream>>>(nc, prm->sens_scale, h->coef_a, h->coef_df); rso::note_launch();
  k_scale_into<<<cdiv(nc, 256), 256, 0, h->stream>>>(nc, prm->vol_scale, h->coef_c, h->coef_dg); rso::note_launch();
  if (ss) { k_scale_into<<<cdiv(nc, 256), 256, 0, h->stream>>>(nc, prm->ss_scale, h->coef_b, h->coef_dg + nc); rso::note_launch(); }
  RSO_TRY(launch_check(h, "MMA inputs"));
  double g[2] = {prm->vol_scale * (ev.volume - prm->volume_ratio), prm->ss_scale * ev.ss};
  int conv = 0;
  double minfo[4];
  rso_status s = rso_mma_update(mma, h->coef_df, h->coef_dg, g, &conv, minfo);
  if (s != RSO_OK) { h->err = "MMA update failed"; return s; }
  const double t5 = now_ms();
  if (info) {
    info->c_worst = ev.c_worst; info->lambda = ev.lambda; info->volume = ev.volume; info->ss_value = ev.ss;
    info->ms_operators = ev.t_ops; info->ms_worst = ev.t_worst; info->ms_selfsupport = ev.t_ss;
    info->ms_adjoint = ev.t_adj; info->ms_mma = t5 - t4;
    info->ms_total = ev.t_ops + ev.t_worst + ev.t_ss + ev.t_adj + (t5 - t4);
    info->solve_iterations = ev.iters; info->mma_converged = conv;
  }
  return RSO_OK;
}

}  // namespace rso

using namespace rso;

extern "C" void rso_default_iter_params(rso_iter_params* p) {
  if (!p) return;
  p->beta = 8.0;
  p->volume_ratio = 0.3;
  p->filter_radius = 2.0;
  p->filter_mode = 0;
  p->lanczos_steps = 20;
  p->solve_tol = 1e-6;
  p->constrain_direction = 0;
  p->ss_mode = 4;  // overhang_ss (Grid.h:177-184)
  p->opt_angle = 0.75 * M_PI;
  p->default_angle = 0.75 * M_PI;
  p->sens_scale = 1e6;
  p->vol_scale = 1e3;
  p->ss_scale = 1e3;
  p->seed = 1234;
  p->ss_points = 0;
  p->ss_mc_res = 64;
}

extern "C" rso_status rso_design_iteration(rso_handle* h, rso_mma* mma, const rso_iter_params* prm,
                                           rso_iter_info* info) {
  if (!h || !mma || !prm) return RSO_ERR_INVALID_ARG;
  return design_iteration(h, mma, prm, info);
}

extern "C" rso_status rso_design_iteration_host(rso_handle* h, rso_mma* mma, const rso_iter_params* prm,
                                                const double* cin, double* cout, float* rho_out,
                                                rso_iter_info* info) {
  if (!h || !mma || !prm) return RSO_ERR_INVALID_ARG;
  const long long nc = h->sp.n_coeff;
  if (cin) RSO_CHECK_CUDA(h, cudaMemcpyAsync(mma_x(mma), cin, sizeof(double) * nc, cudaMemcpyHostToDevice, h->stream));
  RSO_TRY(design_iteration(h, mma, prm, info));
  if (cout) RSO_CHECK_CUDA(h, cudaMemcpy(cout, mma_x(mma), sizeof(double) * nc, cudaMemcpyDeviceToHost));
  if (rho_out) {
    float* d = h->e_a;
    RSO_TRY(unpad_elems_f(h, h->rho, d));
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(rho_out, d, sizeof(float) * h->L[0].ne, cudaMemcpyDeviceToHost, h->stream));
  }
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_design_gradient(rso_handle* h, const double* coeff_dev, const rso_iter_params* prm,
                                          double* values_host, double* dlambda_dc_dev, double* dvolume_dc_dev,
                                          double* dss_dc_dev) {
  if (!h || !coeff_dev || !prm) return RSO_ERR_INVALID_ARG;
  DesignEval ev;
  RSO_TRY(evaluate_design(h, coeff_dev, prm, &ev));
  const size_t nb = sizeof(double) * h->sp.n_coeff;
  if (dlambda_dc_dev) RSO_CHECK_CUDA(h, cudaMemcpyAsync(dlambda_dc_dev, h->coef_a, nb, cudaMemcpyDeviceToDevice, h->stream));
  if (dvolume_dc_dev) RSO_CHECK_CUDA(h, cudaMemcpyAsync(dvolume_dc_dev, h->coef_c, nb, cudaMemcpyDeviceToDevice, h->stream));
  if (dss_dc_dev) {
    if (prm->ss_mode >= 0) RSO_CHECK_CUDA(h, cudaMemcpyAsync(dss_dc_dev, h->coef_b, nb, cudaMemcpyDeviceToDevice, h->stream));
    else RSO_CHECK_CUDA(h, cudaMemsetAsync(dss_dc_dev, 0, nb, h->stream));
  }
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  if (values_host) {
    values_host[0] = ev.lambda;
    values_host[1] = ev.volume;
    values_host[2] = ev.ss;
  }
  return RSO_OK;
}
