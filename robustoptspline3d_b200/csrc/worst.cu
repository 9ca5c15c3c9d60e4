// Worst-case load machinery: admissible-load projection on the load nodes,
// Lanczos for lambda_max of P K^-1 P with full FP64 reorthogonalisation
// (each step one multigrid solve; classical Gram-Schmidt twice on the
// device), and the reference's modified power method.
#include "rso_internal.cuh"
#include <cmath>
#include <vector>

namespace rso {

// gather the load-node forces into a load-space vector (3 per load node),
// optionally keeping only the component along the load normal
// (forceProject: f -= Nd^T Nd f, optimization/projection.cpp:289-360)
__global__ void k_gather_load(const double* __restrict__ f, long long NP, const int* __restrict__ nodes,
                              const double* __restrict__ nrm, int nl, int cf, double* __restrict__ v) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nl) return;
  const long long n = nodes[k];
  double a = f[n], b = f[n + NP], c = f[n + 2 * NP];
  if (cf) {
    const double s = a * nrm[3 * k] + b * nrm[3 * k + 1] + c * nrm[3 * k + 2];
    a = s * nrm[3 * k]; b = s * nrm[3 * k + 1]; c = s * nrm[3 * k + 2];
  }
  v[3 * k] = a; v[3 * k + 1] = b; v[3 * k + 2] = c;
}

__global__ void k_scatter_load(const double* __restrict__ v, const int* __restrict__ nodes, int nl, long long NP,
                               double a, double* __restrict__ f) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nl) return;
  const long long n = nodes[k];
  f[n] += a * v[3 * k]; f[n + NP] += a * v[3 * k + 1]; f[n + 2 * NP] += a * v[3 * k + 2];
}

// Reorthogonalisation against all previous Lanczos vectors on the device:
// classical Gram-Schmidt applied twice ("twice is enough"), so a Lanczos step
// needs one host synchronisation instead of one per previous vector.
// s[j] = V_j . w for j < nj, partial sums in a fixed order (reproducible).
constexpr int MD_PARTS = 32, MD_THREADS = 256, MD_MAX = 128;
__global__ void __launch_bounds__(MD_THREADS) k_multi_dot_part(const double* __restrict__ V, long long ls,
                                                               const double* __restrict__ w,
                                                               double* __restrict__ part) {
  const int j = blockIdx.y;
  const double* v = V + ls * j;
  double s = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ls; i += (long long)gridDim.x * blockDim.x)
    s += v[i] * w[i];
  __shared__ double ws[MD_THREADS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
#pragma unroll
    for (int k = 0; k < MD_THREADS / 32; k++) t += ws[k];
    part[j * MD_PARTS + blockIdx.x] = t;
  }
}
__global__ void k_multi_dot_final(const double* __restrict__ part, int nj, double* __restrict__ s) {
  const int j = threadIdx.x;
  if (j >= nj) return;
  double t = 0;
  for (int p = 0; p < MD_PARTS; p++) t += part[j * MD_PARTS + p];
  s[j] = t;
}
// w -= sum_j s[j] V_j
__global__ void k_multi_axpy(const double* __restrict__ V, long long ls, int nj, const double* __restrict__ s,
                             double* __restrict__ w) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= ls) return;
  double acc = w[i];
  for (int j = 0; j < nj; j++) acc -= s[j] * V[ls * j + i];
  w[i] = acc;
}

static rso_status reorthogonalise(rso_handle* h, const double* V, long long ls, int nj, double* w, double* part,
                                  double* s) {
  k_multi_dot_part<<<dim3(MD_PARTS, nj), MD_THREADS, 0, h->stream>>>(V, ls, w, part); note_launch();
  k_multi_dot_final<<<1, MD_MAX, 0, h->stream>>>(part, nj, s); note_launch();
  k_multi_axpy<<<cdiv(ls, 256), 256, 0, h->stream>>>(V, ls, nj, s, w); note_launch();
  return launch_check(h, "reorthogonalise");
}

__global__ void k_rand_load(double* v, int nl, uint64_t seed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 3 * nl) v[i] = rso_urand(seed, (uint64_t)i);
}

__global__ void k_project_ls(double* v, const double* __restrict__ nrm, int nl) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nl) return;
  const double s = v[3 * k] * nrm[3 * k] + v[3 * k + 1] * nrm[3 * k + 1] + v[3 * k + 2] * nrm[3 * k + 2];
  v[3 * k] = s * nrm[3 * k]; v[3 * k + 1] = s * nrm[3 * k + 1]; v[3 * k + 2] = s * nrm[3 * k + 2];
}

// worst-case scratch of at least n doubles, kept on the handle (grown with a
// synchronous reallocation, so loops that reuse it allocate nothing)
static rso_status wc_scratch(rso_handle* h, size_t n, double** out) {
  if (h->wc_cap < n) {
    RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
    cudaFree(h->wc_buf);
    h->wc_buf = nullptr;
    h->wc_cap = 0;
    RSO_CHECK_CUDA(h, cudaMalloc(&h->wc_buf, sizeof(double) * n));
    h->wc_cap = n;
  }
  *out = h->wc_buf;
  return RSO_OK;
}

// the projection vector lives in the last 3 n_load entries of the worst-case
// scratch (the modified power method keeps its two vectors in front of it)
rso_status force_project(rso_handle* h, double* f, int cf) {
  const Level& l = h->L[0];
  const int nl = h->n_load;
  const size_t ls = (size_t)3 * (nl > 0 ? nl : 1);
  if (h->wc_cap < 3 * ls) {
    double* b = nullptr;
    RSO_TRY(wc_scratch(h, 3 * ls, &b));
  }
  double* v = h->wc_buf + 2 * ls;
  if (nl) { k_gather_load<<<cdiv(nl, 128), 128, 0, h->stream>>>(f, l.NP, h->load_nodes, h->load_normals, nl, cf, v); rso::note_launch(); }
  RSO_TRY(rigid_project_load(h, v, cf));  // support-free problems: f -= Rd Rd^T f
  RSO_CHECK_CUDA(h, cudaMemsetAsync(f, 0, sizeof(double) * 3 * l.NP, h->stream));
  if (nl) { k_scatter_load<<<cdiv(nl, 128), 128, 0, h->stream>>>(v, h->load_nodes, nl, l.NP, 1.0, f); rso::note_launch(); }
  return launch_check(h, "force_project");
}

// symmetric tridiagonal eigenproblem of the Lanczos matrix (tiny, host)
static void tri_eig(int m, const std::vector<double>& al, const std::vector<double>& be, std::vector<double>& w,
                    std::vector<double>& V) {
  std::vector<double> A((size_t)m * m, 0.0);
  for (int i = 0; i < m; i++) {
    A[(size_t)i * m + i] = al[i];
    if (i + 1 < m) A[(size_t)i * m + i + 1] = A[(size_t)(i + 1) * m + i] = be[i];
  }
  V.assign((size_t)m * m, 0.0);
  for (int i = 0; i < m; i++) V[(size_t)i * m + i] = 1;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0;
    for (int i = 0; i < m; i++)
      for (int j = i + 1; j < m; j++) off += A[(size_t)i * m + j] * A[(size_t)i * m + j];
    if (off < 1e-30) break;
    for (int p = 0; p < m; p++)
      for (int q = p + 1; q < m; q++) {
        const double apq = A[(size_t)p * m + q];
        if (std::fabs(apq) < 1e-300) continue;
        const double th = (A[(size_t)q * m + q] - A[(size_t)p * m + p]) / (2 * apq);
        const double t = (th >= 0 ? 1 : -1) / (std::fabs(th) + std::sqrt(th * th + 1));
        const double c = 1 / std::sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < m; k++) {
          const double akp = A[(size_t)k * m + p], akq = A[(size_t)k * m + q];
          A[(size_t)k * m + p] = c * akp - s * akq;
          A[(size_t)k * m + q] = s * akp + c * akq;
        }
        for (int k = 0; k < m; k++) {
          const double apk = A[(size_t)p * m + k], aqk = A[(size_t)q * m + k];
          A[(size_t)p * m + k] = c * apk - s * aqk;
          A[(size_t)q * m + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < m; k++) {
          const double vkp = V[(size_t)k * m + p], vkq = V[(size_t)k * m + q];
          V[(size_t)k * m + p] = c * vkp - s * vkq;
          V[(size_t)k * m + q] = s * vkp + c * vkq;
        }
      }
  }
  w.resize(m);
  for (int i = 0; i < m; i++) w[i] = A[(size_t)i * m + i];
}

rso_status worst_case(rso_handle* h, int steps, int cf, double tol, uint64_t seed, double* f_out, double* u_out,
                      double* lambda, double* ritz, int* iters) {
  const Level& l0 = h->L[0];
  const int nl = h->n_load;
  if (nl == 0) { h->err = "no load nodes"; return RSO_ERR_STATE; }
  if (steps < 1) return RSO_ERR_INVALID_ARG;
  if (steps >= MD_MAX) { h->err = "at most 127 Lanczos steps"; return RSO_ERR_INVALID_ARG; }
  const long long n3 = 3 * l0.NP;
  const long long ls = 3LL * nl;
  while ((int)h->lanczos_u.size() < steps) {
    double* p = nullptr;
    RSO_CHECK_CUDA(h, cudaMalloc(&p, sizeof(double) * n3));
    h->lanczos_u.push_back(p);
  }
  // (steps+1) load-space vectors V, the work vector wv, and the
  // reorthogonalisation scratch: partials, two coefficient vectors, (alpha, beta^2)
  double* buf = nullptr;
  RSO_TRY(wc_scratch(h, (size_t)ls * (steps + 2) + MD_MAX * MD_PARTS + 2 * MD_MAX + 2, &buf));
  double* V = buf;
  double* wv = V + (size_t)ls * (steps + 1);
  double* rw = wv + ls;
  double *part = rw, *s1 = rw + MD_MAX * MD_PARTS, *s2 = s1 + MD_MAX, *ab = s2 + MD_MAX;
  k_rand_load<<<cdiv(ls, 128), 128, 0, h->stream>>>(V, nl, seed); rso::note_launch();
  if (cf) { k_project_ls<<<cdiv(nl, 128), 128, 0, h->stream>>>(V, h->load_normals, nl); rso::note_launch(); }
  RSO_TRY(rigid_project_load(h, V, cf));
  double nv = 0;
  RSO_TRY(dot_host(h, V, V, ls, &nv));
  RSO_TRY(axpby(h, ls, 0.0, V, 1.0 / std::sqrt(nv), V));
  std::vector<double> al, be;
  int total_it = 0;
  for (int it = 0; it < steps; it++) {
    double* v = V + ls * it;
    RSO_CHECK_CUDA(h, cudaMemsetAsync(h->w, 0, sizeof(double) * n3, h->stream));
    k_scatter_load<<<cdiv(nl, 128), 128, 0, h->stream>>>(v, h->load_nodes, nl, l0.NP, 1.0, h->w); rso::note_launch();
    // support-free problems: v is free of the load set's rigid motions up to
    // rounding, which the Lanczos normalisation can magnify once beta is
    // small; the solve takes the load exactly without them
    RSO_TRY(displacement_project(h, h->w));
    double* u = h->lanczos_u[it];
    RSO_CHECK_CUDA(h, cudaMemsetAsync(u, 0, sizeof(double) * n3, h->stream));
    rso_solve_info si = {0, 0, 0};
    // high-contrast designs (void at rho_min^p = 1e-9) can need hundreds of CG steps
    RSO_TRY(solve_pcg(h, h->w, u, tol, 4000, &si, true));
    total_it += si.iterations;
    k_gather_load<<<cdiv(nl, 128), 128, 0, h->stream>>>(u, l0.NP, h->load_nodes, h->load_normals, nl, cf, wv); rso::note_launch();
    RSO_TRY(rigid_project_load(h, wv, cf));
    // alpha = v . w is the first pass's coefficient on v (the newest vector)
    RSO_TRY(reorthogonalise(h, V, ls, it + 1, wv, part, s1));
    RSO_TRY(reorthogonalise(h, V, ls, it + 1, wv, part, s2));
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(ab, s1 + it, sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    RSO_TRY(dot(h, wv, wv, ls, ab + 1));
    double hab[2];
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(hab, ab, sizeof(hab), cudaMemcpyDeviceToHost, h->stream));
    RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
    const double a = hab[0], b2 = hab[1];
    al.push_back(a);
    const double b = std::sqrt(b2);
    if (it == steps - 1 || b < 1e-14 * std::fabs(a)) break;
    be.push_back(b);
    RSO_TRY(axpby(h, ls, 1.0 / b, wv, 0.0, V + ls * (it + 1)));
  }
  const int m = (int)al.size();
  std::vector<double> w, EV;
  tri_eig(m, al, be, w, EV);
  int best = 0;
  for (int i = 1; i < m; i++) if (w[i] > w[best]) best = i;
  if (ritz) for (int i = 0; i < m; i++) ritz[i] = w[i];
  if (lambda) *lambda = w[best];
  RSO_CHECK_CUDA(h, cudaMemsetAsync(f_out, 0, sizeof(double) * n3, h->stream));
  RSO_CHECK_CUDA(h, cudaMemsetAsync(u_out, 0, sizeof(double) * n3, h->stream));
  for (int k = 0; k < m; k++) {
    const double y = EV[(size_t)k * m + best];
    k_scatter_load<<<cdiv(nl, 128), 128, 0, h->stream>>>(V + ls * k, h->load_nodes, nl, l0.NP, y, f_out); rso::note_launch();
    RSO_TRY(axpby(h, n3, y, h->lanczos_u[k], 1.0, u_out));
  }
  RSO_TRY(launch_check(h, "worst_case"));
  if (iters) *iters = total_it;
  return RSO_OK;
}

rso_status modified_pm(rso_handle* h, int cf, uint64_t seed, int max_itn, double* f, double* u, double* c_worst,
                       int* itn_out) {
  const Level& l0 = h->L[0];
  const int nl = h->n_load;
  if (nl == 0) { h->err = "no load nodes"; return RSO_ERR_STATE; }
  const long long n3 = 3 * l0.NP, ls = 3LL * nl;
  // two load-space vectors and the projection vector of force_project, kept on the handle
  double* buf = nullptr;
  RSO_TRY(wc_scratch(h, (size_t)3 * ls, &buf));
  double *fs = buf, *fs_old = buf + ls;
  k_rand_load<<<cdiv(ls, 128), 128, 0, h->stream>>>(fs, nl, seed); rso::note_launch();
  RSO_CHECK_CUDA(h, cudaMemsetAsync(f, 0, sizeof(double) * n3, h->stream));
  k_scatter_load<<<cdiv(nl, 128), 128, 0, h->stream>>>(fs, h->load_nodes, nl, l0.NP, 1.0, f); rso::note_launch();
  RSO_TRY(force_project(h, f, cf));
  double fn2 = 0;
  RSO_TRY(dot_host(h, f, f, n3, &fn2));
  RSO_TRY(axpby(h, n3, 0.0, f, 1.0 / std::sqrt(fn2), f));
  RSO_CHECK_CUDA(h, cudaMemsetAsync(u, 0, sizeof(double) * n3, h->stream));
  k_gather_load<<<cdiv(nl, 128), 128, 0, h->stream>>>(f, l0.NP, h->load_nodes, h->load_normals, nl, 0, fs_old); rso::note_launch();
  double fch = 1, rr = 1;
  int itn = 0;
  while (itn++ < max_itn && (fch > 1e-4 || rr > 1e-2)) {
    RSO_TRY(vcycle_fp64(h, u, f, 1, 1, 0, &rr));
    if (!std::isfinite(rr) || rr > 1e4) { h->err = "modified power method diverged"; return RSO_ERR_DIVERGED; }
    RSO_TRY(displacement_project(h, u));  // support-free problems (optimization.cpp:284-286)
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(f, u, sizeof(double) * n3, cudaMemcpyDeviceToDevice, h->stream));
    RSO_TRY(force_project(h, f, cf));
    RSO_TRY(dot_host(h, f, f, n3, &fn2));
    RSO_TRY(axpby(h, n3, 0.0, f, 1.0 / std::sqrt(fn2), f));
    k_gather_load<<<cdiv(nl, 128), 128, 0, h->stream>>>(f, l0.NP, h->load_nodes, h->load_normals, nl, 0, fs); rso::note_launch();
    double so = 0;
    RSO_TRY(dot_host(h, fs_old, fs_old, ls, &so));
    RSO_TRY(axpby(h, ls, 1.0, fs, -1.0, fs_old));  // fs_old <- fs - fs_old
    double d2 = 0;
    RSO_TRY(dot_host(h, fs_old, fs_old, ls, &d2));
    fch = std::sqrt(d2) / std::sqrt(so);
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(fs_old, fs, sizeof(double) * ls, cudaMemcpyDeviceToDevice, h->stream));
  }
  if (itn_out) *itn_out = itn;
  if (c_worst) RSO_TRY(dot_host(h, f, u, n3, c_worst));
  return RSO_OK;
}

}  // namespace rso

using namespace rso;

extern "C" rso_status rso_force_project(rso_handle* h, double* f, int cf) {
  if (!h || !f) return RSO_ERR_INVALID_ARG;
  RSO_TRY(pad_nodes(h, 0, f, h->w));
  RSO_TRY(force_project(h, h->w, cf));
  RSO_TRY(unpad_nodes(h, 0, h->w, f));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

// the padded worst-case force and displacement the handle keeps between calls
// (allocated by the first call that needs them, here or in a design iteration)
static rso_status worst_buffers(rso_handle* h) {
  if (h->fw) return RSO_OK;
  const long long n3 = 3 * h->L[0].NP;
  RSO_CHECK_CUDA(h, cudaMalloc(&h->fw, sizeof(double) * n3));
  RSO_CHECK_CUDA(h, cudaMalloc(&h->uw, sizeof(double) * n3));
  return RSO_OK;
}

extern "C" rso_status rso_worst_case(rso_handle* h, int steps, int cf, double tol, uint64_t seed, double* f_worst,
                                     double* u_worst, double* lambda, double* ritz) {
  if (!h || !f_worst || !u_worst || steps < 1 || !(tol > 0)) return RSO_ERR_INVALID_ARG;
  if (!h->operators_ready) { h->err = "call rso_update_operators first"; return RSO_ERR_STATE; }
  RSO_TRY(worst_buffers(h));
  double* fo = h->fw;
  double* uo = h->uw;
  rso_status s = worst_case(h, steps, cf, tol, seed, fo, uo, lambda, ritz, nullptr);
  if (s == RSO_OK) {
    RSO_TRY(unpad_nodes(h, 0, fo, f_worst));
    RSO_TRY(unpad_nodes(h, 0, uo, u_worst));
  }
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return s;
}

extern "C" rso_status rso_modified_pm(rso_handle* h, int cf, uint64_t seed, int max_itn, double* f, double* u,
                                      double* c_worst, int* itn) {
  if (!h || !f || !u || max_itn < 1) return RSO_ERR_INVALID_ARG;
  if (!h->operators_ready) { h->err = "call rso_update_operators first"; return RSO_ERR_STATE; }
  RSO_TRY(worst_buffers(h));
  double* fo = h->fw;
  double* uo = h->uw;
  rso_status s = modified_pm(h, cf, seed, max_itn, fo, uo, c_worst, itn);
  if (s == RSO_OK) {
    RSO_TRY(unpad_nodes(h, 0, fo, f));
    RSO_TRY(unpad_nodes(h, 0, uo, u));
  }
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return s;
}
