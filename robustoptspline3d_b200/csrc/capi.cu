// C ABI: set-up, topology queries, operator and multigrid entry points.
// (design-variable, worst-case and MMA entry points live in design.cu,
// worst.cu and mma.cu.)
#include "rso_internal.cuh"
#include <cmath>
#include <cstring>
#include <new>
#include <mutex>

using namespace rso;

// ---------------------------------------------------------------- K0
// 24x24 trilinear hexahedron stiffness, 2x2x2 Gauss, isotropic D(E, nu),
// node-major xyz DOFs with local node a -> (a%2, a/2%2, a/4), scaled by
// (h/2)^3 (element/templateMatrix.cpp:31-124).
extern "C" rso_status rso_element_matrix(double E, double nu, double hh, double* K0) {
  if (!K0 || !(hh > 0) || !(nu > -1 && nu < 0.5)) return RSO_ERR_INVALID_ARG;
  double D[6][6] = {{0}};
  const double c = E / ((1 + nu) * (1 - 2 * nu));
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) D[i][j] = c * (i == j ? 1 - nu : nu);
  for (int i = 3; i < 6; i++) D[i][i] = c * (1 - 2 * nu) / 2;
  for (int i = 0; i < 576; i++) K0[i] = 0;
  const double g = std::sqrt(3.0) / 3;
  for (int q = 0; q < 8; q++) {
    const double gp[3] = {((2 * (q & 1) - 1) * g + 1) / 2, ((2 * ((q >> 1) & 1) - 1) * g + 1) / 2,
                          ((2 * (q >> 2) - 1) * g + 1) / 2};
    double dN[8][3];
    for (int a = 0; a < 8; a++) {
      const int id[3] = {a & 1, (a >> 1) & 1, a >> 2};
      double r[3];
      for (int k = 0; k < 3; k++) r[k] = id[k] ? gp[k] : 1 - gp[k];
      for (int k = 0; k < 3; k++) dN[a][k] = (id[k] ? 1.0 : -1.0) / hh * r[(k + 1) % 3] * r[(k + 2) % 3];
    }
    double B[6][24] = {{0}};
    for (int a = 0; a < 8; a++) {
      for (int k = 0; k < 3; k++) B[k][3 * a + k] = dN[a][k];
      B[3][3 * a + 1] = dN[a][2]; B[3][3 * a + 2] = dN[a][1];
      B[4][3 * a + 0] = dN[a][2]; B[4][3 * a + 2] = dN[a][0];
      B[5][3 * a + 0] = dN[a][1]; B[5][3 * a + 1] = dN[a][0];
    }
    for (int i = 0; i < 24; i++)
      for (int j = 0; j < 24; j++) {
        double s = 0;
        for (int k = 0; k < 6; k++) {
          double db = 0;
          for (int m = 0; m < 6; m++) db += D[k][m] * B[m][j];
          s += B[k][i] * db;
        }
        K0[i * 24 + j] += s;
      }
  }
  const double sc = std::pow(hh / 2, 3);
  for (int i = 0; i < 576; i++) K0[i] *= sc;
  return RSO_OK;
}

// T_pos = P_pos^T K0 P_pos for every child position of a coarsening factor F
static void galerkin_table(const double* K0, int F, std::vector<double>& T) {
  const int np = F * F * F;
  T.assign((size_t)np * 576, 0.0);
  for (int pos = 0; pos < np; pos++) {
    const int px = pos % F, py = (pos / F) % F, pz = pos / (F * F);
    double P[8][8];
    auto w = [&](int o, int A) { return A ? (double)o / F : (double)(F - o) / F; };
    for (int a = 0; a < 8; a++)
      for (int A = 0; A < 8; A++)
        P[a][A] = w(px + (a & 1), A & 1) * w(py + ((a >> 1) & 1), (A >> 1) & 1) * w(pz + (a >> 2), A >> 2);
    double KP[24][24];
    for (int r = 0; r < 24; r++)
      for (int A = 0; A < 8; A++)
        for (int j = 0; j < 3; j++) {
          double s = 0;
          for (int b = 0; b < 8; b++) s += K0[r * 24 + b * 3 + j] * P[b][A];
          KP[r][A * 3 + j] = s;
        }
    for (int A = 0; A < 8; A++)
      for (int i = 0; i < 3; i++)
        for (int c = 0; c < 24; c++) {
          double s = 0;
          for (int a = 0; a < 8; a++) s += P[a][A] * KP[a * 3 + i][c];
          T[(size_t)pos * 576 + (A * 3 + i) * 24 + c] = s;
        }
  }
}

extern "C" void rso_default_config(rso_config* c) {
  if (!c) return;
  c->youngs_modulus = 1e6;
  c->poisson_ratio = 0.3;
  c->penal = 3.0;
  c->rho_min = 1e-3;
  c->n_levels = 0;
  c->first_factor = 4;
  c->smoother = RSO_SMOOTH_JACOBI;
  c->omega = 0.6;
  c->pre = 2;
  c->post = 2;
  c->precision = RSO_MIXED;
  c->mode = RSO_WITH_SUPPORT_FREE_FORCE;
  c->cheb_lower = 0.25;
}

static void free_handle(rso_handle* h) {
  if (!h) return;
  for (auto& l : h->L) {
    cudaFree(l.emask); cudaFree(l.vclass); cudaFree(l.KE); cudaFree(l.st64); cudaFree(l.st32);
    cudaFree(l.u64); cudaFree(l.f64); cudaFree(l.r64); cudaFree(l.t64);
    cudaFree(l.u32); cudaFree(l.f32); cudaFree(l.r32); cudaFree(l.t32);
  }
  cudaFree(h->K0_dev); cudaFree(h->rho); cudaFree(h->rp32); cudaFree(h->rp64);
  cudaFree(h->load_nodes); cudaFree(h->load_normals); cudaFree(h->T1);
  cudaFree(h->efix); cudaFree(h->gfix);
  cudaFree(h->filt_taps);
  batch_release(h);
  cudaFree(h->c_nodes); cudaFree(h->c_K); cudaFree(h->c_f); cudaFree(h->c_flag);
  cudaFree(h->rigid_q); cudaFree(h->rigid_m); cudaFree(h->rigid_scr); cudaFree(h->c_R);
  cudaFree(h->red); cudaFree(h->gbar); cudaFree(h->scal); cudaFree(h->xfer); cudaFree(h->fpart);
  if (h->h_scal) cudaFreeHost(h->h_scal);
  cudaFree(h->x); cudaFree(h->r); cudaFree(h->p); cudaFree(h->q); cudaFree(h->z); cudaFree(h->w);
  cudaFree(h->stage_a); cudaFree(h->stage_b);
  for (int a = 0; a < 3; a++) {
    cudaFree(h->sp.idx[a]); cudaFree(h->sp.N[a]); cudaFree(h->sp.dN[a]); cudaFree(h->sp.ranges[a]);
  }
  cudaFree(h->sp.knots_dev);
  for (auto p : h->sp.work) cudaFree(p);
  for (auto p : h->lanczos_u) cudaFree(p);
  cudaFree(h->e_a); cudaFree(h->e_b); cudaFree(h->e_c); cudaFree(h->e_d); cudaFree(h->e_rhohat);
  cudaFree(h->shell_pad);
  cudaFree(h->coef_a); cudaFree(h->coef_b); cudaFree(h->coef_c);
  cudaFree(h->coef_df); cudaFree(h->coef_dg); cudaFree(h->fw); cudaFree(h->uw);
  cudaFree(h->wc_buf);
  vcycle_graphs_free(h);
  solve_graphs_free(h);
  surface_free(h);
  prof_free(h);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

#define ALLOC(ptr, bytes) RSO_CHECK_CUDA(h, cudaMalloc((void**)&(ptr), (bytes)))

static rso_status setup(rso_handle* h, int ex, int ey, int ez, const uint8_t* em, const uint8_t* fa,
                        const uint8_t* la, const double* ln) {
  RSO_CHECK_CUDA(h, cudaGetDevice(&h->device));
  RSO_CHECK_CUDA(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  h->own_stream = true;
  RSO_TRY(rso_element_matrix(h->cfg.youngs_modulus, h->cfg.poisson_ratio, 1.0, h->K0));
  ALLOC(h->K0_dev, sizeof(double) * 576);
  RSO_CHECK_CUDA(h, cudaMemcpy(h->K0_dev, h->K0, sizeof(double) * 576, cudaMemcpyHostToDevice));
  RSO_TRY(upload_K0(h));
  ALLOC(h->red, sizeof(double) * 4096);
  ALLOC(h->gbar, sizeof(unsigned) * 4);
  RSO_CHECK_CUDA(h, cudaMemset(h->gbar, 0, sizeof(unsigned) * 4));
  ALLOC(h->scal, sizeof(double) * 64);
  RSO_CHECK_CUDA(h, cudaMallocHost((void**)&h->h_scal, sizeof(double) * 64));
  RSO_CHECK_CUDA(h, cudaMemset(h->scal, 0, sizeof(double) * 64));
  h->L.push_back(make_level(ex, ey, ez, 0));
  RSO_TRY(build_topology(h, em, fa, la, ln));
  {
    // restriction scratch, sized once the hierarchy exists: z-filtered fine
    // columns of the largest restriction, 3 * nx * ny * nz_coarse values
    size_t xf = 1;
    for (size_t li = 1; li < h->L.size(); li++)
      xf = std::max(xf, (size_t)3 * h->L[li - 1].nx * h->L[li - 1].ny * h->L[li].nz);
    ALLOC(h->xfer, sizeof(double) * xf);
    h->xfer_n = xf;
  }
  {
    // one partial per CTA of the fine operator kernels: 31 x 7 nodes per
    // z-chunk of 32 planes (FP64), 31 x 3 or 31 x 7 (packed FP32, 2 or 4 rows)
    const Level& f0 = h->L[0];
    // the smallest fine-kernel tile: 2 thread rows (3 new element rows), z chunks of kFineZcMin planes
    h->fpart_n = (long long)cdiv(f0.nx, 31) * cdiv(f0.ny, 3) * cdiv(f0.nz, kFineZcMin);
    ALLOC(h->fpart, sizeof(double) * h->fpart_n);
  }
  // per-level buffers
  for (size_t li = 0; li < h->L.size(); li++) {
    Level& l = h->L[li];
    const size_t v64 = sizeof(double) * 3 * l.NP, v32 = sizeof(float) * 3 * l.NP;
    ALLOC(l.u64, v64); ALLOC(l.f64, v64); ALLOC(l.r64, v64); ALLOC(l.t64, v64);
    ALLOC(l.u32, v32); ALLOC(l.f32, v32); ALLOC(l.r32, v32); ALLOC(l.t32, v32);
    RSO_CHECK_CUDA(h, cudaMemset(l.u64, 0, v64)); RSO_CHECK_CUDA(h, cudaMemset(l.f64, 0, v64));
    RSO_CHECK_CUDA(h, cudaMemset(l.r64, 0, v64)); RSO_CHECK_CUDA(h, cudaMemset(l.t64, 0, v64));
    RSO_CHECK_CUDA(h, cudaMemset(l.u32, 0, v32)); RSO_CHECK_CUDA(h, cudaMemset(l.f32, 0, v32));
    RSO_CHECK_CUDA(h, cudaMemset(l.r32, 0, v32)); RSO_CHECK_CUDA(h, cudaMemset(l.t32, 0, v32));
    if (li > 0) {
      ALLOC(l.KE, sizeof(double) * 576 * l.ne);
      ALLOC(l.st64, sizeof(double) * 243 * l.NP);
      ALLOC(l.st32, sizeof(float) * st32_len(l.NP));
      RSO_CHECK_CUDA(h, cudaMemset(l.KE, 0, sizeof(double) * 576 * l.ne));
      RSO_CHECK_CUDA(h, cudaMemset(l.st64, 0, sizeof(double) * 243 * l.NP));
      RSO_CHECK_CUDA(h, cudaMemset(l.st32, 0, sizeof(float) * st32_len(l.NP)));
    }
  }
  Level& l0 = h->L[0];
  ALLOC(h->rho, sizeof(float) * l0.NQ); ALLOC(h->rp32, sizeof(float) * l0.NQ); ALLOC(h->rp64, sizeof(double) * l0.NQ);
  RSO_CHECK_CUDA(h, cudaMemset(h->rho, 0, sizeof(float) * l0.NQ));
  const size_t v64 = sizeof(double) * 3 * l0.NP;
  ALLOC(h->x, v64); ALLOC(h->r, v64); ALLOC(h->p, v64); ALLOC(h->q, v64); ALLOC(h->z, v64); ALLOC(h->w, v64);
  for (double* p : {h->x, h->r, h->p, h->q, h->z, h->w}) RSO_CHECK_CUDA(h, cudaMemset(p, 0, v64));
  ALLOC(h->e_a, sizeof(float) * l0.NQ); ALLOC(h->e_b, sizeof(float) * l0.NQ); ALLOC(h->e_c, sizeof(float) * l0.NQ);
  ALLOC(h->e_d, sizeof(float) * l0.NQ); ALLOC(h->e_rhohat, sizeof(float) * l0.NQ);
  for (float* p : {h->e_a, h->e_b, h->e_c, h->e_d, h->e_rhohat}) RSO_CHECK_CUDA(h, cudaMemset(p, 0, sizeof(float) * l0.NQ));
  // default density 1 on active elements
  {
    std::vector<float> ones(l0.ne, 1.0f);
    float* d = nullptr;
    ALLOC(d, sizeof(float) * l0.ne);
    RSO_CHECK_CUDA(h, cudaMemcpy(d, ones.data(), sizeof(float) * l0.ne, cudaMemcpyHostToDevice));
    RSO_TRY(pad_elems_f(h, d, h->rho));
    RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
    cudaFree(d);
    RSO_TRY(penalise(h));
  }
  // Galerkin table of the first coarsening
  if (h->L.size() > 1) {
    std::vector<double> T;
    galerkin_table(h->K0, h->L[1].factor, T);
    ALLOC(h->T1, sizeof(double) * T.size());
    RSO_CHECK_CUDA(h, cudaMemcpy(h->T1, T.data(), sizeof(double) * T.size(), cudaMemcpyHostToDevice));
    RSO_TRY(galerkin_setup(h));
    // coarsest node list + node->row map
    const Level& c = h->L.back();
    const std::vector<uint8_t>& cvm = h->h_vmask.back();
    std::vector<int> nodes;
    std::vector<int> crow(c.NP, -1);
    for (int z = 0; z < c.nz; z++)
      for (int y = 0; y < c.ny; y++)
        for (int x = 0; x < c.nx; x++) {
          const long long i = x + (long long)c.nx * (y + (long long)c.ny * z);
          if (!cvm[i]) continue;
          crow[c.nidx(x, y, z)] = (int)nodes.size();
          nodes.push_back((int)c.nidx(x, y, z));
        }
    h->nc = (int)nodes.size();
    if (h->nc > 4000) { h->err = "coarsest level too large for the dense solve (add levels)"; return RSO_ERR_INVALID_ARG; }
    std::vector<int> packed(nodes);
    packed.insert(packed.end(), crow.begin(), crow.end());
    ALLOC(h->c_nodes, sizeof(int) * packed.size());
    RSO_CHECK_CUDA(h, cudaMemcpy(h->c_nodes, packed.data(), sizeof(int) * packed.size(), cudaMemcpyHostToDevice));
    const size_t N = 3 * (size_t)h->nc;
    ALLOC(h->c_K, sizeof(double) * 3 * N * N);  // factor, inverse, L^-1 scratch
    ALLOC(h->c_f, sizeof(double) * N);
    ALLOC(h->c_flag, sizeof(int));
  }
  if (!h->has_support) RSO_TRY(rigid_setup(h));
  int counts[4];
  RSO_TRY(rso_ref_numbering(h, 0, counts, nullptr, nullptr, nullptr, nullptr, nullptr));
  h->n_gs_elements = counts[3];
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

static thread_local std::string g_create_err;

// K0 and its sum/difference blocks live in per-device constant memory, shared
// by every handle on the device: live handles on one device must agree on
// (E, nu).  Registry of the material of the live handles per device.
namespace {
std::mutex g_mat_mu;
struct DevMaterial { double E = 0, nu = 0; int live = 0; };
DevMaterial g_mat[64];
}  // namespace

static rso_status claim_material(rso_handle* h) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) { g_create_err = "no CUDA device"; return RSO_ERR_CUDA; }
  std::lock_guard<std::mutex> lock(g_mat_mu);
  DevMaterial& m = g_mat[dev];
  if (m.live > 0 && (m.E != h->cfg.youngs_modulus || m.nu != h->cfg.poisson_ratio)) {
    g_create_err = "another live handle on this device uses a different Young's modulus or Poisson ratio "
                   "(the element matrix is held in per-device constant memory)";
    return RSO_ERR_UNSUPPORTED;
  }
  m.E = h->cfg.youngs_modulus;
  m.nu = h->cfg.poisson_ratio;
  m.live++;
  h->material_dev = dev;
  return RSO_OK;
}

static void release_material(rso_handle* h) {
  if (h->material_dev < 0) return;
  std::lock_guard<std::mutex> lock(g_mat_mu);
  g_mat[h->material_dev].live--;
  h->material_dev = -1;
}

extern "C" rso_status rso_create(const rso_config* cfg, int ex, int ey, int ez, const uint8_t* em,
                                 const uint8_t* fa, const uint8_t* la, const double* ln, rso_handle** out) {
  if (!out || !em || ex <= 0 || ey <= 0 || ez <= 0) return RSO_ERR_INVALID_ARG;
  *out = nullptr;
  rso_handle* h = new (std::nothrow) rso_handle();
  if (!h) return RSO_ERR_OOM;
  if (cfg) h->cfg = *cfg;
  else rso_default_config(&h->cfg);
  // mixed precision runs the PCG recurrence in FP32 with true-residual
  // replacement every 1e-2 of reduction (rso_set_krylov_fp32)
  h->krylov32 = h->cfg.precision == RSO_MIXED ? 1e-2 : 0.0;
  if (h->cfg.first_factor != 2 && h->cfg.first_factor != 4) { delete h; return RSO_ERR_INVALID_ARG; }
  if (h->cfg.pre < 0 || h->cfg.post < 0 || h->cfg.penal <= 0 || h->cfg.pre > 16 || h->cfg.post > 16) {
    delete h;
    return RSO_ERR_INVALID_ARG;
  }
  if (h->cfg.smoother < RSO_SMOOTH_GS || h->cfg.smoother > RSO_SMOOTH_CHEBYSHEV) { delete h; return RSO_ERR_INVALID_ARG; }
  if (h->cfg.smoother == RSO_SMOOTH_CHEBYSHEV && !(h->cfg.cheb_lower > 0 && h->cfg.cheb_lower < 1)) {
    delete h;
    return RSO_ERR_INVALID_ARG;
  }
  if (h->cfg.mode < RSO_NO_SUPPORT_CONSTRAIN_FORCE_DIRECTION || h->cfg.mode > RSO_WITH_SUPPORT_FREE_FORCE) {
    delete h;
    return RSO_ERR_INVALID_ARG;
  }
  // support-free modes: no node is fixed (the fixed area is not read); the
  // operator is singular on the rigid motions, handled by rigid.cu
  h->has_support = h->cfg.mode == RSO_WITH_SUPPORT_CONSTRAIN_FORCE_DIRECTION ||
                   h->cfg.mode == RSO_WITH_SUPPORT_FREE_FORCE;
  if (!h->has_support) fa = nullptr;
  if (rso_status sm = claim_material(h); sm != RSO_OK) {
    delete h;
    return sm;
  }
  rso_status s = setup(h, ex, ey, ez, em, fa, la, ln);
  if (s != RSO_OK) {
    g_create_err = h->err;
    release_material(h);
    free_handle(h);
    return s;
  }
  *out = h;
  return RSO_OK;
}

extern "C" void rso_destroy(rso_handle* h) {
  if (!h) return;
  cudaStreamSynchronize(h->stream);
  release_material(h);
  free_handle(h);
}

extern "C" const char* rso_last_error(const rso_handle* h) { return h ? h->err.c_str() : g_create_err.c_str(); }

extern "C" rso_status rso_set_stream(rso_handle* h, void* stream) {
  if (!h) return RSO_ERR_INVALID_ARG;
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  if (stream) {
    if (h->own_stream) cudaStreamDestroy(h->stream);
    h->stream = (cudaStream_t)stream;
    h->own_stream = false;
  }
  return RSO_OK;
}

extern "C" rso_status rso_synchronize(rso_handle* h) {
  if (!h) return RSO_ERR_INVALID_ARG;
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" int rso_n_levels(const rso_handle* h) { return h ? (int)h->L.size() : 0; }

extern "C" rso_status rso_level_dims(const rso_handle* h, int level, int* d) {
  if (!h || !d || level < 0 || level >= (int)h->L.size()) return RSO_ERR_INVALID_ARG;
  const Level& l = h->L[level];
  d[0] = l.ex; d[1] = l.ey; d[2] = l.ez; d[3] = l.nx; d[4] = l.ny; d[5] = l.nz;
  return RSO_OK;
}

// ---------------------------------------------------------------- operator
extern "C" rso_status rso_set_density(rso_handle* h, const float* rho) {
  if (!h || !rho) return RSO_ERR_INVALID_ARG;
  RSO_TRY(pad_elems_f(h, rho, h->rho));
  RSO_TRY(penalise(h));
  h->operators_ready = false;
  return RSO_OK;
}

extern "C" rso_status rso_get_density(rso_handle* h, float* rho) {
  if (!h || !rho) return RSO_ERR_INVALID_ARG;
  RSO_TRY(unpad_elems_f(h, h->rho, rho));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_set_density_points(rso_handle* h, int n, const int32_t* pos, const float* values) {
  if (!h || n < 0 || (n > 0 && (!pos || !values))) return RSO_ERR_INVALID_ARG;
  const Level& l0 = h->L[0];
  const std::vector<uint8_t>& em = h->h_emask[0];
  std::vector<float> dense((size_t)l0.ne, 0.0f);
  for (int i = 0; i < n; i++) {
    const int x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    if (x < 0 || y < 0 || z < 0 || x >= l0.ex || y >= l0.ey || z >= l0.ez) {
      h->err = "density point outside the grid (unmatched grid and file)";
      return RSO_ERR_INVALID_ARG;
    }
    const size_t e = x + (size_t)l0.ex * (y + (size_t)l0.ey * z);
    if (!em[e]) {
      h->err = "density point on an inactive element (unmatched grid and file)";
      return RSO_ERR_INVALID_ARG;
    }
    dense[e] = values[i];
  }
  // staged in a padded element buffer of the handle (at least ex*ey*ez floats)
  float* d = h->e_b;
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(d, dense.data(), sizeof(float) * l0.ne, cudaMemcpyHostToDevice, h->stream));
  RSO_TRY(rso_set_density(h, d));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_update_operators(rso_handle* h) {
  if (!h) return RSO_ERR_INVALID_ARG;
  RSO_TRY(galerkin(h));
  RSO_TRY(coarsest_factor(h));
  if (h->cfg.smoother != RSO_SMOOTH_GS) RSO_TRY(estimate_lambda(h));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  h->operators_ready = true;
  return RSO_OK;
}

static rso_status need_ops(rso_handle* h) {
  if (!h->operators_ready) { h->err = "call rso_update_operators after rso_set_density"; return RSO_ERR_STATE; }
  return RSO_OK;
}

extern "C" rso_status rso_apply_K(rso_handle* h, const double* u, double* f) {
  if (!h || !u || !f) return RSO_ERR_INVALID_ARG;
  Level& l0 = h->L[0];
  RSO_TRY(pad_nodes(h, 0, u, l0.u64));
  RSO_TRY(zero_support(h, l0.u64));
  RSO_TRY(fine_applyK<double>(h, l0.u64, l0.r64, h->rp64));
  RSO_TRY(unpad_nodes(h, 0, l0.r64, f));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_residual(rso_handle* h, const double* u, const double* f, double* r) {
  if (!h || !u || !f || !r) return RSO_ERR_INVALID_ARG;
  Level& l0 = h->L[0];
  RSO_TRY(pad_nodes(h, 0, u, l0.u64));
  RSO_TRY(pad_nodes(h, 0, f, l0.f64));
  RSO_TRY(zero_support(h, l0.u64));
  RSO_TRY(zero_support(h, l0.f64));
  RSO_TRY(fine_residual<double>(h, l0.u64, l0.f64, l0.r64, h->rp64));
  RSO_TRY(unpad_nodes(h, 0, l0.r64, r));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_coarse_sweep_fp32(rso_handle* h, int level, int op, const double* u, const double* f,
                                            const double* uprev, double omega, double c1, double* out) {
  if (!h || !u || !f || !out || level < 1 || level >= (int)h->L.size() || (op != 0 && op != 2))
    return RSO_ERR_INVALID_ARG;
  RSO_TRY(need_ops(h));
  Level& l = h->L[level];
  const long long n3 = 3 * l.NP;
  RSO_TRY(pad_nodes(h, level, u, l.u64));
  RSO_TRY(to_f32(h, l.u64, l.u32, n3));
  RSO_TRY(pad_nodes(h, level, f, l.f64));
  RSO_TRY(to_f32(h, l.f64, l.f32, n3));
  const float* up = nullptr;
  if (uprev && op == 2) {
    RSO_TRY(pad_nodes(h, level, uprev, l.t64));
    RSO_TRY(to_f32(h, l.t64, l.t32, n3));
    up = l.t32;
  }
  if (op == 0) RSO_TRY(coarse_residual<float>(h, level, l.u32, l.f32, l.r32));
  else RSO_TRY(coarse_jacobi<float>(h, level, l.u32, l.f32, l.r32, omega, up, c1));
  RSO_TRY(to_f64(h, l.r32, l.r64, n3));
  RSO_TRY(unpad_nodes(h, level, l.r64, out));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_prolong_fp32(rso_handle* h, int cl, const double* uc, const double* uf, double* out) {
  if (!h || !uc || !uf || !out || cl < 1 || cl >= (int)h->L.size()) return RSO_ERR_INVALID_ARG;
  Level& c = h->L[cl];
  Level& f = h->L[cl - 1];
  RSO_TRY(pad_nodes(h, cl, uc, c.u64));
  RSO_TRY(to_f32(h, c.u64, c.u32, 3 * c.NP));
  RSO_TRY(pad_nodes(h, cl - 1, uf, f.u64));
  RSO_TRY(to_f32(h, f.u64, f.u32, 3 * f.NP));
  RSO_TRY(prolong<float>(h, cl, c.u32, f.u32));
  RSO_TRY(to_f64(h, f.u32, f.u64, 3 * f.NP));
  RSO_TRY(unpad_nodes(h, cl - 1, f.u64, out));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_restrict_fp32(rso_handle* h, int cl, const double* rf, double* fc) {
  if (!h || !rf || !fc || cl < 1 || cl >= (int)h->L.size()) return RSO_ERR_INVALID_ARG;
  Level& c = h->L[cl];
  Level& f = h->L[cl - 1];
  RSO_TRY(pad_nodes(h, cl - 1, rf, f.r64));
  RSO_TRY(to_f32(h, f.r64, f.r32, 3 * f.NP));
  RSO_TRY(restrict_<float>(h, cl, f.r32, c.f32));
  RSO_TRY(to_f64(h, c.f32, c.f64, 3 * c.NP));
  RSO_TRY(unpad_nodes(h, cl, c.f64, fc));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_set_vcycle_graphs(rso_handle* h, int on) {
  if (!h) return RSO_ERR_INVALID_ARG;
  h->vc_graphs = on != 0;
  return RSO_OK;
}

extern "C" rso_status rso_set_fine_zchunk(rso_handle* h, int planes) {
  if (!h || (planes != 0 && planes != 4 && planes != 8 && planes != 16 && planes != 32)) return RSO_ERR_INVALID_ARG;
  h->tune.fine_zc = planes;
  return RSO_OK;
}

extern "C" int rso_fine_zchunk(const rso_handle* h) { return h ? fine_zc(h) : 0; }

extern "C" rso_status rso_set_bottom_kernel(rso_handle* h, int kind) {
  if (!h || (kind != 0 && kind != 1)) return RSO_ERR_INVALID_ARG;
  h->tune.bottom_kind = kind;
  return RSO_OK;
}

extern "C" int rso_bottom_kernel(const rso_handle* h) { return h ? h->tune.bottom_kind : -1; }

extern "C" rso_status rso_set_solve_graphs(rso_handle* h, int on) {
  if (!h) return RSO_ERR_INVALID_ARG;
  h->solve_graphs = on != 0;
  return RSO_OK;
}

extern "C" rso_status rso_set_krylov_fp32(rso_handle* h, double replace_factor) {
  if (!h || !(replace_factor >= 0.0) || !(replace_factor < 1.0)) return RSO_ERR_INVALID_ARG;
  h->krylov32 = replace_factor;
  return RSO_OK;
}

extern "C" rso_status rso_set_krylov_fp32_cycles(rso_handle* h, int max_cycles) {
  if (!h || max_cycles < 0) return RSO_ERR_INVALID_ARG;
  h->krylov32_cycles = max_cycles;
  return RSO_OK;
}

extern "C" rso_status rso_fine_sweep_fp32(rso_handle* h, int op, const double* u, const double* f,
                                          const double* uprev, double omega, double c1, double* out) {
  if (!h || !u || !out || op < 0 || op > 3 || (op != 1 && !f)) return RSO_ERR_INVALID_ARG;
  Level& l0 = h->L[0];
  const long long n3 = 3 * l0.NP;
  RSO_TRY(pad_nodes(h, 0, u, l0.u64));
  RSO_TRY(zero_support(h, l0.u64));
  RSO_TRY(to_f32(h, l0.u64, l0.u32, n3));
  if (f) {
    RSO_TRY(pad_nodes(h, 0, f, l0.f64));
    RSO_TRY(zero_support(h, l0.f64));
    RSO_TRY(to_f32(h, l0.f64, l0.f32, n3));
  }
  const float* up = nullptr;
  if (uprev && op == 2) {
    RSO_TRY(pad_nodes(h, 0, uprev, l0.t64));
    RSO_TRY(zero_support(h, l0.t64));
    RSO_TRY(to_f32(h, l0.t64, l0.t32, n3));
    up = l0.t32;
  }
  if (op == 0) RSO_TRY(fine_residual<float>(h, l0.u32, l0.f32, l0.r32, h->rp32));
  else if (op == 1) RSO_TRY(fine_applyK<float>(h, l0.u32, l0.r32, h->rp32));
  else if (op == 2) RSO_TRY(fine_jacobi<float>(h, l0.u32, l0.f32, l0.r32, h->rp32, omega, up, c1));
  else RSO_TRY(fine_jacobi0<float>(h, l0.f32, l0.r32, h->rp32, omega));
  RSO_TRY(to_f64(h, l0.r32, l0.r64, n3));
  RSO_TRY(unpad_nodes(h, 0, l0.r64, out));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return fine_stage_check(h);
}

__global__ void k_unpad_planes(Level L, const double* __restrict__ pad, double* __restrict__ dense, int planes) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= L.nn) return;
  int x = i % L.nx, y = (i / L.nx) % L.ny, z = i / ((long long)L.nx * L.ny);
  long long j = L.nidx(x, y, z);
  for (int p = 0; p < planes; p++) dense[i + p * L.nn] = pad[j + p * L.NP];
}

extern "C" rso_status rso_get_stencil(rso_handle* h, int level, double* out) {
  if (!h || !out || level < 1 || level >= (int)h->L.size()) return RSO_ERR_INVALID_ARG;
  RSO_TRY(need_ops(h));
  const Level& l = h->L[level];
  k_unpad_planes<<<cdiv(l.nn, 256), 256, 0, h->stream>>>(l, l.st64, out, 243); rso::note_launch();
  RSO_TRY(launch_check(h, "get_stencil"));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_coarse_residual(rso_handle* h, int level, const double* u, const double* f, double* r) {
  if (!h || !u || !f || !r || level < 1 || level >= (int)h->L.size()) return RSO_ERR_INVALID_ARG;
  RSO_TRY(need_ops(h));
  Level& l = h->L[level];
  RSO_TRY(pad_nodes(h, level, u, l.u64));
  RSO_TRY(pad_nodes(h, level, f, l.f64));
  RSO_TRY(coarse_residual<double>(h, level, l.u64, l.f64, l.r64));
  RSO_TRY(unpad_nodes(h, level, l.r64, r));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_smooth(rso_handle* h, int level, double* u, const double* f, int kind, double omega,
                                 int sweeps, int reverse) {
  if (!h || !u || !f || level < 0 || level >= (int)h->L.size() || sweeps < 0) return RSO_ERR_INVALID_ARG;
  if (level > 0) RSO_TRY(need_ops(h));
  Level& l = h->L[level];
  RSO_TRY(pad_nodes(h, level, u, l.u64));
  RSO_TRY(pad_nodes(h, level, f, l.f64));
  if (level == 0) { RSO_TRY(zero_support(h, l.u64)); RSO_TRY(zero_support(h, l.f64)); }
  for (int s = 0; s < sweeps; s++) {
    if (kind == RSO_SMOOTH_GS) {
      for (int ci = 0; ci < 8; ci++) {
        const int c = reverse ? 7 - ci : ci;
        if (level == 0) RSO_TRY(fine_gs<double>(h, l.u64, l.f64, h->rp64, c, reverse));
        else RSO_TRY(coarse_gs<double>(h, level, l.u64, l.f64, c, reverse));
      }
    } else {
      if (level == 0) RSO_TRY(fine_jacobi<double>(h, l.u64, l.f64, l.t64, h->rp64, omega));
      else RSO_TRY(coarse_jacobi<double>(h, level, l.u64, l.f64, l.t64, omega));
      std::swap(l.u64, l.t64);
    }
  }
  RSO_TRY(unpad_nodes(h, level, l.u64, u));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_restrict(rso_handle* h, int cl, const double* rf, double* fc) {
  if (!h || !rf || !fc || cl < 1 || cl >= (int)h->L.size()) return RSO_ERR_INVALID_ARG;
  RSO_TRY(pad_nodes(h, cl - 1, rf, h->L[cl - 1].r64));
  RSO_TRY(restrict_<double>(h, cl, h->L[cl - 1].r64, h->L[cl].f64));
  RSO_TRY(unpad_nodes(h, cl, h->L[cl].f64, fc));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_prolong(rso_handle* h, int cl, const double* uc, double* uf) {
  if (!h || !uc || !uf || cl < 1 || cl >= (int)h->L.size()) return RSO_ERR_INVALID_ARG;
  RSO_TRY(pad_nodes(h, cl, uc, h->L[cl].u64));
  RSO_TRY(pad_nodes(h, cl - 1, uf, h->L[cl - 1].u64));
  RSO_TRY(prolong<double>(h, cl, h->L[cl].u64, h->L[cl - 1].u64));
  RSO_TRY(unpad_nodes(h, cl - 1, h->L[cl - 1].u64, uf));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_coarsest_solve(rso_handle* h, const double* f, double* u) {
  if (!h || !f || !u || h->L.size() < 2) return RSO_ERR_INVALID_ARG;
  RSO_TRY(need_ops(h));
  const int cl = (int)h->L.size() - 1;
  Level& c = h->L[cl];
  RSO_TRY(pad_nodes(h, cl, f, c.f64));
  RSO_CHECK_CUDA(h, cudaMemsetAsync(c.u64, 0, sizeof(double) * 3 * c.NP, h->stream));
  RSO_TRY(coarsest_solve<double>(h, c.f64, c.u64));
  RSO_TRY(unpad_nodes(h, cl, c.u64, u));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_level_lambda(rso_handle* h, int level, double* lam) {
  if (!h || !lam || level < 0 || level >= (int)h->L.size()) return RSO_ERR_INVALID_ARG;
  *lam = h->L[level].lam;
  return RSO_OK;
}

extern "C" rso_status rso_vcycle(rso_handle* h, double* u, const double* f, int pre, int post, int symmetric,
                                 double* rel) {
  if (!h || !u || !f || pre < 0 || post < 0) return RSO_ERR_INVALID_ARG;
  RSO_TRY(need_ops(h));
  RSO_TRY(pad_nodes(h, 0, u, h->x));
  RSO_TRY(pad_nodes(h, 0, f, h->w));
  RSO_TRY(zero_support(h, h->x));
  RSO_TRY(zero_support(h, h->w));
  RSO_TRY(vcycle_fp64(h, h->x, h->w, pre, post, symmetric, rel));
  RSO_TRY(unpad_nodes(h, 0, h->x, u));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}

extern "C" rso_status rso_solve(rso_handle* h, const double* f, double* u, double tol, int max_iter, int method,
                                rso_solve_info* info) {
  if (!h || !f || !u || !(tol > 0) || max_iter < 0) return RSO_ERR_INVALID_ARG;
  RSO_TRY(need_ops(h));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  RSO_TRY(pad_nodes(h, 0, u, h->x));
  RSO_TRY(pad_nodes(h, 0, f, h->w));
  RSO_TRY(zero_support(h, h->x));
  RSO_TRY(zero_support(h, h->w));
  // support-free problems: no displacement balances the rigid-motion part of
  // a load, so the solve takes the load without it
  RSO_TRY(displacement_project(h, h->w));
  cudaEventRecord(e0, h->stream);
  rso_status s = method == RSO_SOLVE_PCG ? solve_pcg(h, h->w, h->x, tol, max_iter, info)
                                         : solve_vcycles(h, h->w, h->x, tol, max_iter, info);
  cudaEventRecord(e1, h->stream);
  if (s == RSO_OK || s == RSO_ERR_BUDGET_EXCEEDED) {
    rso_status s2 = unpad_nodes(h, 0, h->x, u);
    if (s2 != RSO_OK) s = s2;
  }
  cudaStreamSynchronize(h->stream);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  if (info) info->ms = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return s;
}

extern "C" rso_status rso_dot(rso_handle* h, const double* a, const double* b, double* out) {
  if (!h || !a || !b || !out) return RSO_ERR_INVALID_ARG;
  return dot_host(h, a, b, 3 * h->L[0].nn, out);
}
