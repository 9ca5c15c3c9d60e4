// Internal definitions of the B200 voxel-FEM library (librso).
//
// Device data layout ("padded box"): every level stores its nodes on a box
// padded by one zero node on each side, x fastest, the padded x extent
// rounded up to a multiple of 4 so that rows stay 32-byte aligned:
//   node (x,y,z), x in [-1, nx] -> (x+1) + px*((y+1) + py*(z+1))
// Element fields use the same scheme with their own extents.  Halo entries
// are zero, so the matrix-free operator needs no bounds tests, and a padded
// element with zero density contributes nothing.  Nodal vectors are three
// consecutive component planes of NP entries each.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <type_traits>
#include <vector>
#include "../../include/rso.h"

namespace rso {

enum : uint8_t { NC_ACTIVE = 1, NC_SURFACE = 2, NC_SUPPORT = 4, NC_LOAD = 8 };

struct Level {
  int ex = 0, ey = 0, ez = 0;     // element extents
  int nx = 0, ny = 0, nz = 0;     // node extents
  int px = 0, py = 0, pz = 0;     // padded node extents
  int qx = 0, qy = 0, qz = 0;     // padded element extents
  long long NP = 0, NQ = 0;       // padded node / element counts
  long long nn = 0, ne = 0;       // unpadded counts
  int factor = 0;                 // coarsening factor from the finer level
  int nb = 1;                     // systems carried by the level vectors (batched solves): each of
                                  // u/f/r/t then holds nb consecutive vectors of 3 NP entries
  long long n_active_e = 0, n_active_v = 0;
  uint8_t* emask = nullptr;       // padded element mask
  uint8_t* vclass = nullptr;      // padded node class
  double* KE = nullptr;           // coarse element matrices, 576 per unpadded element
  double* st64 = nullptr;         // stencil [243][NP]
  float* st32 = nullptr;          // stencil in tiles of 128 nodes (st_at), 243 x round_up(NP, 128)
  double *u64 = nullptr, *f64 = nullptr, *r64 = nullptr, *t64 = nullptr;
  float *u32 = nullptr, *f32 = nullptr, *r32 = nullptr, *t32 = nullptr;
  double lam = 1.0;               // lambda_max(D^-1 K) estimate
  __host__ __device__ long long nidx(int x, int y, int z) const {
    return (long long)(x + 1) + (long long)px * ((y + 1) + (long long)py * (z + 1));
  }
  __host__ __device__ long long eidx(int x, int y, int z) const {
    return (long long)(x + 1) + (long long)qx * ((y + 1) + (long long)qy * (z + 1));
  }
};

// Index of stencil entry k (0..242) of padded node n.  FP64 stencils are
// [243][NP]; FP32 stencils, the ones the mixed V-cycle streams, are stored in
// tiles of 128 consecutive padded nodes, [NP/128][243][128], so that the
// threads of a warp reading a run of nodes stream one contiguous block
// (243 x 512 bytes) instead of 243 blocks of 512 bytes a stencil row apart.
constexpr long long ST_TILE = 128;
template <typename T>
__host__ __device__ __forceinline__ long long st_at(long long NP, int k, long long n) {
  if constexpr (sizeof(T) == 4) return ((n / ST_TILE) * 243 + k) * ST_TILE + (n % ST_TILE);
  else return (long long)k * NP + n;
}
__host__ __device__ __forceinline__ long long st32_len(long long NP) {
  return 243 * ((NP + ST_TILE - 1) / ST_TILE) * ST_TILE;
}

// Level is passed to kernels by value: it must stay a plain, trivially
// copyable record (host-side data such as the unpadded masks lives in the
// handle), or every launch would copy it member by member on the host.
static_assert(std::is_trivially_copyable<Level>::value, "Level must be trivially copyable");

struct Spline {
  int order = 0, part[3] = {0, 0, 0}, nb[3] = {0, 0, 0};
  float bmin[3], bmax[3], step[3];
  std::vector<float> knots[3];
  std::vector<int> h_idx[3];
  std::vector<double> h_N[3], h_dN[3];
  int* idx[3] = {nullptr, nullptr, nullptr};       // per element coordinate, -1 outside
  double* N[3] = {nullptr, nullptr, nullptr};      // order values per coordinate
  double* dN[3] = {nullptr, nullptr, nullptr};
  long long n_coeff = 0;
  float* knots_dev = nullptr;                      // the three knot vectors back to back
  int* ranges[3] = {nullptr, nullptr, nullptr};    // per basis index: first/last element coordinate in its support
  double* work[10] = {};                           // adjoint and self-support scratch
};

}  // namespace rso

struct rso_handle {
  rso_config cfg;
  std::string err;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int device = 0;
  int material_dev = -1;            // device whose constant-memory element matrix this handle holds
  std::vector<rso::Level> L;
  std::vector<std::vector<uint8_t>> h_emask, h_vmask;  // per level, unpadded host copies (set-up only)
  double K0[576];
  double* K0_dev = nullptr;
  // fine-level design fields (padded elements)
  float* rho = nullptr;
  float* rp32 = nullptr;
  double* rp64 = nullptr;
  bool operators_ready = false;
  // load nodes
  std::vector<int> h_load_nodes;      // dense node ids, reference order
  int n_load = 0;
  int* load_nodes = nullptr;          // padded node ids
  double* load_normals = nullptr;     // 3 per load node
  // Galerkin tables
  double* T1 = nullptr;               // F^3 x 576 table for the first coarsening
  uint8_t* efix = nullptr;            // per padded fine element: bit a set if local node a is a support node
  int* gfix = nullptr;                // coarse elements with a child that touches a support node
  int n_gfix = 0;
  void* filt_taps = nullptr;          // sensitivity-filter tap table of the last radius used
  long long filt_cap = 0;
  double filt_radius = -1.0;
  // batched solves (rso_solve_batch): system-major slabs, allocated on first use
  struct Batch {
    int cap = 0;                                      // systems the slabs hold
    std::vector<float*> u32, f32, r32, t32;           // per level, cap * 3 NP each
    std::vector<double*> u64, f64, r64, t64;
    double *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *z = nullptr;  // fine FP64, cap * 3 NP
    double *cf = nullptr, *red = nullptr, *fpart = nullptr, *xfer = nullptr;
    double *scal = nullptr, *h_scal = nullptr;
    double* ralpha = nullptr;                         // step sizes of the deferred steps, [ring slot][system]
    int* done = nullptr;
  } batch;
  double* c_fb = nullptr;             // coarsest right-hand sides of a batch (cap x 3 nc)

  // coarsest dense solve
  int nc = 0;                         // active coarsest nodes
  int* c_nodes = nullptr;             // padded node ids of active coarsest nodes
  double* c_K = nullptr;              // N x N workspace / inverse
  double* c_f = nullptr;
  int* c_flag = nullptr;              // factorisation status
  // support-free problems (RSO_NO_SUPPORT_* modes, rigid.cu): the rigid
  // motions of the load set (orthonormal, load space, ff and normal-projected
  // cf), the inverse Gram matrix of the fine nodes' rigid motions about their
  // centroid (displacement projection), and those of the coarsest nodes
  bool has_support = true;
  double* rigid_q = nullptr;          // [2][6][3 n_load]
  int rigid_k[2] = {0, 0};
  double* rigid_m = nullptr;          // 6 x 6 inverse Gram matrix, then the centroid (39 doubles)
  double* rigid_scr = nullptr;        // partial sums of the projections
  double* c_R = nullptr;              // coarsest rigid motions, 3 nc x 6 row-major, orthonormal
  // reductions
  double* red = nullptr;              // partials
  unsigned* gbar = nullptr;           // grid barrier of the persistent bottom kernel: arrivals, generation, gave-up flag
  double* xfer = nullptr;             // restriction scratch: z-filtered fine columns
  size_t xfer_n = 0;                  // its capacity in doubles
  double* fpart = nullptr;            // per-CTA partial sums of the fine operator kernel
  long long fpart_n = 0;
  double* scal = nullptr;             // device scalars
  double* h_scal = nullptr;           // pinned host mirror
  // PCG / solver vectors (fine, FP64, padded)
  double *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *z = nullptr, *w = nullptr;
  // public-layout staging
  double* stage_a = nullptr;
  double* stage_b = nullptr;
  // spline
  rso::Spline sp;
  // worst case storage
  std::vector<double*> lanczos_u;
  long long n_gs_elements = 0;
  // design-iteration scratch
  float *e_a = nullptr, *e_b = nullptr, *e_c = nullptr, *e_d = nullptr, *e_rhohat = nullptr;
  uint8_t* shell_pad = nullptr;       // padded copy of a caller's shell mask (design_capi.cu), made on first use
  double *coef_a = nullptr, *coef_b = nullptr, *coef_c = nullptr;
  double *coef_df = nullptr, *coef_dg = nullptr;   // MMA inputs
  double *fw = nullptr, *uw = nullptr;             // worst-case force / displacement (padded)
  unsigned prof_on = 0;                            // classes with per-kernel event timing (prof.cu)
  void* prof = nullptr;
  // launch shapes chosen by rso_autotune (autotune.cu); -1 / -2 keep the built-in rules
  struct Tune {
    int fine_rows = 4;      // thread rows of a CTA of the packed FP32 fine kernel (2, 4 or 8)
    int fine_zc = 0;        // node planes per z chunk of that kernel (4, 8, 16 or 32; 0: by size)
    int rowsplit[16];       // per level: 0 one thread per node, 1 per (node, row), 2 nine per node, -1 by size
    int bottom = -2;        // first level of the bottom kernel, -1 none, -2 by size
    int bottom_kind = 1;    // bottom kernel: 1 the persistent grid-wide kernel, 0 the 8-CTA cluster kernel
    Tune() { for (int& r : rowsplit) r = -1; }
  } tune;
  // reliable-update PCG (mixed precision): the Krylov recurrence in FP32,
  // the true FP64 residual replacing the recursive one once it has dropped by
  // this factor since the last replacement (0: FP64 recurrence); rso_create
  // sets 1e-2 for mixed precision
  double krylov32 = 0.0;
  // replacement cycles the FP32 recurrence may run before the solve goes on
  // with the FP64 recurrence (0: no limit; rso_set_krylov_fp32_cycles)
  int krylov32_cycles = 0;
  // worst-case scratch kept between calls (worst.cu): Lanczos load-space
  // vectors, reorthogonalisation sums, the force-projection vector
  double* wc_buf = nullptr;
  size_t wc_cap = 0;
  void* vcg = nullptr;                             // captured FP32 V-cycles (solver.cu)
  void* cap_prof = nullptr;                        // event pairs of the V-cycle capture in progress (prof.cu)
  bool vc_graphs = true;                           // replay captured V-cycles (rso_set_vcycle_graphs)
  // run the FP32-Krylov PCG loop as one captured graph whose iterations and
  // residual replacements are decided on the device (rso_set_solve_graphs)
  bool solve_graphs = false;
  void* sgc = nullptr;                             // captured solve graphs (solver.cu)
  // when set, the FP32 V-cycle's last fine sweep also sums f . u into this
  // device scalar (the CG step's r . z; solver.cu)
  double* vc_zdot = nullptr;
  int vc_zdot_stride = 1;             // its spacing between systems (batched solves)
  void* surf = nullptr;                            // surface-point self-support state (surface.cu)
};

namespace rso {
// launch accounting and profiling (prof.cu)
enum ProfClass {
  PC_FINE_JAC32, PC_FINE_RES32, PC_FINE_GS32, PC_FINE_APPLYK64, PC_FINE_RES64, PC_FINE_JAC64, PC_FINE_GS64,
  PC_COARSE32, PC_COARSE64, PC_COARSE32_STREAM, PC_BOTTOM, PC_N
};
void note_launch();
void note_launches(long long n);
void prof_begin(rso_handle* h, int cls, double nodes);
void prof_end(rso_handle* h, int cls);
void prof_free(rso_handle* h);
// event pairs recorded into a captured V-cycle: created before the capture,
// read after each replay
void* prof_pairs_new(int capacity);
void prof_pairs_free(void* pairs);
bool prof_pairs_used(const void* pairs);
void prof_harvest(rso_handle* h, void* pairs);
// captured V-cycles (solver.cu)
void vcycle_graphs_harvest(rso_handle* h);
void vcycle_graphs_free(rso_handle* h);
void solve_graphs_free(rso_handle* h);
// node planes per z chunk of the packed FP32 fine kernel (fine_op.cu)
constexpr int kFineZcMax = 32, kFineZcMin = 4;
int fine_zc(const rso_handle* h);
// kernel variant of a coarse level: 0 per node, 1 per (node, row), 2 nine threads per node (coarse_op.cu)
int coarse_variant_of(const rso_handle* h, int level);
// surface-point self-support state (surface.cu)
void surface_free(rso_handle* h);
// bounding box {xmin, ymin, zmin, xmax, ymax, zmax} of the active elements
void active_box(rso_handle* h, float box[6]);
// the rho = 0.5 samples (kept on the handle) and the constraint at them;
// c: n_coeff doubles on the device, dc (device, may be NULL) divided by the count
rso_status surface_points(rso_handle* h, const double* c, int mc, int npts, const float* box, rso_surface_info* info);
rso_status surface_selfsupport(rso_handle* h, const double* c, double beta, int mode, double opt_angle,
                               double default_angle, float* per_out, double* dc, double* value, double* count,
                               double* dirsum);
}  // namespace rso

// ---------------------------------------------------------------- helpers
#define RSO_CHECK_CUDA(h, call)                                                          \
  do {                                                                                   \
    cudaError_t _e = (call);                                                             \
    if (_e != cudaSuccess) {                                                             \
      (h)->err = std::string(#call) + ": " + cudaGetErrorString(_e);                      \
      return RSO_ERR_CUDA;                                                               \
    }                                                                                    \
  } while (0)

#define RSO_TRY(call)                 \
  do {                                \
    rso_status _s = (call);           \
    if (_s != RSO_OK) return _s;      \
  } while (0)

namespace rso {

inline int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

rso_status launch_check(rso_handle* h, const char* what);

// reductions (reduce.cu)
rso_status dot(rso_handle* h, const double* a, const double* b, long long n, double* dev_out);
rso_status dot_host(rso_handle* h, const double* a, const double* b, long long n, double* out);
rso_status cg_resid_rr(rso_handle* h, long long n, const double* alpha, const double* q, double* r, float* r32,
                       double* rr_dev);
rso_status reduce_partials(rso_handle* h, const double* part, int n, double* dev_out);
rso_status reduce_partials_batch(rso_handle* h, const double* part, int nper, int nb, double* dev_out,
                                 int stride = 1);
rso_status pow_step(rso_handle* h, long long n, const float* u, const float* t, float* r, double* uu, double* rr);
rso_status dot_df(rso_handle* h, const double* a, const float* b, long long n, double* dev_out);
rso_status dot_ff(rso_handle* h, const float* a, const float* b, long long n, double* dev_out);
rso_status cg32_resid_rr(rso_handle* h, long long n, const double* alpha, const float* q, float* r, double* rr_dev);
rso_status fine_applyK_dot32(rso_handle* h, const float* u, float* f, double* dot_dev, int stride = 1);
rso_status sum_float(rso_handle* h, const float* a, long long n, double* dev_out);

// conversion between the public dense layout and padded layout
rso_status pad_nodes(rso_handle* h, int level, const double* dense, double* padded);
rso_status unpad_nodes(rso_handle* h, int level, const double* padded, double* dense);
rso_status pad_elems_f(rso_handle* h, const float* dense, float* padded);
rso_status unpad_elems_f(rso_handle* h, const float* padded, float* dense);
rso_status zero_support(rso_handle* h, double* padded);
rso_status to_f32(rso_handle* h, const double* a, float* b, long long n);
rso_status fine_stage_check(rso_handle* h);
rso_status to_f64(rso_handle* h, const float* a, double* b, long long n);

// topology (topology.cu)
Level make_level(int ex, int ey, int ez, int factor);
rso_status build_topology(rso_handle* h, const uint8_t* emask, const uint8_t* fixed_area,
                          const uint8_t* load_area, const double* load_normals);

// fine operator (fine_op.cu)
template <typename T>
rso_status fine_residual(rso_handle* h, const T* u, const T* f, T* r, const T* rp);
template <typename T>
rso_status fine_applyK(rso_handle* h, const T* u, T* f, const T* rp);
constexpr int kMaxSweeps = 16;
void smoother_steps(const rso_handle* h, double lam, int m, double* om, double* c1);
// levels of at most this many nodes are the bottom kernels' (the built-in
// rule's first level; the largest rso_autotune tries)
constexpr long long kBottomMaxNodes = 60000;
int bottom_level(const rso_handle* h, bool fp32 = true);
template <typename T>
rso_status bottom_vcycle(rso_handle* h, int lb, int pre, int post);
rso_status fine_applyK_dot(rso_handle* h, const double* u, double* f, const double* rp, double* dot_dev,
                           int stride = 1);
template <typename T>
rso_status fine_jacobi(rso_handle* h, const T* u_in, const T* f, T* u_out, const T* rp, double omega,
                       const T* u_prev = nullptr, double c1 = 0.0);
// the FP32 Jacobi / Chebyshev step with dot_dev = f . u_out from the same pass
rso_status fine_jacobi_dot32(rso_handle* h, const float* u_in, const float* f, float* u_out, double omega,
                             const float* u_prev, double c1, double* dot_dev, int stride = 1);
// the FP64 residual with its FP32 copy and r . r from the same pass
rso_status fine_residual64_rr(rso_handle* h, const double* u, const double* f, double* r, float* r32,
                              double* dot_dev);
template <typename T>
rso_status fine_jacobi0(rso_handle* h, const T* f, T* u_out, const T* rp, double omega);
template <typename T>
rso_status fine_gs(rso_handle* h, T* u, const T* f, const T* rp, int colour, int reverse);
rso_status upload_K0(rso_handle* h);
rso_status penalise(rso_handle* h);

// coarse levels (coarse_op.cu)
template <typename T>
rso_status coarse_residual(rso_handle* h, int level, const T* u, const T* f, T* r);
template <typename T>
rso_status coarse_jacobi(rso_handle* h, int level, const T* u_in, const T* f, T* u_out, double omega,
                         const T* u_prev = nullptr, double c1 = 0.0);
template <typename T>
rso_status coarse_gs(rso_handle* h, int level, T* u, const T* f, int colour, int reverse);
template <typename T>
rso_status restrict_(rso_handle* h, int coarse_level, const T* rf, T* fc);
template <typename T>
rso_status prolong(rso_handle* h, int coarse_level, const T* uc, T* uf);
template <typename T>
rso_status coarsest_solve(rso_handle* h, const T* f, T* u);
rso_status galerkin_setup(rso_handle* h);
// coarsest dense solve (dense.cu): A (N x N) -> Cholesky factor in its lower
// triangle, X = A^-1, Y scratch; *flag_dev set on a pivot that is not positive
rso_status dense_spd_inverse(rso_handle* h, double* A, double* X, double* Y, int N, int* flag_dev);
// A += a R R^T, R row-major N x nr
rso_status dense_rank_update(rso_handle* h, double* A, int N, const double* R, int nr, double a);
rso_status galerkin(rso_handle* h);
rso_status coarsest_factor(rso_handle* h);
rso_status estimate_lambda(rso_handle* h);

// solver (solver.cu)
template <typename T>
rso_status vcycle_levels(rso_handle* h, int pre, int post, int symmetric, bool u0_zero);
rso_status precondition(rso_handle* h, const double* r, double* z);
rso_status vcycle_mixed(rso_handle* h);
void batch_release(rso_handle* h);
rso_status solve_pcg_batch(rso_handle* h, int k, const double* F_dense, double* U_dense, double tol, int max_iter,
                           rso_solve_info* infos);
// u_zero: the caller set u to zero, so the first residual is f itself (the
// FP64 operator pass on zero is skipped; the same values)
rso_status solve_pcg(rso_handle* h, const double* f, double* u, double tol, int max_iter, rso_solve_info* info,
                     bool u_zero = false);
// the FP32 recurrence stalls when a replacement's true residual is not below
// this fraction of the previous one (claimed: the recursive residual's reduction)
double stall_ratio(double factor, double claimed);
rso_status solve_vcycles(rso_handle* h, const double* f, double* u, double tol, int max_iter,
                         rso_solve_info* info);
rso_status vcycle_fp64(rso_handle* h, double* u, const double* f, int pre, int post, int symmetric,
                       double* rel_res);

// elementwise kernels shared by several files
rso_status axpby(rso_handle* h, long long n, double a, const double* x, double b, double* y);
rso_status fill_d(rso_handle* h, double* p, long long n, double v);
rso_status fill_f(rso_handle* h, float* p, long long n, float v);

// design (design.cu)
rso_status sensitivity(rso_handle* h, const double* u_pad, float* sens_pad, int energy);
rso_status heaviside(rso_handle* h, const float* in_pad, double beta, const uint8_t* shell_pad, float* out_pad);
rso_status heaviside_chain(rso_handle* h, const float* rho_pad, double beta, const float* gin, float* gout);
rso_status filter(rso_handle* h, double radius, const float* in_pad, float* out_pad, int adjoint);
rso_status coeff2density(rso_handle* h, const double* c, const uint8_t* shell_pad, float* out_pad);
rso_status density2coeff(rso_handle* h, const float* g_pad, const uint8_t* shell_pad, double* dc);
rso_status selfsupport(rso_handle* h, const double* c, double beta, int mode, double opt_angle,
                       double default_angle, float* per_pad, double* dc, double* value, double* count,
                       double* dirsum);
rso_status volume(rso_handle* h, const float* rho_pad, double* vol);
rso_status spline_setup(rso_handle* h, int order, int px, int py, int pz);

// worst case (worst.cu)
rso_status force_project(rso_handle* h, double* f_pad, int cf);
// support-free problems (rigid.cu): set-up of the rigid motions; removal of
// the load set's rigid motions from a load-space vector (3 per load node);
// removal of the fine nodes' rigid motions from a padded FP64 nodal vector
// (displacementProject); both no-ops when the problem has supports
rso_status rigid_setup(rso_handle* h);
rso_status rigid_project_load(rso_handle* h, double* v, int cf);
rso_status displacement_project(rso_handle* h, double* u_pad);
// sum of the diagonal of a dense N x N matrix into *out (device)
rso_status dense_trace(rso_handle* h, const double* A, int N, double* out_dev);
rso_status worst_case(rso_handle* h, int steps, int cf, double tol, uint64_t seed, double* f_pad,
                      double* u_pad, double* lambda, double* ritz, int* iters);
rso_status modified_pm(rso_handle* h, int cf, uint64_t seed, int max_itn, double* f_pad, double* u_pad,
                       double* c_worst, int* itn);

// MMA state accessors (mma.cu)
double* mma_x(rso_mma* s);
int mma_n(rso_mma* s);
int mma_m(rso_mma* s);

}  // namespace rso

// deterministic uniform [-1,1) stream shared with the oracle
__host__ __device__ inline uint64_t rso_splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__host__ __device__ inline double rso_urand(uint64_t seed, uint64_t i) {
  uint64_t h = rso_splitmix64(seed * 0x100000001B3ull ^ rso_splitmix64(i));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}
