/*
 * rso.h - C ABI of the B200-native voxel-FEM worst-case topology-optimisation
 * path (capabilities of NanXYZH/RobustOptSpline3D).
 *
 * Conventions
 *  - Box of ex*ey*ez hexahedral voxels with unit edge, origin 0.  Elements are
 *    numbered e = x + ex*(y + ey*z); nodes n = x + nx*(y + ny*z), nx = ex+1.
 *  - Nodal vectors are structure-of-arrays: v[c*Nn + n], c = 0,1,2, double.
 *  - Element fields (densities, sensitivities) and spline coefficients are
 *    float, as in the reference (rho_e, g_sens, coeffs are float there).
 *  - Pointers named *_dev are CUDA device pointers owned by the caller and
 *    borrowed for the duration of the call; *_host are host pointers.
 *  - Every call returns rso_status and never aborts; rso_last_error() gives a
 *    message.  Calls on one handle are ordered on the handle's stream (its
 *    own non-blocking stream unless rso_set_stream binds another): device
 *    inputs written on a different stream must be complete (synchronised, or
 *    ordered by an event) before the call.  Handles are not thread-safe;
 *    distinct handles are independent and may be used from different host
 *    threads at once, provided the live handles on one device share the
 *    same Young's modulus and Poisson ratio (rso_create refuses otherwise).
 *  - Dirichlet (support) DOFs are homogeneous: entries of f and u at support
 *    nodes are ignored on input and returned as zero.
 *
 * Each entry point cites the reference interface it replaces (file:line in
 * the reference project).
 */
#ifndef RSO_H
#define RSO_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  RSO_OK = 0,
  RSO_ERR_INVALID_ARG = 1,
  RSO_ERR_OOM = 2,
  RSO_ERR_CUDA = 3,
  RSO_ERR_DIVERGED = 4,
  RSO_ERR_NONFINITE = 5,
  RSO_ERR_BUDGET_EXCEEDED = 6,
  RSO_ERR_UNSUPPORTED = 7,
  RSO_ERR_STATE = 8
} rso_status;

/* smoothers */
enum { RSO_SMOOTH_GS = 0, RSO_SMOOTH_JACOBI = 1, RSO_SMOOTH_CHEBYSHEV = 2 };
/* RSO_SMOOTH_CHEBYSHEV (no counterpart in the reference, which smooths with
 * damped Jacobi or coloured Gauss-Seidel): `pre`/`post` Chebyshev steps for
 * D^-1 K on [cheb_lower * lambda_max, lambda_max] (cheb_lower defaults to
 * 0.25), D the 3x3 diagonal blocks; omega is not used.  A polynomial in D^-1 K, so the V-cycle stays symmetric. */
/* V-cycle arithmetic */
enum { RSO_FP64 = 0, RSO_MIXED = 1 };
/* solve methods */
enum { RSO_SOLVE_VCYCLE = 0, RSO_SOLVE_PCG = 1 };
/* worst-case modes: grid/Grid.h:170-175 HierarchyGrid::Mode */
enum {
  RSO_NO_SUPPORT_CONSTRAIN_FORCE_DIRECTION = 0,
  RSO_NO_SUPPORT_FREE_FORCE = 1,
  RSO_WITH_SUPPORT_CONSTRAIN_FORCE_DIRECTION = 2,
  RSO_WITH_SUPPORT_FREE_FORCE = 3
};

typedef struct rso_handle rso_handle;
typedef struct rso_mma rso_mma;

/* Problem parameters; replaces the Parameter struct and HierarchySetting
 * (optimization/optimization.h:15-35, grid/Grid.h:836-862). */
typedef struct {
  double youngs_modulus;   /* E  (reference default 1e6) */
  double poisson_ratio;    /* nu */
  double penal;            /* SIMP power p */
  double rho_min;          /* density floor */
  int n_levels;            /* 0: reference policy, coarsen while > 400 active elements */
  int first_factor;        /* 4: non-dyadic first coarsening (skip layer 1, reference); 2: dyadic */
  int smoother;            /* RSO_SMOOTH_GS, _JACOBI or _CHEBYSHEV */
  double omega;            /* damped Jacobi factor relative to the bound 2/lambda_max(D^-1 K) */
  int pre, post;           /* smoothing sweeps */
  int precision;           /* RSO_FP64 or RSO_MIXED (FP32 V-cycle and CG recurrence, FP64 iterate and residual replacement) */
  int mode;                /* RSO_WITH_SUPPORT_* / RSO_NO_SUPPORT_* */
  double cheb_lower;       /* Chebyshev smoother: lower end of the damped interval, as a fraction of lambda_max */
} rso_config;

typedef struct {
  int iterations;
  double rel_res;
  double ms;
} rso_solve_info;

/* ---------------------------------------------------------------- mesh input */
/* Solid voxelisation of a closed triangle mesh, the mesh -> voxel-mask step of
 * the reference's drivers (voxelize_mesh, voxelizer/voxelize_main.cpp:344-399,
 * with the vendored cuda_voxelizer's solid mode, voxelizer/cpu_voxelizer.cpp:
 * 206-330): a cubic grid of R^3 voxels, R the smallest power of two above
 * preferred_resolution, around the mesh's bounding box enlarged to
 * max_len * R / preferred_resolution per axis and centred; a voxel is solid
 * when its centre has an odd number of mesh crossings along +x (top-left rule
 * on projected edges).  vertices: 3 n_vertices floats; faces: 3 n_faces
 * vertex indices.  solid_host: R^3 bytes, x fastest (NULL with box_out NULL
 * asks for R only); box_out: NULL or 6 floats (min xyz, max xyz).  Uses the
 * current device; allocates its own scratch. */
rso_status rso_voxelize(const float* vertices_host, int n_vertices, const int* faces_host, int n_faces,
                        int preferred_resolution, uint8_t* solid_host, int* resolution_out, float* box_out);

/* Shell elements of a voxelised mesh (HierarchyGrid::setSolidShellElement,
 * grid/Grid.cpp:253-322): with h = (box max x - box min x) / R (FP32
 * quotient) and w = shell_width * h, solid element e = (x, y, z) of the R^3
 * grid is a shell element when some face's index box (its bounding box grown
 * by 1.3 w, mapped to element indices by truncation, upper end exclusive and
 * clamped to R - 1) contains e and the squared distance from e's centre to
 * the mesh is below w^2.  box: 6 floats as rso_voxelize returns them;
 * solid_host, shell_host: R^3 bytes, x fastest.  Allocates its own scratch. */
rso_status rso_shell_elements(const float* vertices_host, int n_vertices, const int* faces_host, int n_faces,
                              const float* box_host, int resolution, double shell_width, const uint8_t* solid_host,
                              uint8_t* shell_host);

/* Outward unit normals at points (Grid::outwardNormal, grid/Grid.cpp:
 * 2838-2854): q = closest point of the mesh to p (lowest face index on a
 * tie), t = (v0 - v2) x (v1 - v2) of that face; the normal is t / |t| when
 * |q - p| < 1e-6, else (q - p) / |q - p| oriented so that its dot with t is
 * non-negative.  points, normals: 3 n_points doubles (xyz per point).  Meshes
 * of 256 faces or more are searched through a uniform face grid, with the
 * same result as scanning every face. */
rso_status rso_mesh_normals(const float* vertices_host, int n_vertices, const int* faces_host, int n_faces,
                            const double* points_host, int n_points, double* normals_host);

/* Regions of space for boundary conditions (dynamic_range::range_t and its
 * sphere / box / half-space / cylinder kinds, boundary/BoundaryCondition.h:
 * 379-538; the static_range kinds :17-175 are the same tests without the
 * complement flag).  p by kind:
 *   SPHERE    centre xyz, radius: |p - c|^2 < r^2, closed adds |p - c|^2 - r^2 < 1e-8
 *   BOX       min xyz, max xyz:  min < p < max on every axis, closed min <= p <= max
 *   HALFSPACE a b c d:           a x + b y + c z + d > 0, closed adds = 0 (CGAL Plane_3)
 *   CYLINDER  bottom centre xyz, radius, axis vector xyz: 0 <= axial <= |axis|
 *             and radial distance < radius (closed and complement are ignored)
 * complement negates the test (sphere, box, half-space). */
enum { RSO_REGION_SPHERE = 0, RSO_REGION_BOX = 1, RSO_REGION_HALFSPACE = 2, RSO_REGION_CYLINDER = 3 };
typedef struct {
  int kind;
  int closed;
  int complement;
  int reserved;
  double p[8];
} rso_region;

/* A vector field restricted to a region (dynamic_range::rangeField_t and
 * vectorField_t, boundary/BoundaryCondition.h:570-700): inside the region the
 * value is norm(p) * dir(p), outside zero.
 *   norm: CONSTANT value | RADIAL centre xyz, amplifier, damp: a exp(-|c - p|^(2 damp))
 *         | TWIST axis start xyz, axis end xyz, amplifier: a |(p - s) x unit(e - s)|
 *   dir:  CONSTANT unit(d) | RADIAL unit(c - p) | TWIST unit((p - s) x (e - s))
 * unit(v) = v / |v| for |v| > 0, else v (Eigen normalized()). */
enum { RSO_FIELD_CONSTANT = 0, RSO_FIELD_RADIAL = 1, RSO_FIELD_TWIST = 2 };
typedef struct {
  rso_region region;
  int norm_kind;
  int dir_kind;
  double norm_p[7];
  double dir_p[6];
} rso_field;

/* Node mask of the union of regions (rangeUnion::generate, boundary/
 * BoundaryCondition.h:342-361 and :540-558) on the node grid
 * p = origin + (i, j, k) h, i fastest over nx (the node positions of
 * computeProjectionMatrix, grid/Grid.cpp:2694-2740).  mask_host: nx ny nz
 * bytes.  The result is the fixed_area / load_area argument of rso_create. */
rso_status rso_region_mask(const rso_region* regions_host, int n_regions, const double* origin_host, double h,
                           int nx, int ny, int nz, uint8_t* mask_host);

/* Sum of region fields at points (Field_t::at, boundary/BoundaryCondition.h:
 * 702-741; the load force of computeProjectionMatrix).  points, vectors:
 * 3 n_points doubles. */
rso_status rso_region_field(const rso_field* fields_host, int n_fields, const double* points_host,
                            int n_points, double* vectors_host);

/* ---------------------------------------------------------------- setup */
void rso_default_config(rso_config* cfg);

/* Build the hierarchy, topology, support/load node sets and all device
 * buffers.  emask: ex*ey*ez bytes (1 = solid voxel).  fixed_area/load_area:
 * node masks (Nn bytes) that play the role of the reference's
 * _inFixedArea/_inLoadArea predicates; load_normals: 3*Nn unit normals used
 * in constrained-direction modes (may be NULL otherwise).  In the
 * support-free modes (cfg->mode RSO_NO_SUPPORT_*, HierarchyGrid::Mode
 * grid/Grid.h:170-175) no node is fixed and fixed_area is not read: the
 * operator is singular on the rigid motions, the coarsest solve becomes a
 * pseudo-inverse (the reference's BDCSVD, grid/Grid.cpp:4123-4185), every
 * solution has its rigid motion removed (displacementProject) and every
 * admissible load the rigid motions of the load set (forceProject).
 * Replaces HierarchyGrid::genFromMesh(solid_bit, reso) (grid/Grid.cpp:978-1237),
 * Grid::build (grid/Grid.cpp:2973-3215), computeProjectionMatrix
 * (grid/Grid.cpp:2694-2836), setNodes/setLoadNodes (optimization/projection.cpp:46-269)
 * and uploadTemplateMatrix (optimization/optimization.cu:815-827). */
rso_status rso_create(const rso_config* cfg, int ex, int ey, int ez, const uint8_t* emask_host,
                      const uint8_t* fixed_area_host, const uint8_t* load_area_host,
                      const double* load_normals_host, rso_handle** out);
void rso_destroy(rso_handle* h);
const char* rso_last_error(const rso_handle* h);
/* stream is a cudaStream_t; NULL = the handle's own stream */
rso_status rso_set_stream(rso_handle* h, void* stream);
rso_status rso_synchronize(rso_handle* h);

/* element stiffness matrix (24x24 row-major, host); element/templateMatrix.cpp:31-124 */
rso_status rso_element_matrix(double E, double nu, double h, double* K0_host);

/* ---------------------------------------------------------------- topology */
/* HierarchyGrid::n_grid (grid/Grid.h:1000) */
int rso_n_levels(const rso_handle* h);
/* dims[0..2] element dims, dims[3..5] node dims of a level */
rso_status rso_level_dims(const rso_handle* h, int level, int* dims_host);
/* per-level element/vertex masks; elesatlist/vrtsatlist (grid/Grid.cpp:1011-1034) */
rso_status rso_level_masks(rso_handle* h, int level, uint8_t* emask_host, uint8_t* vmask_host);
/* per-level masks as 32-bit words, the BitSAT bit arrays (grid/Grid.h:116-158) */
rso_status rso_level_bitwords(rso_handle* h, int level, uint32_t* ebits_host, uint32_t* vbits_host);
/* BitSAT rank of every set bit and -1 elsewhere (gBitSAT operator(), culib/lib.cuh:1474-1550) */
rso_status rso_bitsat_rank(rso_handle* h, const uint32_t* words_dev, int64_t nbits, int32_t* rank_dev);
/* fine-level node classes: bit0 active, bit1 surface, bit2 support, bit3 load;
 * mark_surface_nodes_kernel (grid/Grid.cu:2824-2858) + computeProjectionMatrix */
rso_status rso_node_class(rso_handle* h, uint8_t* class_host);
/* reference compact numbering of a level: lexicographic vertex/element ids,
 * GS colour order padded to 32 per colour, flag words (padding -1).
 * compute_gscolor (grid/Grid.cu:1310-1385), enumerate_gs_subset
 * (grid/Grid.cpp:4187-4248), lexico2gsorder_g (grid/Grid.cu:1465-1495).
 * counts[4] = {n_vertices, n_elements, n_gs_vertices, n_gs_elements};
 * any output may be NULL (call once with NULL arrays to size them). */
rso_status rso_ref_numbering(rso_handle* h, int level, int* counts_host, int* gs_num_host,
                             int* vlexi2gs_host, int* elexi2gs_host, int* vflag_host, int* eflag_host);
/* load nodes (dense node ids) in the reference's order (sorted by GS id);
 * getLoadNodes (optimization/projection.cpp:272) */
rso_status rso_load_nodes(rso_handle* h, int* nodes_host, int* n_load);

/* ---------------------------------------------------------------- operator and multigrid */
/* element densities (ex*ey*ez floats, inactive entries ignored); Grid rho_e buffer */
rso_status rso_set_density(rso_handle* h, const float* rho_dev);
/* The current element densities (ex*ey*ez floats, device), the field
 * HierarchyGrid::writeDensity saves (grid/Grid.cpp:1267-1300, there as an
 * OpenVDB grid of element positions and values). */
rso_status rso_get_density(rso_handle* h, float* rho_dev);
/* Restart from saved densities: HierarchyGrid::readDensity (grid/Grid.cpp:
 * 1914-1945) with the points already read from the file: n element positions
 * (x, y, z per point, host) and their values (host); every other element gets
 * density 0.  A point outside the grid or on an inactive element is refused
 * with RSO_ERR_INVALID_ARG ("unmatched grid and file", where the reference
 * exits).  Then as rso_set_density (call rso_update_operators next). */
rso_status rso_set_density_points(rso_handle* h, int n, const int32_t* pos_host, const float* values_host);
/* Galerkin coarse operators and coarsest factorisation; update_stencil
 * (grid/Grid.cpp:4250-4261, grid/Grid.cu:882-1308, grid/Grid.cpp:3697-3752) */
rso_status rso_update_operators(rso_handle* h);
/* f = K(rho) u with support rows passing u; Grid::applyK (grid/Grid.cu:4358-4450) */
rso_status rso_apply_K(rso_handle* h, const double* u_dev, double* f_dev);
/* r = f - K u; Grid::update_residual (grid/Grid.cu:2463-2497) */
rso_status rso_residual(rso_handle* h, const double* u_dev, const double* f_dev, double* r_dev);
/* One sweep of the FP32 fine-level kernel that the mixed-precision V-cycle
 * runs (no counterpart in the reference, whose V-cycle is FP64 only; the
 * operator is update_residual_OTFA_WS_kernel grid/Grid.cu:2320-2376): the
 * FP64 inputs are rounded to FP32, op 0 gives r = f - K u, op 1 K u (support
 * rows pass u; f may be NULL), op 2 the damped block-Jacobi / Chebyshev step
 * u + c1 (u - uprev) + omega D^-1 (f - K u) (uprev NULL reads as zero), op 3
 * the first step from a zero iterate, omega D^-1 f (u is ignored); the FP32
 * result comes back widened to FP64. */
rso_status rso_fine_sweep_fp32(rso_handle* h, int op, const double* u_dev, const double* f_dev,
                               const double* uprev_dev, double omega, double c1, double* out_dev);
/* The same for a coarse level's FP32 stencil kernels (no counterpart in the
 * reference; its coarse levels are FP64, update_residual_kernel_1
 * grid/Grid.cu:2169-2267): op 0 r = f - K u, op 2 the Jacobi / Chebyshev step;
 * the kernel variant follows the handle's launch shapes. */
rso_status rso_coarse_sweep_fp32(rso_handle* h, int level, int op, const double* u_dev, const double* f_dev,
                                 const double* uprev_dev, double omega, double c1, double* out_dev);
/* FP32 prolongation out = uf + P uc (Grid::prolongate_correction,
 * grid/Grid.cu:2717-2734, in the precision of the mixed V-cycle). */
rso_status rso_prolong_fp32(rso_handle* h, int coarse_level, const double* uc_dev, const double* uf_dev,
                            double* out_dev);
/* FP32 restriction fc = R rf (Grid::restrict_residual, grid/Grid.cu:2615-2635,
 * in the precision of the mixed V-cycle). */
rso_status rso_restrict_fp32(rso_handle* h, int coarse_level, const double* rf_dev, double* fc_dev);
/* coarse-level stencil (243 x Nn_level doubles, [d][row][col][node]); rxStencil */
rso_status rso_get_stencil(rso_handle* h, int level, double* out_dev);
/* coarse residual on stored stencils; update_residual_kernel_1 (grid/Grid.cu:2169-2267) */
rso_status rso_coarse_residual(rso_handle* h, int level, const double* u_dev, const double* f_dev,
                               double* r_dev);
/* smoothing sweeps on a level (omega absolute for Jacobi); Grid::gs_relax (grid/Grid.cu:1887-1930) */
rso_status rso_smooth(rso_handle* h, int level, double* u_dev, const double* f_dev, int kind,
                      double omega, int sweeps, int reverse);
/* Grid::restrict_residual (grid/Grid.cu:2615-2635) */
rso_status rso_restrict(rso_handle* h, int coarse_level, const double* rf_dev, double* fc_dev);
/* Grid::prolongate_correction (grid/Grid.cu:2717-2734) */
rso_status rso_prolong(rso_handle* h, int coarse_level, const double* uc_dev, double* uf_dev);
/* coarsest dense solve; Grid::solve_fem_host (grid/Grid.cpp:4123-4185) */
rso_status rso_coarsest_solve(rso_handle* h, const double* f_dev, double* u_dev);
/* lambda_max(D^-1 K) estimate of a level used by damped Jacobi */
rso_status rso_level_lambda(rso_handle* h, int level, double* lambda);
/* one V-cycle updating u in place; HierarchyGrid::v_cycle (grid/Grid.cpp:2431-2476).
 * symmetric=1 reverses the post-smoothing order (needed for PCG). */
rso_status rso_vcycle(rso_handle* h, double* u_dev, const double* f_dev, int pre, int post,
                      int symmetric, double* rel_res);
/* solve K u = f to tol; u holds the initial guess.  method RSO_SOLVE_VCYCLE
 * repeats V-cycles (solveFEM, optimization/optimization.cpp:178-184),
 * RSO_SOLVE_PCG runs CG preconditioned by one V-cycle: FP64 throughout, or in
 * mixed mode an FP32 V-cycle and (rso_set_krylov_fp32) an FP32 recurrence with
 * FP64 iterate and residual replacement. */
rso_status rso_solve(rso_handle* h, const double* f_dev, double* u_dev, double tol, int max_iter,
                     int method, rso_solve_info* info);
/* k systems K u_i = f_i on the same operator solved together (load cases of
 * one design; no counterpart in the reference, which solves them one after
 * the other): one PCG recurrence per system with per-system scalars, every
 * V-cycle kernel launch carrying all k systems.  F_dev, U_dev: k * 3*Nn
 * doubles, system-major (U holds the initial guesses and returns the
 * solutions); infos: k entries or NULL.  1 <= k <= 64; damped Jacobi or
 * Chebyshev smoother (Gauss-Seidel returns RSO_ERR_UNSUPPORTED).  Device
 * buffers for k systems are allocated on the first call with that k and kept. */
rso_status rso_solve_batch(rso_handle* h, int k, const double* F_dev, double* U_dev, double tol, int max_iter,
                           rso_solve_info* infos);
/* Launch-shape autotuner (no counterpart in the reference, whose launch
 * shapes are fixed): times, on this handle's hierarchy with CUDA events, the
 * thread rows of the packed FP32 fine kernel (2, 4 or 8), one thread per node or
 * per (node, row) on every coarse level, the z chunk of the fine kernel, and
 * the first level and kind of the bottom kernel (or none), each timed as
 * mixed-precision solves of a random load, and keeps the fastest for this
 * handle (a candidate must beat the built-in rule by 3 %).  The candidates compute the same arithmetic.  Needs
 * rso_update_operators first, mixed precision and a Jacobi or Chebyshev
 * smoother; overwrites the solver's work vectors; takes a few dozen solves.  choices_host (NULL or
 * 2 + number of levels ints): fine rows, bottom level (-1 none; its kind is
 * read with rso_bottom_kernel), then per level 0 = node per thread, 1 = row
 * split, 2 = nine per node, -1 not tuned. */
rso_status rso_autotune(rso_handle* h, int* choices_host);
/* Sets the launch shapes directly, in rso_autotune's format (n >= 2 ints;
 * bottom level -2 restores the built-in size rule, a row-split entry of -1
 * too), e.g. to reuse choices measured once for many handles.  The built-in
 * bottom rule, for the FP32 V-cycle of mixed precision with bottom kernel
 * kind 1: the persistent kernel from the first coarse level of at most 60,000
 * nodes above the coarsest. */
rso_status rso_set_launch_shapes(rso_handle* h, const int* choices_host, int n);
/* Node planes per z chunk of the packed FP32 fine kernel (4, 8, 16 or 32; 0
 * restores the size rule: the longest chunk that gives the grid 4 CTAs per
 * SM).  A CTA marches its chunk plane by plane and re-reads the plane below
 * it, so short chunks fill the GPU on small grids at the price of that plane;
 * rso_autotune measures the lengths.  rso_fine_zchunk returns the length in
 * use. */
rso_status rso_set_fine_zchunk(rso_handle* h, int planes);
int rso_fine_zchunk(const rso_handle* h);
/* Kernel of the bottom of the FP32 V-cycle, when the launch shapes give it a
 * first level (no counterpart in the reference, which launches every level's
 * kernels): kind 1 (default) one persistent cooperative kernel over the whole
 * GPU, every CTA resident at once, its phases (sweeps, residuals, transfers,
 * the coarsest solve) separated by a grid-wide barrier whose waits give up
 * after about 2 s (the solve then fails with RSO_ERR_CUDA); kind 0 one kernel
 * on an 8-CTA thread-block cluster.  rso_autotune measures both;
 * rso_bottom_kernel returns the kind in use. */
rso_status rso_set_bottom_kernel(rso_handle* h, int kind);
int rso_bottom_kernel(const rso_handle* h);
/* Self-test of the persistent kernel's bounded barrier wait (no counterpart in
 * the reference): a cooperative launch of 4 CTAs passes 8 grid barriers whose
 * arrival target is the grid plus short_by (0 or 1); with short_by = 1 no
 * barrier completes, every wait gives up after limit_ms (0 < limit_ms <= 1000)
 * and the kernel returns.  *gave_up receives whether a wait gave up; the
 * barrier state is reset afterwards, so the handle stays usable.  No fault and
 * no hang either way. */
rso_status rso_grid_barrier_selftest(rso_handle* h, int short_by, double limit_ms, int* gave_up);
/* Replay of the FP32 V-cycle (the mixed-precision preconditioner) from CUDA
 * graphs (no counterpart in the reference, which launches every kernel):
 * on by default.  The V-cycle is captured the second time its launch
 * arguments (level vectors, sizes, smoother step sizes, configuration,
 * profiling mask) occur and replayed whenever they recur; the results are
 * the same launches with the same arguments.  A capture needs a stream of the
 * handle's own or one set by rso_set_stream other than the legacy default
 * stream; if a capture fails the handle keeps to plain launches. */
rso_status rso_set_vcycle_graphs(rso_handle* h, int on);
/* Device-controlled solves (no counterpart in the reference): with on != 0
 * the mixed-precision PCG loop with the FP32 recurrence runs as one CUDA
 * graph per solve: 16 unrolled iterations, each of conditional IF nodes for
 * the iteration (q = K p, the residual update), the FP64 residual
 * replacement, and the V-cycle with the direction update (a straight-line
 * graph: a launch ends whatever the device decides); the decisions the
 * host takes between iterations otherwise (replace, stop, stall) are taken by
 * one-thread kernels on the same scalars, so the iterations, iterates and
 * residuals are those of the host-driven loop.  Used when the V-cycle graphs
 * are on and per-kernel profiling is off; a failed capture falls back to the
 * host-driven loop.  Off by default. */
rso_status rso_set_solve_graphs(rso_handle* h, int on);
/* Krylov recurrence of the mixed-precision PCG (no counterpart in the
 * reference, whose CG is FP64).  0 < replace_factor < 1 (1e-2 by default in
 * mixed precision): the recurrence runs in FP32 (FP32 operator, FP32
 * vectors, FP64 sums and FP64 iterate) and the true FP64 residual f - K x
 * replaces the recursive one whenever that has dropped by replace_factor
 * since the last replacement and before the solve stops, so the tolerance is
 * always met by a true FP64 residual; a cycle between replacements lasts at
 * most 30 iterations, and one that does not bring the true residual below
 * max(0.5, sqrt(replace_factor), sqrt(claimed)) of the previous one (claimed:
 * the reduction the recursive residual showed over that cycle) hands the solve
 * over to the FP64 recurrence from the current iterate, iterations counted on.
 * replace_factor 0: p, q = K p and r are FP64 and only the V-cycle is FP32.
 * rso_solve_batch follows the same setting, each system replacing its
 * residual on its own rule; a hand-over there moves the whole batch to the
 * FP64 recurrence, so systems still converging in FP32 leave the sequence of
 * their own single solves from that point (same tolerance, true residuals). */
rso_status rso_set_krylov_fp32(rso_handle* h, double replace_factor);
/* Upper bound on the replacement cycles of the FP32 recurrence (no
 * counterpart in the reference): after max_cycles replacements that did not
 * end the solve, it continues with the FP64 recurrence from the current
 * iterate, as after a stall (0, the default: no bound).  Caps the FP32 work a
 * solve may spend before the FP64 recurrence takes over. */
rso_status rso_set_krylov_fp32_cycles(rso_handle* h, int max_cycles);
/* Grid::compliance (grid/Grid.cpp:4118-4121): c = f . u */
rso_status rso_dot(rso_handle* h, const double* a_dev, const double* b_dev, double* out);

/* ---------------------------------------------------------------- design variables and sensitivities */
/* dC/drho_e = -p rho^(p-1) u_e^T K0 u_e; computeSensitivity_kernel (optimization/optimization.cu:102-165) */
rso_status rso_sensitivity(rso_handle* h, const double* u_dev, float* sens_dev);
/* rho^p u_e^T K0 u_e; elementCompliance_kernel (grid/Grid.cu:5569-5610) */
rso_status rso_element_energy(rso_handle* h, const double* u_dev, float* energy_dev);
/* rho_out = clamp(H_beta(rho_in), rho_min, 1), shell -> 1; computeProjection_kernel
 * (optimization/optimization.cu:324-348) */
rso_status rso_heaviside(rso_handle* h, const float* rho_in_dev, double beta, const uint8_t* shell_dev,
                         float* rho_out_dev);
/* g_out = g_in * H'(rho_in); computeProjectionSensitivity_kernel (optimization/optimization.cu:167-189) */
rso_status rso_heaviside_chain(rso_handle* h, const float* rho_in_dev, double beta, const float* g_in_dev,
                               float* g_out_dev);
/* sensitivity filter; filterSensitivity_kernel (grid/Grid.cu:4210-4326) */
rso_status rso_filter(rso_handle* h, double radius, const float* in_dev, float* out_dev);
/* consistent density filter (same weights) and its adjoint (build mode) */
rso_status rso_density_filter(rso_handle* h, double radius, const float* in_dev, float* out_dev);
rso_status rso_density_filter_adjoint(rso_handle* h, double radius, const float* in_dev, float* out_dev);
/* The sensitivity filter of rso_filter, computed without any device memory
 * allocation; it has no counterpart in the reference.  rso_filter keeps its
 * tap table in a device allocation of the handle, made on its first call and
 * again whenever the radius grows; this entry point never allocates, not
 * even on first use: it keeps the table in a fixed array of the library (52,728 bytes
 * per device), for callers that cannot allocate device memory inside their
 * loop: all free memory already handed to their own pool, a fixed device
 * footprint, or no room for the pool growth and synchronisation an allocation
 * can bring.  Limits: int(radius + 0.5) <= RSO_FILTER_NOALLOC_MAX_REACH
 * (radius < 6.5); larger radii return RSO_ERR_INVALID_ARG with a message.
 * The first call on a device looks the array up on that device (this may
 * load the module there), so make it before any stream capture.  All calls
 * on one device share the array: each call rewrites the entries it reads,
 * and calls that overlap on one device (other threads or unordered streams)
 * race and must be serialised by the caller.  Synchronises h's stream. */
#define RSO_FILTER_NOALLOC_MAX_REACH 6
rso_status rso_filter_noalloc(rso_handle* h, double radius, const float* in_dev, float* out_dev);
/* Optimality-criteria density update (the reference's alternative to MMA):
 * variant 0 is updateDensities (optimization/optimization.cu:394-471),
 * variant 1 updateDensities2 (:473-598, built without ENABLE_HEAVISIDE, as the
 * reference's build is).  Bisection on the sensitivity threshold g in
 * [0, max |sens|] of rho' = clamp(clamp(rho (|min(sens, 0)| / g)^damp,
 * rho - step, rho + step), rho_min, 1) (trySensMultiplier_kernel :366-392),
 * shell elements 1, until the volume fraction over the active elements is
 * within 1e-4 of vgoal or after 31 trials (variant 1: also stops when the
 * bracket's relative width is below 1e-3, at most 51 trials).  rho_out =
 * the update at the last threshold (may alias rho_src).  Dense element
 * arrays; info_host (NULL or 5 doubles): g, final volume, trials, max and
 * mean |rho_out - rho_src|. */
rso_status rso_oc_update_density(rso_handle* h, int variant, const float* rho_src_dev, const float* sens_dev,
                                 const uint8_t* shell_dev, double vgoal, double step, double damp, float* rho_out_dev,
                                 double* info_host);
/* Optimality-criteria update of the spline coefficients, updateCoeff
 * (optimization/optimization.cu:600-706, tryCSensMultiplier_kernel :560-598):
 * the same bisection on the coefficient sensitivities with the coefficients
 * clamped to [cmin, cmax] and the volume of coeff2density of each trial; as in
 * the reference the final threshold is applied to the last trial's
 * coefficients.  coeff_dev (n_coeff floats) is updated in place; rho_out_dev
 * (NULL or ex*ey*ez floats) receives the final densities; info_host (NULL or 3
 * doubles): g, final volume, trials. */
rso_status rso_oc_update_coeff(rso_handle* h, float* coeff_dev, const float* csens_dev, double vgoal, double step,
                               double damp, double cmin, double cmax, float* rho_out_dev, double* info_host);
/* volume fraction sum(rho)/n_gs_elements; Grid::volumeRatio (grid/Grid.cu:5642-5650) */
rso_status rso_volume(rso_handle* h, const float* rho_dev, double* vol);

/* B-spline map: HierarchyGrid::set_spline_partition (grid/Grid.cu:3187-3256),
 * Grid::set_spline_knot_series (grid/Grid.cpp:3307-3431).  Returns n_coeff. */
rso_status rso_spline_setup(rso_handle* h, int order, int px, int py, int pz, int* n_coeff);
/* per-axis tables: first-knot index (-1 outside) and order basis values/derivatives (host) */
rso_status rso_spline_axis(rso_handle* h, int axis, int* idx_host, double* N_host, double* dN_host);
/* Grid::coeff2density (grid/Grid.cu:3405-3536) */
rso_status rso_coeff2density(rso_handle* h, const float* coeff_dev, const uint8_t* shell_dev,
                             float* rho_hat_dev);
/* race-free adjoint; Grid::ddensity2dcoeff (grid/Grid.cu:3566-3721),
 * ddensity2dcoeff_update (:3723-3828), dvol2dcoeff (:3830-3939) */
rso_status rso_density2coeff_adjoint(rso_handle* h, const float* g_dev, const uint8_t* shell_dev,
                                     float* dc_dev);
/* self-support constraint on element centres; deal_background_points
 * (optimization/optimization.cpp:1223-1242) -> grid/Grid.cu:7449-8250.
 * per_element (ex*ey*ez) and dc (n_coeff, already divided by the count) may be NULL. */
rso_status rso_selfsupport(rso_handle* h, const float* coeff_dev, double beta, int mode, double opt_angle,
                           double default_angle, float* per_element_dev, float* dc_dev, double* value,
                           double* count, double* direction_sum);

/* ---------------------------------------------------------------- surface-point self-support
 * deal_surface_points (optimization/optimization.cpp:1185-1221).  Points are
 * element-unit coordinates, SoA (x[0..n), y[0..n), z[0..n)). */
typedef struct rso_surface_info {
  long long n_crossings;   /* background-grid edges crossing rho = 0.5 */
  long long n_first_pick;  /* candidates after the first equal-distance pick */
  long long n_in_model;    /* candidates inside an active element */
  int n_points;            /* points kept (= n_points requested) */
  int reserved;
} rso_surface_info;
/* Grid::generate_spline_surface_nodes (grid/Grid.cpp:4067-4112) with
 * compute_background_mcPoints_value (grid/Grid.cu:4066-4175) and
 * compute_surface_nodes_in_model (grid/Grid.cpp:3861-4060): the crossings of
 * rho = 0.5 on the (mc_res+2)^3 background grid of the model box (NULL: the
 * bounding box of the active elements; else {xmin, ymin, zmin, xmax, ymax,
 * zmax}), one per crossing grid edge in edge order, thinned to n_points as the
 * reference does.  The points stay on the handle. */
rso_status rso_surface_points(rso_handle* h, const float* coeff_dev, int mc_res, int n_points,
                              const float* model_box_host, rso_surface_info* info);
/* Grid::uploadSurfacePoints: use the given points (3 n floats, device or host) */
rso_status rso_set_surface_points(rso_handle* h, const float* xyz, int n_points);
/* copy the points out (3 n floats; xyz may be NULL to query n) */
rso_status rso_get_surface_points(rso_handle* h, float* xyz, int capacity, int* n_points);
/* compute_spline_surface_point_normal .. scale_spline_selfsupp_constraint_dcoeff
 * (grid/Grid.cu:5709-6505, grid/Grid.cpp:4263-4280): normals, orientation,
 * flags, the per-point constraint of GlobalSSMode `mode` (p-norm 8,
 * h-function 10, sigmoid 0.09), its mean (p-norm: (mean)^(1/8) - 1) and its
 * coefficient gradient divided by the count.  per_point (n) and dc (n_coeff)
 * may be NULL. */
rso_status rso_surface_selfsupport(rso_handle* h, const float* coeff_dev, double beta, int mode,
                                   double opt_angle, double default_angle, float* per_point_dev,
                                   float* dc_dev, double* value, double* count, double* direction_sum);
/* outward normals of the last evaluation (3 n doubles, SoA) and the flags
 * (2 n bytes: at the default angle, compute_selfsupp_flag_actual
 * grid/Grid.cu:5945-5992, then at the optimisation angle, :5994-6040);
 * either may be NULL */
rso_status rso_get_surface_normals(rso_handle* h, double* normals, uint8_t* flags);

/* ---------------------------------------------------------------- worst case */
/* forceProject (optimization/projection.cu:165-231, projection.cpp:289-360):
 * forces kept on the load nodes, only along the load normal in
 * constrained-direction mode, and in support-free modes without the rigid
 * motions of the load set (orthonormal, nearly dependent motions dropped) */
rso_status rso_force_project(rso_handle* h, double* f_dev, int constrain_direction);
/* displacementProject (optimization/projection.cpp:374-411): u minus its
 * projection on the rigid motions of the active fine nodes; a no-op for
 * problems with supports */
rso_status rso_displacement_project(rso_handle* h, double* u_dev);
/* worst-case load: lambda_max of P K^-1 P by Lanczos with full FP64
 * reorthogonalisation, one multigrid solve (to tol) per step.  Replaces
 * modifiedPM (optimization/optimization.cpp:215-353).  ritz_host may be NULL. */
rso_status rso_worst_case(rso_handle* h, int steps, int constrain_direction, double tol, uint64_t seed,
                          double* f_worst_dev, double* u_worst_dev, double* lambda, double* ritz_host);
/* the reference's modified power method itself (optimization/optimization.cpp:215-353) */
rso_status rso_modified_pm(rso_handle* h, int constrain_direction, uint64_t seed, int max_itn,
                           double* f_dev, double* u_dev, double* c_worst, int* itn);

/* ---------------------------------------------------------------- MMA */
/* MMA::mma_t (optimization/mma_t.h:159-266) in FP64 on the device */
rso_status rso_mma_create(int n, int m, const double* xmin_host, const double* xmax_host, rso_mma** out);
/* start from a given design (host); the reference starts from the box midpoint */
rso_status rso_mma_set_x(rso_mma* s, const double* x_host);
/* the same from a device array (n doubles) */
rso_status rso_mma_set_x_dev(rso_mma* s, const double* x_dev);
rso_status rso_mma_get(rso_mma* s, double* x_host, double* L_host, double* U_host, double* alpha_host,
                       double* beta_host);
/* device x (n doubles) of the current design */
const double* rso_mma_x_dev(rso_mma* s);
/* mma_t::update(df, dg, g) (optimization/mma_t.cpp:18-51, mma_t.cu:330-499).
 * df_dev: n doubles, dg_dev: m*n doubles (constraint-major), g_host: m doubles.
 * info_host[4] = {kkt inf-norm, last step, sub-iterations, overflowed}. */
rso_status rso_mma_update(rso_mma* s, const double* df_dev, const double* dg_dev, const double* g_host,
                          int* converged, double* info_host);
/* Checkpoint and resume of the MMA state (no counterpart in the reference,
 * whose drivers restart MMA from scratch): what one update carries to the
 * next, x, the asymptotes L and U, the move limits alpha and beta, the
 * previous step and the stop counter, as 6 n + 1 doubles in that order.
 * Loading a saved state into an MMA of the same n and bounds continues the
 * run exactly as if it had not stopped. */
rso_status rso_mma_state_size(const rso_mma* s, long long* n_doubles);
rso_status rso_mma_save(rso_mma* s, double* state_host);
rso_status rso_mma_load(rso_mma* s, const double* state_host);
void rso_mma_destroy(rso_mma* s);

/* ---------------------------------------------------------------- design iteration */
typedef struct {
  double beta;             /* Heaviside sharpness */
  double volume_ratio;     /* V* */
  double filter_radius;    /* sensitivity filter radius (elements) */
  int filter_mode;         /* 0 reference sensitivity filter, 1 none */
  int lanczos_steps;
  double solve_tol;        /* relative residual of each multigrid solve */
  int constrain_direction; /* 1: cf mode, 0: ff mode */
  int ss_mode;             /* GlobalSSMode, -1 disables the self-support constraint */
  double opt_angle, default_angle;
  double sens_scale, vol_scale, ss_scale;  /* driver scalings (optimization.cpp:1008-1024) */
  uint64_t seed;
  /* self-support variant: 0 evaluates it on the background elements
   * (deal_background_points, optimization/optimization.cpp:1223-1242); n > 0
   * on n surface points sampled from a ss_mc_res^3 background grid of the
   * active elements' bounding box (deal_surface_points, :1185-1221) */
  int ss_points;
  int ss_mc_res;
} rso_iter_params;

typedef struct {
  double c_worst, lambda, volume, ss_value;
  double ms_total, ms_operators, ms_worst, ms_adjoint, ms_selfsupport, ms_mma;
  int solve_iterations;
  int mma_converged;
} rso_iter_info;

void rso_default_iter_params(rso_iter_params* p);
/* one robust spline design iteration: coefficients -> density -> Heaviside ->
 * operators -> worst case -> self-support -> adjoint chain -> MMA update of
 * the coefficients (optimization_ss loop body, optimization/optimization.cpp:859-1075).
 * The coefficients live in the MMA state (rso_mma_x_dev). */
rso_status rso_design_iteration(rso_handle* h, rso_mma* mma, const rso_iter_params* prm, rso_iter_info* info);
/* the same call with host buffers: copies coeff_host in, runs the iteration
 * and copies the updated coefficients and the density field out. */
rso_status rso_design_iteration_host(rso_handle* h, rso_mma* mma, const rso_iter_params* prm,
                                     const double* coeff_in_host, double* coeff_out_host,
                                     float* rho_out_host, rso_iter_info* info);
/* Objective values and coefficient gradients of the design at coeff_dev
 * (n_coeff doubles on the device), without an MMA step: values_host[3] =
 * {lambda_max of the worst case, volume fraction, self-support value} and
 * their gradients with respect to the coefficients (device, n_coeff doubles
 * each, any may be NULL).  This is the objective/gradient part of the
 * optimization_ss loop body (computeSensitivity2,
 * optimization/optimization.cu:249-322, and deal_background_points,
 * optimization/optimization.cpp:1223-1242), unscaled.  With
 * prm->filter_mode == 1 (no sensitivity filter) the gradients are exact. */
rso_status rso_design_gradient(rso_handle* h, const double* coeff_dev, const rso_iter_params* prm,
                               double* values_host, double* dlambda_dc_dev, double* dvolume_dc_dev,
                               double* dss_dc_dev);

/* ---------------------------------------------------------------- instrumentation */
/* Number of kernels this library has launched in the process (all handles).
 * The reference has no counterpart (it prints tictoc timers, utils/tictoc.h:78-80). */
long long rso_launch_count(void);
/* CUDA-event timing of the operator kernels on the handle's stream
 * (replaces the _TIC/_TOC phase timers of test_vcycle, grid/Grid.cpp:2349-2388) */
rso_status rso_set_profiling(rso_handle* h, int on);
/* the same for a subset of kernel classes (bit cls of mask), so that a timed
 * run can record only the kernel whose roofline it reports */
rso_status rso_set_profiling_classes(rso_handle* h, unsigned mask);
rso_status rso_profile_reset(rso_handle* h);
/* per kernel class: launches, total device ms, algorithmic bytes and flops per launch */
rso_status rso_profile_class(rso_handle* h, int cls, char* name, int name_len, long long* launches,
                             double* total_ms, double* bytes_per_launch, double* flops_per_launch);
/* the class with the largest total device time */
rso_status rso_profile_top(rso_handle* h, char* name, int name_len, long long* launches, double* total_ms,
                           double* bytes_per_launch, double* flops_per_launch);

#ifdef __cplusplus
}
#endif
#endif /* RSO_H */
