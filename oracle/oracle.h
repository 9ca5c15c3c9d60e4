/*
 * FP64 CPU oracle for the voxel-FEM worst-case topology-optimisation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library restates the reference method
 * (NanXYZH/RobustOptSpline3D) on the CPU in double precision so that the
 * CUDA path can be checked against it.  Only tests, the smoke check and the
 * CPU-baseline leg of bench.py may load it; the product library never does.
 *
 * Parity pinning: the reference ships no golden vectors and cannot be built
 * here (Eigen/CGAL/OpenVDB/gflags/MATLAB absent, no main()).  The oracle is
 * pinned by the known-answer checks the reference itself carries:
 *   - K0 rigid-mode null space (element/templateMatrix.cpp:105-123),
 *   - K * rigid motion == 0   (optimization/optimization.cpp:1167-1179),
 *   - BitSAT rank property    (optimization/optimization.cu:712-765),
 *   - V-cycle convergence     (grid/Grid.cpp:2311-2390),
 *   - power method vs dense aggregated eigenproblem
 *                             (utils/test_utils.cpp:2598-2645, 2859-2928),
 *   - MMA analytic problems   (optimization/mma_t.cpp:167-486),
 * plus an independent scipy.sparse assembly in the tests.  Everything else
 * (e.g. the coarsest-grid solve, whose reference uses Eigen BDCSVD) is
 * "parity unpinned" beyond those properties.
 *
 * Layout (shared with the CUDA path's dense-box layout):
 *   elements  e = x + ex*(y + ey*z)           (ex*ey*ez)
 *   nodes     n = x + nx*(y + ny*z), nx=ex+1  (nx*ny*nz)
 *   vectors   SoA  v[c*Nn + n], c in {0,1,2}
 *   stencils  s[(d*9 + r*3 + c)*Nn + n], d = (dx+1)+3(dy+1)+9(dz+1)
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_problem or_problem;

/* element stiffness matrix, 24x24 row-major; element_templateMatrix.cpp:31-124 */
void or_k0(double E, double nu, double h, double* K0);

/* problem set-up.  emask: ex*ey*ez bytes (1 = active element).
 * fixed_area / load_area: node masks (nx*ny*nz bytes) standing in for the
 * reference's _inFixedArea/_inLoadArea predicates (Grid.cpp:2715-2745).
 * load_normals: 3*Nn doubles (unit outward normals; used in cf modes).
 * n_levels: 0 = reference policy (coarsen while active elements > 400).
 * first_factor: 4 = reference skip-layer-1 hierarchy, 2 = dyadic. */
or_problem* or_create(int ex, int ey, int ez, const uint8_t* emask,
                      const uint8_t* fixed_area, const uint8_t* load_area,
                      const double* load_normals,
                      double E, double nu, double penal, double rhomin,
                      int n_levels, int first_factor);
void or_destroy(or_problem* p);

int  or_n_levels(const or_problem* p);
/* dims[0..2] = element dims, dims[3..5] = node dims */
void or_level_dims(const or_problem* p, int level, int* dims);
void or_level_masks(const or_problem* p, int level, uint8_t* emask, uint8_t* vmask);
/* reference word-level bit masks of one level (uint32 words, lexicographic) */
int  or_level_bitwords(const or_problem* p, int level, uint32_t* ebits, uint32_t* vbits);
/* node classes at level 0: bit0 active, bit1 surface, bit2 support, bit3 load */
void or_node_class(const or_problem* p, uint8_t* out);
/* reference compact numbering of one level (Grid.cpp:2973-3215, 4187-4248).
 * Returns n_gs_vertices; fills counts[0]=n_vertices, counts[1]=n_elements,
 * counts[2]=n_gs_vertices, counts[3]=n_gs_elements, gs_num[8] (vertex colour
 * set sizes padded to 32), vlexi2gs[n_vertices], elexi2gs[n_elements],
 * vflag_gs[n_gs_vertices], eflag_gs[n_gs_elements] (padding = -1).
 * Any output pointer may be NULL. */
int  or_ref_numbering(const or_problem* p, int level, int* counts, int* gs_num,
                      int* vlexi2gs, int* elexi2gs, int* vflag_gs, int* eflag_gs);
/* load nodes (dense node index), sorted by reference gs id as setLoadNodes does */
int  or_load_nodes(const or_problem* p, int* nodes);

void or_set_density(or_problem* p, const double* rho);       /* ex*ey*ez */
void or_apply_K(const or_problem* p, const double* u, double* f);
void or_residual(const or_problem* p, const double* u, const double* f, double* r);

void or_update_stencil(or_problem* p);
/* lambda_max(D^-1 K) estimate of a level (damped Jacobi uses omega*2/lambda) */
double or_level_lambda(const or_problem* p, int level);
void or_get_stencil(const or_problem* p, int level, double* out);
void or_coarse_residual(const or_problem* p, int level, const double* u, const double* f, double* r);

/* smoother: kind 0 = 8-colour Gauss-Seidel (reference), 1 = damped block Jacobi
 * (omega absolute here; or_vcycle/or_solve take omega relative to 2/lambda_max) */
void or_smooth(const or_problem* p, int level, double* u, const double* f,
               int kind, double omega, int sweeps, int reverse_colours);
void or_restrict(const or_problem* p, int coarse_level, const double* rf, double* fc);
void or_prolong(const or_problem* p, int coarse_level, const double* uc, double* uf);
/* coarsest dense solve */
void or_coarsest_solve(const or_problem* p, const double* f, double* u);

/* one V-cycle with the reference's sequencing (Grid.cpp:2431-2476).
 * u is updated in place; returns ||f - K u|| / ||f||. */
double or_vcycle(or_problem* p, double* u, const double* f, int pre, int post,
                 int kind, double omega, int symmetric);
/* solve K u = f.  method 0 = repeated V-cycles, 1 = V-cycle preconditioned CG.
 * returns iterations; *rel_res receives the final relative residual. */
int or_solve(or_problem* p, double* u, const double* f, double tol, int max_iter,
             int method, int pre, int post, int kind, double omega, double* rel_res);

/* compliance sensitivity dC/drho_e = -p rho^(p-1) u_e^T K0 u_e (optimization.cu:102-165) */
void or_sensitivity(const or_problem* p, const double* u, double* sens);
void or_element_energy(const or_problem* p, const double* u, double* energy);

/* Heaviside projection (optimization.cu:324-348) and its chain (167-189) */
void or_heaviside(int n, const double* rho_in, double beta, double rhomin,
                  const uint8_t* shell, double* rho_out);
void or_heaviside_chain(int n, const double* rho_in, double beta,
                        const double* g_in, double* g_out);
/* sensitivity filter (Grid.cu:4210-4309) on the active elements */
void or_filter(const or_problem* p, double radius, const double* in, double* out);
/* consistent density filter (build mode) and its adjoint */
void or_density_filter(const or_problem* p, double radius, const double* in, double* out);
void or_density_filter_adjoint(const or_problem* p, double radius, const double* in, double* out);

/* B-spline map (Grid.cu:427-509, 3405-3939; Grid.cpp:3307-3431) */
int  or_spline_setup(or_problem* p, int order, int px, int py, int pz);
void or_spline_info(const or_problem* p, int* nbasis, float* bmin, float* step);
/* per-axis element tables: span index (int) and order basis values / derivatives */
void or_spline_axis(const or_problem* p, int axis, int* idx, double* N, double* dN);
void or_coeff2density(const or_problem* p, const double* c, double rhomin,
                      const uint8_t* shell, double* rho_hat);
void or_density2coeff_adjoint(const or_problem* p, const double* g,
                              const uint8_t* shell, double* dc);

/* self-support constraint on element centres (Grid.cu:7449-8250).
 * mode = GlobalSSMode (0..5); angles in radians.  Returns the global value;
 * dc (n_coeff) receives its gradient already divided by the count. */
double or_selfsupport(const or_problem* p, const double* c, double beta, int mode,
                      double opt_angle, double default_angle, double* per_element,
                      double* dc, double* count_out, double* direction_sum);

/* surface-point self-support (or_surface.cpp; grid/Grid.cu:4066-4175,
 * :5709-6505, grid/Grid.cpp:3831-4112).  box = {xmin, ymin, zmin, xmax, ymax,
 * zmax} in element units.  or_mc_values fills (mc+2)^3 background values
 * (x fastest) and, if pos3 is not NULL, their coordinates (SoA); or_equidistant the clamped equal-distance picks (returns their
 * number); or_surface_points writes npts points (SoA, 3*npts) and info[4] =
 * {crossings, after the first pick, inside the model, written}. */
void or_mc_values(const or_problem* p, const double* c, int mc, const float* box, float* val, float* pos3);
long or_equidistant(long range, long m, long* out);
int  or_surface_points(const or_problem* p, const double* c, int mc, int npts, const float* box,
                       float* xyz, long* info);
/* normals (3n SoA), per (n), flags (2n: actual, virtual) and dc (n_coeff,
 * divided by the count) may be NULL; returns the constraint value */
double or_surface_selfsupport(const or_problem* p, const double* c, const float* xyz, long n, double beta,
                              int mode, double opt_angle, double default_angle, double* normals,
                              double* per, uint8_t* flags, double* dc, double* count_out,
                              double* dirsum_out);

/* worst-case machinery */
void or_force_project(const or_problem* p, double* f, int constrain_direction);
/* displacementProject (optimization/projection.cpp:374-411): u -= R R^T u over
 * the rigid motions of the active fine nodes; a no-op with supports */
void or_displacement_project(const or_problem* p, double* u);
/* iterations of all solves on this problem so far */
long or_solve_iterations(const or_problem* p);
int  or_n_load(const or_problem* p);
/* dense aggregated worst case: lambda_max of P K^-1 P on the load space and
 * the worst unit force (utils/test_utils.cpp:2598-2645, 2859-2928) */
double or_dense_worst(or_problem* p, int constrain_direction, double tol,
                      double* f_worst, double* u_worst);
/* Lanczos with full reorthogonalisation; start vector from seed */
double or_lanczos(or_problem* p, int steps, int constrain_direction, double tol,
                  uint64_t seed, double* f_worst, double* u_worst, double* ritz);
/* the reference's modified power method (optimization.cpp:215-353) */
double or_modified_pm(or_problem* p, int constrain_direction, uint64_t seed,
                      int max_itn, double* f_out, double* u_out, int* itn_out);

/* MMA (optimization/mma_t.*) in double precision */
typedef struct or_mma or_mma;
or_mma* or_mma_create(int n, int m, const double* xmin, const double* xmax);
void    or_mma_set_x(or_mma* s, const double* x);
void    or_mma_get(or_mma* s, double* x, double* L, double* U, double* alpha, double* beta);
int     or_mma_update(or_mma* s, const double* df, const double* dg, const double* g,
                      double* info);
void    or_mma_destroy(or_mma* s);

#ifdef __cplusplus
}
#endif
