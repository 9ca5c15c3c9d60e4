// Internal state of the FP64 CPU oracle (test infrastructure only).
#pragma once
#include "oracle.h"
#include <vector>
#include <cstdint>
#include <cmath>
#include <cstring>
#include <algorithm>

namespace orc {

struct Level {
  int ex = 0, ey = 0, ez = 0, nx = 0, ny = 0, nz = 0;
  long ne = 0, nn = 0;
  int factor = 0;                 // coarsening factor from the finer level (0 at level 0)
  std::vector<uint8_t> emask, vmask;
  std::vector<double> KE;         // coarse element matrices (576 per element), levels >= 1
  std::vector<double> stencil;    // 243 * nn, levels >= 1
  long eidx(int x, int y, int z) const { return x + (long)ex * (y + (long)ey * z); }
  long nidx(int x, int y, int z) const { return x + (long)nx * (y + (long)ny * z); }
};

}  // namespace orc

struct or_problem {
  std::vector<orc::Level> L;
  double E = 1e6, nu = 0.3, penal = 3, rhomin = 1e-3;
  double K0[576];
  std::vector<uint8_t> fixed_area, load_area, surface, support, load;
  std::vector<double> normals;
  std::vector<double> rho, rhop;          // per fine element (box)
  std::vector<int> load_nodes;            // dense node ids (sorted by reference gs id)
  // support-free problems (no support node): rigid motions, orthonormal
  bool has_support = true;
  std::vector<double> rigid_full;         // 3 nn x 6 over the active fine nodes, row (c nn + n), col-major by mode
  std::vector<double> rigid_load[2];      // load space 3 nl x k[cf], ff (0) and normal-projected cf (1)
  int rigid_k[2] = {0, 0};
  std::vector<double> rigid_coarse;       // 3 nc x 6 over the coarsest active nodes (row 3 i + c)
  // coarsest dense solve
  std::vector<long> cnode;                // active coarsest nodes
  std::vector<long> crow;                 // node -> row block (-1 absent)
  std::vector<double> Kinv;               // dense inverse (3nc x 3nc)
  int nc = 0;
  long solve_iters = 0;                   // iterations of every or_solve so far (bench statistics)
  std::vector<double> lam;                // lambda_max(D^-1 K) estimate per level
  // spline
  int order = 0, part[3] = {0, 0, 0}, nb[3] = {0, 0, 0};
  float bmin[3], bmax[3], step[3];
  std::vector<float> knots[3];
  std::vector<int> sidx[3];               // per element coordinate: first-knot index i (reference "i")
  std::vector<double> sN[3], sdN[3];      // order values per coordinate
  std::vector<uint8_t> sinside[3];
};

namespace orc {
void build_topology(or_problem* p, int n_levels, int first_factor);
void galerkin(or_problem* p);
void coarsest_factor(or_problem* p);
double dot3(const double* a, const double* b, long nn);
// rigid motions of the given node positions (6 columns, rows 3 k + c for
// node k): translations then rotations p^ (projection.cpp:58-75), turned
// orthonormal by modified Gram-Schmidt in column order; with `drop`, columns
// whose residual falls below 1e-6 of their norm are removed
// (projection.cpp:235-262).  Returns the kept columns (column-major).
// With `nrm` (3 per node), each node's block of every column is first replaced
// by its component along the node's normal (projection.cpp:231-233).
int rigid_basis(const std::vector<double>& pos, const double* nrm, std::vector<double>& Q, bool drop);
void rigid_setup(or_problem* p);
void displacement_project(const or_problem* p, double* u);
}
