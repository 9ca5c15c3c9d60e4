// FP64 CPU oracle: element matrix, hierarchy/topology, operator, smoothers,
// transfers, Galerkin coarse operators, coarsest solve, V-cycle and solves.
// TEST INFRASTRUCTURE ONLY (see oracle.h).
#include "or_internal.h"
#include <cstdio>
#include <cstdlib>

using namespace orc;

static const double DIRICHLET_W = 1e6;  // grid/Grid.cu:14

// ---------------------------------------------------------------- K0
// element/templateMatrix.cpp:15-99: 2x2x2 Gauss, D(E,nu), B with node-major
// xyz DOFs, local node a -> (a%2, a/2%2, a/4), scaled by (h/2)^3.
extern "C" void or_k0(double E, double nu, double h, double* K0) {
  double D[6][6] = {{0}};
  double c = E / ((1 + nu) * (1 - 2 * nu));
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) D[i][j] = c * (i == j ? 1 - nu : nu);
  for (int i = 3; i < 6; i++) D[i][i] = c * (1 - 2 * nu) / 2;
  for (int i = 0; i < 576; i++) K0[i] = 0;
  const double g = std::sqrt(3.0) / 3;
  for (int q = 0; q < 8; q++) {
    double gp[3] = {((2 * (q % 2) - 1) * g + 1) / 2, ((2 * (q / 2 % 2) - 1) * g + 1) / 2,
                    ((2 * (q / 4) - 1) * g + 1) / 2};
    double dN[8][3];
    for (int a = 0; a < 8; a++) {
      int id[3] = {a % 2, a / 2 % 2, a / 4};
      double r[3];
      for (int k = 0; k < 3; k++) r[k] = id[k] ? gp[k] : 1 - gp[k];
      for (int k = 0; k < 3; k++)
        dN[a][k] = (id[k] ? 1.0 / h : -1.0 / h) * r[(k + 1) % 3] * r[(k + 2) % 3];
    }
    double B[6][24] = {{0}};
    for (int a = 0; a < 8; a++) {
      for (int k = 0; k < 3; k++) B[k][3 * a + k] = dN[a][k];
      B[3][3 * a + 1] = dN[a][2]; B[3][3 * a + 2] = dN[a][1];
      B[4][3 * a + 0] = dN[a][2]; B[4][3 * a + 2] = dN[a][0];
      B[5][3 * a + 0] = dN[a][1]; B[5][3 * a + 1] = dN[a][0];
    }
    double DB[6][24];
    for (int i = 0; i < 6; i++)
      for (int j = 0; j < 24; j++) {
        double s = 0;
        for (int k = 0; k < 6; k++) s += D[i][k] * B[k][j];
        DB[i][j] = s;
      }
    for (int i = 0; i < 24; i++)
      for (int j = 0; j < 24; j++) {
        double s = 0;
        for (int k = 0; k < 6; k++) s += B[k][i] * DB[k][j];
        K0[i * 24 + j] += s;
      }
  }
  double sc = std::pow(h / 2, 3);
  for (int i = 0; i < 576; i++) K0[i] *= sc;
}

// ---------------------------------------------------------------- topology
static void vertex_mask(Level& l) {
  l.vmask.assign(l.nn, 0);
  for (int z = 0; z < l.ez; z++)
    for (int y = 0; y < l.ey; y++)
      for (int x = 0; x < l.ex; x++)
        if (l.emask[l.eidx(x, y, z)])
          for (int k = 0; k < 8; k++) l.vmask[l.nidx(x + k % 2, y + k / 2 % 2, z + k / 4)] = 1;
}

static Level make_level(int ex, int ey, int ez) {
  Level l;
  l.ex = ex; l.ey = ey; l.ez = ez;
  l.nx = ex + 1; l.ny = ey + 1; l.nz = ez + 1;
  l.ne = (long)ex * ey * ez; l.nn = (long)l.nx * l.ny * l.nz;
  l.emask.assign(l.ne, 0);
  return l;
}

// coarse element = OR of its children (Grid.cu setSolidElementFromFineGrid)
static Level coarsen(const Level& f, int factor) {
  Level c = make_level((f.ex + factor - 1) / factor, (f.ey + factor - 1) / factor,
                       (f.ez + factor - 1) / factor);
  c.factor = factor;
  for (int z = 0; z < f.ez; z++)
    for (int y = 0; y < f.ey; y++)
      for (int x = 0; x < f.ex; x++)
        if (f.emask[f.eidx(x, y, z)]) c.emask[c.eidx(x / factor, y / factor, z / factor)] = 1;
  vertex_mask(c);
  return c;
}

static long count(const std::vector<uint8_t>& m) {
  long s = 0;
  for (auto v : m) s += v != 0;
  return s;
}

void orc::build_topology(or_problem* p, int n_levels, int first_factor) {
  Level& l0 = p->L[0];
  vertex_mask(l0);
  // reference hierarchy: halve while active elements > 400 (Grid.cpp:1011);
  // layer 1 is a dummy when the first coarsening is non-dyadic.
  std::vector<Level> halves;
  halves.push_back(l0);
  if (n_levels <= 0) {
    while (count(halves.back().emask) > 400) halves.push_back(coarsen(halves.back(), 2));
    std::vector<Level> out;
    out.push_back(l0);
    for (size_t i = 1; i < halves.size(); i++) {
      if (first_factor == 4 && i == 1) continue;
      if (first_factor == 4 && i == 2) {
        Level c = coarsen(l0, 4);
        out.push_back(c);
      } else {
        out.push_back(halves[i]);
        out.back().factor = 2;
      }
    }
    // the coarsest level is solved directly from its stencil, so at least one
    // coarse level is kept (the reference would be left with only a dummy layer)
    if (out.size() == 1) out.push_back(coarsen(l0, 2));
    p->L = out;
  } else {
    std::vector<Level> out;
    out.push_back(l0);
    for (int i = 1; i < n_levels; i++) {
      int f = (i == 1) ? first_factor : 2;
      out.push_back(coarsen(out.back(), f));
    }
    p->L = out;
  }
  // fine-level node classes
  Level& f = p->L[0];
  p->surface.assign(f.nn, 0);
  p->support.assign(f.nn, 0);
  p->load.assign(f.nn, 0);
  for (int z = 0; z < f.nz; z++)
    for (int y = 0; y < f.ny; y++)
      for (int x = 0; x < f.nx; x++) {
        long n = f.nidx(x, y, z);
        if (!f.vmask[n]) continue;
        // mark_surface_nodes_kernel (Grid.cu:2824-2858)
        bool solid[2][2][2];
        for (int k = 0; k < 8; k++) {
          int exx = x - 1 + k % 2, eyy = y - 1 + k / 2 % 2, ezz = z - 1 + k / 4;
          bool s = exx >= 0 && eyy >= 0 && ezz >= 0 && exx < f.ex && eyy < f.ey && ezz < f.ez &&
                   f.emask[f.eidx(exx, eyy, ezz)];
          solid[k % 2][k / 2 % 2][k / 4] = s;
        }
        bool ax[3] = {false, false, false};
        for (int i = 0; i < 2; i++)
          for (int j = 0; j < 2; j++) {
            ax[0] |= solid[0][i][j] && solid[1][i][j];
            ax[1] |= solid[i][0][j] && solid[i][1][j];
            ax[2] |= solid[i][j][0] && solid[i][j][1];
          }
        bool surf = !ax[0] || !ax[1] || !ax[2];
        p->surface[n] = surf;
        // computeProjectionMatrix (Grid.cpp:2715-2745)
        if (surf && p->fixed_area[n]) p->support[n] = 1;
        else if (surf && p->load_area[n]) p->load[n] = 1;
      }
}

// ---------------------------------------------------------------- create
extern "C" or_problem* or_create(int ex, int ey, int ez, const uint8_t* emask,
                                 const uint8_t* fixed_area, const uint8_t* load_area,
                                 const double* load_normals, double E, double nu,
                                 double penal, double rhomin, int n_levels,
                                 int first_factor) {
  or_problem* p = new or_problem();
  p->E = E; p->nu = nu; p->penal = penal; p->rhomin = rhomin;
  or_k0(E, nu, 1.0, p->K0);
  Level l0 = make_level(ex, ey, ez);
  for (long i = 0; i < l0.ne; i++) l0.emask[i] = emask[i] ? 1 : 0;
  p->L.push_back(l0);
  long nn = p->L[0].nn;
  p->fixed_area.assign(fixed_area, fixed_area + nn);
  p->load_area.assign(load_area, load_area + nn);
  if (load_normals) p->normals.assign(load_normals, load_normals + 3 * nn);
  else p->normals.assign(3 * nn, 0.0);
  build_topology(p, n_levels, first_factor);
  // load nodes sorted by reference gs id (projection.cpp:139-145)
  std::vector<int> vl2g(count(p->L[0].vmask));
  or_ref_numbering(p, 0, nullptr, nullptr, vl2g.data(), nullptr, nullptr, nullptr);
  std::vector<std::pair<int, int>> ln;
  long lex = 0;
  for (long n = 0; n < nn; n++) {
    if (!p->L[0].vmask[n]) continue;
    if (p->load[n]) ln.push_back({vl2g[lex], (int)n});
    lex++;
  }
  std::sort(ln.begin(), ln.end());
  for (auto& q : ln) p->load_nodes.push_back(q.second);
  p->has_support = std::any_of(p->support.begin(), p->support.end(), [](uint8_t s) { return s != 0; });
  if (!p->has_support) rigid_setup(p);
  p->rho.assign(p->L[0].ne, 1.0);
  p->rhop.assign(p->L[0].ne, 1.0);
  return p;
}

extern "C" void or_destroy(or_problem* p) { delete p; }
extern "C" long or_solve_iterations(const or_problem* p) { return p->solve_iters; }
extern "C" int or_n_levels(const or_problem* p) { return (int)p->L.size(); }
extern "C" void or_level_dims(const or_problem* p, int level, int* d) {
  const Level& l = p->L[level];
  d[0] = l.ex; d[1] = l.ey; d[2] = l.ez; d[3] = l.nx; d[4] = l.ny; d[5] = l.nz;
}
extern "C" void or_level_masks(const or_problem* p, int level, uint8_t* em, uint8_t* vm) {
  const Level& l = p->L[level];
  if (em) std::copy(l.emask.begin(), l.emask.end(), em);
  if (vm) std::copy(l.vmask.begin(), l.vmask.end(), vm);
}
extern "C" int or_level_bitwords(const or_problem* p, int level, uint32_t* eb, uint32_t* vb) {
  const Level& l = p->L[level];
  long nwe = (l.ne + 31) / 32, nwv = (l.nn + 31) / 32;
  if (eb) {
    for (long w = 0; w < nwe; w++) eb[w] = 0;
    for (long i = 0; i < l.ne; i++) if (l.emask[i]) eb[i / 32] |= 1u << (i % 32);
  }
  if (vb) {
    for (long w = 0; w < nwv; w++) vb[w] = 0;
    for (long i = 0; i < l.nn; i++) if (l.vmask[i]) vb[i / 32] |= 1u << (i % 32);
  }
  return (int)nwv;
}
extern "C" void or_node_class(const or_problem* p, uint8_t* out) {
  const Level& l = p->L[0];
  for (long n = 0; n < l.nn; n++)
    out[n] = (l.vmask[n] ? 1 : 0) | (p->surface[n] ? 2 : 0) | (p->support[n] ? 4 : 0) |
             (p->load[n] ? 8 : 0);
}
extern "C" int or_n_load(const or_problem* p) { return (int)p->load_nodes.size(); }
extern "C" int or_load_nodes(const or_problem* p, int* nodes) {
  for (size_t i = 0; i < p->load_nodes.size(); i++) nodes[i] = p->load_nodes[i];
  return (int)p->load_nodes.size();
}

// reference compact numbering: lexicographic rank, GS colour
// (x%2)+2(y%2)+4(z%2) (Grid.cu:1310-1385), colour-major order with each colour
// padded to a multiple of 32 (Grid.cpp:4187-4248); flag words
// (Grid.h:399-439, Grid.cpp:2858-2882).
extern "C" int or_ref_numbering(const or_problem* p, int level, int* counts, int* gs_num,
                                int* vlexi2gs, int* elexi2gs, int* vflag_gs, int* eflag_gs) {
  const Level& l = p->L[level];
  long nv = 0, ne = 0;
  long vc[8] = {0}, ecnt[8] = {0};
  for (int z = 0; z < l.nz; z++)
    for (int y = 0; y < l.ny; y++)
      for (int x = 0; x < l.nx; x++)
        if (l.vmask[l.nidx(x, y, z)]) { vc[x % 2 + 2 * (y % 2) + 4 * (z % 2)]++; nv++; }
  for (int z = 0; z < l.ez; z++)
    for (int y = 0; y < l.ey; y++)
      for (int x = 0; x < l.ex; x++)
        if (l.emask[l.eidx(x, y, z)]) { ecnt[x % 2 + 2 * (y % 2) + 4 * (z % 2)]++; ne++; }
  long vpad[8], epad[8], voff[8], eoff[8], nvgs = 0, negs = 0;
  for (int c = 0; c < 8; c++) {
    vpad[c] = (vc[c] + 31) / 32 * 32; epad[c] = (ecnt[c] + 31) / 32 * 32;
    voff[c] = nvgs; eoff[c] = negs; nvgs += vpad[c]; negs += epad[c];
    if (gs_num) gs_num[c] = (int)vpad[c];
  }
  if (counts) { counts[0] = (int)nv; counts[1] = (int)ne; counts[2] = (int)nvgs; counts[3] = (int)negs; }
  if (vflag_gs) for (long i = 0; i < nvgs; i++) vflag_gs[i] = -1;
  if (eflag_gs) for (long i = 0; i < negs; i++) eflag_gs[i] = -1;
  long acc[8] = {0}, lex = 0;
  for (int z = 0; z < l.nz; z++)
    for (int y = 0; y < l.ny; y++)
      for (int x = 0; x < l.nx; x++) {
        long n = l.nidx(x, y, z);
        if (!l.vmask[n]) continue;
        int c = x % 2 + 2 * (y % 2) + 4 * (z % 2);
        long gs = voff[c] + acc[c]++;
        if (vlexi2gs) vlexi2gs[lex] = (int)gs;
        if (vflag_gs) {
          int w = (x % 8) | ((y % 8) << 3) | ((z % 8) << 6) | (c << 9);
          if (level == 0) {
            if (p->surface[n]) w |= 1 << 13;
            if (p->load[n]) w |= 1 << 14;
            if (p->support[n]) w |= 1 << 19;
          }
          vflag_gs[gs] = w;
        }
        lex++;
      }
  long eacc[8] = {0};
  lex = 0;
  for (int z = 0; z < l.ez; z++)
    for (int y = 0; y < l.ey; y++)
      for (int x = 0; x < l.ex; x++) {
        if (!l.emask[l.eidx(x, y, z)]) continue;
        int c = x % 2 + 2 * (y % 2) + 4 * (z % 2);
        long gs = eoff[c] + eacc[c]++;
        if (elexi2gs) elexi2gs[lex] = (int)gs;
        if (eflag_gs) eflag_gs[gs] = c << 9;
        lex++;
      }
  return (int)nvgs;
}

// ---------------------------------------------------------------- operator
extern "C" void or_set_density(or_problem* p, const double* rho) {
  const Level& l = p->L[0];
  for (long e = 0; e < l.ne; e++) {
    p->rho[e] = l.emask[e] ? rho[e] : 0.0;
    p->rhop[e] = l.emask[e] ? std::pow(rho[e], p->penal) : 0.0;
  }
}

// f = K u with the reference's support treatment (applyK_OTFA_kernel,
// Grid.cu:4358-4436): fixed neighbours read as zero, fixed rows pass u.
// mode 0: applyK, mode 1: residual r = f - K u (update_residual_OTFA_WS).
static void fine_apply(const or_problem* p, const double* u, const double* fin, double* out, int mode) {
  const Level& l = p->L[0];
  const long nn = l.nn;
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < l.nz; z++)
    for (int y = 0; y < l.ny; y++)
      for (int x = 0; x < l.nx; x++) {
        long n = l.nidx(x, y, z);
        double acc[3] = {0, 0, 0};
        if (l.vmask[n] && !p->support[n]) {
          for (int k = 0; k < 8; k++) {
            int exx = x - 1 + k % 2, eyy = y - 1 + k / 2 % 2, ezz = z - 1 + k / 4;
            if (exx < 0 || eyy < 0 || ezz < 0 || exx >= l.ex || eyy >= l.ey || ezz >= l.ez) continue;
            long e = l.eidx(exx, eyy, ezz);
            if (!l.emask[e]) continue;
            double rp = p->rhop[e];
            int vi = 7 - k;
            for (int vj = 0; vj < 8; vj++) {
              long j = l.nidx(exx + vj % 2, eyy + vj / 2 % 2, ezz + vj / 4);
              if (p->support[j]) continue;
              for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++)
                  acc[r] += rp * p->K0[(vi * 3 + r) * 24 + vj * 3 + c] * u[c * nn + j];
            }
          }
        }
        for (int r = 0; r < 3; r++) {
          if (mode == 0) out[r * nn + n] = (l.vmask[n] && p->support[n]) ? u[r * nn + n] : acc[r];
          else out[r * nn + n] = fin[r * nn + n] - acc[r];
        }
      }
}

extern "C" void or_apply_K(const or_problem* p, const double* u, double* f) { fine_apply(p, u, nullptr, f, 0); }
extern "C" void or_residual(const or_problem* p, const double* u, const double* f, double* r) { fine_apply(p, u, f, r, 1); }

double orc::dot3(const double* a, const double* b, long nn) {
  double s = 0;
#pragma omp parallel for reduction(+ : s)
  for (long i = 0; i < 3 * nn; i++) s += a[i] * b[i];
  return s;
}

// ---------------------------------------------------------------- Galerkin
// Coarse operator K_c = P^T K_mod P (the definition behind the reference's
// restrict_stencil_nondyadic_OTFA_WS_kernel, Grid.cu:1154-1268, and
// restrict_stencil_dyadic_kernel, Grid.cu:882-939), evaluated element by
// element: K_mod zeroes the rows/columns of support DOFs and puts 1e6 on
// their diagonal; P is trilinear interpolation.
static void prolong_weights(int f, int pos, double* w /*[2][2] per axis: node offset o in {0,1} -> corner A*/) {
  // fine node at offset pos+o in [0,f]; corner A=0 weight (f-(pos+o))/f, A=1 weight (pos+o)/f
  for (int o = 0; o < 2; o++) {
    w[o * 2 + 0] = double(f - (pos + o)) / f;
    w[o * 2 + 1] = double(pos + o) / f;
  }
}

static void triple(const double* Ke, int f, int px, int py, int pz, double* out) {
  // out += P^T Ke P, P[(a,i),(A,j)] = delta_ij * wx*wy*wz
  double wx[4], wy[4], wz[4];
  prolong_weights(f, px, wx); prolong_weights(f, py, wy); prolong_weights(f, pz, wz);
  double P[8][8];
  for (int a = 0; a < 8; a++)
    for (int A = 0; A < 8; A++)
      P[a][A] = wx[(a % 2) * 2 + A % 2] * wy[(a / 2 % 2) * 2 + A / 2 % 2] * wz[(a / 4) * 2 + A / 4];
  double KP[24][24];
  for (int r = 0; r < 24; r++)
    for (int A = 0; A < 8; A++)
      for (int j = 0; j < 3; j++) {
        double s = 0;
        for (int b = 0; b < 8; b++) s += Ke[r * 24 + b * 3 + j] * P[b][A];
        KP[r][A * 3 + j] = s;
      }
  for (int A = 0; A < 8; A++)
    for (int i = 0; i < 3; i++)
      for (int c = 0; c < 24; c++) {
        double s = 0;
        for (int a = 0; a < 8; a++) s += P[a][A] * KP[a * 3 + i][c];
        out[(A * 3 + i) * 24 + c] += s;
      }
}

static void assemble_stencil(Level& c) {
  c.stencil.assign(243 * c.nn, 0.0);
  for (int z = 0; z < c.ez; z++)
    for (int y = 0; y < c.ey; y++)
      for (int x = 0; x < c.ex; x++) {
        long E = c.eidx(x, y, z);
        if (!c.emask[E]) continue;
        const double* K = &c.KE[E * 576];
        for (int a = 0; a < 8; a++) {
          long na = c.nidx(x + a % 2, y + a / 2 % 2, z + a / 4);
          for (int b = 0; b < 8; b++) {
            int d = (b % 2 - a % 2 + 1) + 3 * (b / 2 % 2 - a / 2 % 2 + 1) + 9 * (b / 4 - a / 4 + 1);
            for (int r = 0; r < 3; r++)
              for (int cc = 0; cc < 3; cc++)
                c.stencil[(d * 9 + r * 3 + cc) * c.nn + na] += K[(a * 3 + r) * 24 + b * 3 + cc];
          }
        }
      }
}

void orc::galerkin(or_problem* p) {
  Level& f0 = p->L[0];
  for (size_t li = 1; li < p->L.size(); li++) {
    Level& c = p->L[li];
    const Level& fl = p->L[li - 1];
    int fct = c.factor;
    c.KE.assign(576 * c.ne, 0.0);
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int Z = 0; Z < c.ez; Z++)
      for (int Y = 0; Y < c.ey; Y++)
        for (int X = 0; X < c.ex; X++) {
          long E = c.eidx(X, Y, Z);
          if (!c.emask[E]) continue;
          double* out = &c.KE[E * 576];
          for (int pz = 0; pz < fct; pz++)
            for (int py = 0; py < fct; py++)
              for (int px = 0; px < fct; px++) {
                int x = X * fct + px, y = Y * fct + py, z = Z * fct + pz;
                if (x >= fl.ex || y >= fl.ey || z >= fl.ez) continue;
                long e = fl.eidx(x, y, z);
                if (!fl.emask[e]) continue;
                double Ke[576];
                if (li == 1) {
                  double rp = p->rhop[e];
                  bool fx[8];
                  for (int a = 0; a < 8; a++) fx[a] = p->support[f0.nidx(x + a % 2, y + a / 2 % 2, z + a / 4)];
                  for (int r = 0; r < 24; r++)
                    for (int cc = 0; cc < 24; cc++) {
                      double v = rp * p->K0[r * 24 + cc];
                      if (fx[r / 3] || fx[cc / 3]) v = (r == cc) ? DIRICHLET_W : 0.0;
                      Ke[r * 24 + cc] = v;
                    }
                } else {
                  std::memcpy(Ke, &fl.KE[e * 576], sizeof(Ke));
                }
                triple(Ke, fct, px, py, pz, out);
              }
        }
    assemble_stencil(c);
  }
}

static void jacobi_sweep(const or_problem* p, int level, double* u, const double* f, double omega);

// lambda_max(D^-1 K) per level by 20 power iterations from a fixed start;
// damped Jacobi uses omega relative to the stability bound 2/lambda_max.
static void estimate_lambda(or_problem* p) {
  p->lam.assign(p->L.size(), 1.0);
  for (size_t l = 0; l + 1 < p->L.size() || (l == 0 && p->L.size() == 1); l++) {
    const Level& lv = p->L[l];
    std::vector<double> u(3 * lv.nn), v(3 * lv.nn), z(3 * lv.nn, 0.0);
    for (long i = 0; i < 3 * lv.nn; i++) {
      uint64_t h = (uint64_t)i * 0x9E3779B97F4A7C15ull + 12345;
      h ^= h >> 29; h *= 0xBF58476D1CE4E5B9ull; h ^= h >> 32;
      u[i] = (double)(h >> 11) / 9007199254740992.0 - 0.5;
    }
    double lam = 0;
    for (int it = 0; it < 20; it++) {
      v = u;
      jacobi_sweep(p, (int)l, v.data(), z.data(), 1.0);  // v = u - D^-1 K u
      double nu = 0, nw = 0;
      for (long i = 0; i < 3 * lv.nn; i++) { double w = u[i] - v[i]; nw += w * w; nu += u[i] * u[i]; u[i] = w; }
      lam = std::sqrt(nw / nu);
      double s = 1 / std::sqrt(nw);
      for (auto& x : u) x *= s;
    }
    p->lam[l] = 1.05 * lam;
    if (p->L.size() == 1) break;
  }
}

extern "C" void or_update_stencil(or_problem* p) {
  orc::galerkin(p);
  orc::coarsest_factor(p);
  estimate_lambda(p);
}

extern "C" double or_level_lambda(const or_problem* p, int level) { return p->lam[level]; }

extern "C" void or_get_stencil(const or_problem* p, int level, double* out) {
  const Level& l = p->L[level];
  std::copy(l.stencil.begin(), l.stencil.end(), out);
}

static void coarse_apply(const Level& l, const double* u, const double* f, double* r) {
  const long nn = l.nn;
#pragma omp parallel for collapse(2)
  for (int z = 0; z < l.nz; z++)
    for (int y = 0; y < l.ny; y++)
      for (int x = 0; x < l.nx; x++) {
        long n = l.nidx(x, y, z);
        double acc[3] = {0, 0, 0};
        if (l.vmask[n]) {
          for (int d = 0; d < 27; d++) {
            int xx = x + d % 3 - 1, yy = y + d / 3 % 3 - 1, zz = z + d / 9 - 1;
            if (xx < 0 || yy < 0 || zz < 0 || xx >= l.nx || yy >= l.ny || zz >= l.nz) continue;
            long j = l.nidx(xx, yy, zz);
            for (int rr = 0; rr < 3; rr++)
              for (int c = 0; c < 3; c++) acc[rr] += l.stencil[(d * 9 + rr * 3 + c) * nn + n] * u[c * nn + j];
          }
        }
        for (int rr = 0; rr < 3; rr++) r[rr * nn + n] = f[rr * nn + n] - acc[rr];
      }
}

extern "C" void or_coarse_residual(const or_problem* p, int level, const double* u, const double* f, double* r) {
  coarse_apply(p->L[level], u, f, r);
}

// ---------------------------------------------------------------- smoothers
// Fine 8-colour Gauss-Seidel: gs_relax_OTFA_WS_kernel (Grid.cu:1742-1885).
static void fine_gs_colour(const or_problem* p, double* u, const double* f, int col, bool rev) {
  const Level& l = p->L[0];
  const long nn = l.nn;
  int cx = col % 2, cy = col / 2 % 2, cz = col / 4;
#pragma omp parallel for collapse(2)
  for (int z = cz; z < l.nz; z += 2)
    for (int y = cy; y < l.ny; y += 2)
      for (int x = cx; x < l.nx; x += 2) {
        long n = l.nidx(x, y, z);
        if (!l.vmask[n]) continue;
        bool fix = p->support[n];
        double S[9] = {0}, KU[3] = {0, 0, 0};
        for (int k = 0; k < 8; k++) {
          int exx = x - 1 + k % 2, eyy = y - 1 + k / 2 % 2, ezz = z - 1 + k / 4;
          if (exx < 0 || eyy < 0 || ezz < 0 || exx >= l.ex || eyy >= l.ey || ezz >= l.ez) continue;
          long e = l.eidx(exx, eyy, ezz);
          if (!l.emask[e]) continue;
          double rp = p->rhop[e];
          int vi = 7 - k;
          if (fix) { S[0] += 1; S[4] += 1; S[8] += 1; continue; }
          for (int vj = 0; vj < 8; vj++) {
            long j = l.nidx(exx + vj % 2, eyy + vj / 2 % 2, ezz + vj / 4);
            if (vj == vi) {
              for (int i = 0; i < 9; i++) S[i] += rp * p->K0[(vi * 3 + i / 3) * 24 + vi * 3 + i % 3];
              continue;
            }
            if (p->support[j]) continue;
            for (int r = 0; r < 3; r++)
              for (int c = 0; c < 3; c++) KU[r] += rp * p->K0[(vi * 3 + r) * 24 + vj * 3 + c] * u[c * nn + j];
          }
        }
        if (fix) { KU[0] = KU[1] = KU[2] = 0; }
        double v[3] = {u[n], u[nn + n], u[2 * nn + n]};
        for (int t = 0; t < 3; t++) {
          int r = rev ? 2 - t : t;  // the backward sweep reverses the in-node order too
          double s = f[r * nn + n] - KU[r];
          for (int c = 0; c < 3; c++) if (c != r) s -= S[r * 3 + c] * v[c];
          v[r] = s / S[r * 3 + r];
        }
        u[n] = v[0]; u[nn + n] = v[1]; u[2 * nn + n] = v[2];
      }
}

// Coarse 8-colour Gauss-Seidel on stored stencils: gs_relax_kernel (Grid.cu:1497-1609).
static void coarse_gs_colour(const Level& l, double* u, const double* f, int col, bool rev) {
  const long nn = l.nn;
  int cx = col % 2, cy = col / 2 % 2, cz = col / 4;
#pragma omp parallel for collapse(2)
  for (int z = cz; z < l.nz; z += 2)
    for (int y = cy; y < l.ny; y += 2)
      for (int x = cx; x < l.nx; x += 2) {
        long n = l.nidx(x, y, z);
        if (!l.vmask[n]) continue;
        double Au[3] = {0, 0, 0};
        for (int d = 0; d < 27; d++) {
          if (d == 13) continue;
          int xx = x + d % 3 - 1, yy = y + d / 3 % 3 - 1, zz = z + d / 9 - 1;
          if (xx < 0 || yy < 0 || zz < 0 || xx >= l.nx || yy >= l.ny || zz >= l.nz) continue;
          long j = l.nidx(xx, yy, zz);
          for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) Au[r] += l.stencil[(d * 9 + r * 3 + c) * nn + n] * u[c * nn + j];
        }
        const double* S = nullptr;
        double s[9];
        for (int i = 0; i < 9; i++) s[i] = l.stencil[(13 * 9 + i) * nn + n];
        S = s;
        double v[3] = {u[n], u[nn + n], u[2 * nn + n]};
        for (int t = 0; t < 3; t++) {
          int r = rev ? 2 - t : t;
          double s = f[r * nn + n] - Au[r];
          for (int c = 0; c < 3; c++) if (c != r) s -= S[r * 3 + c] * v[c];
          v[r] = s / S[r * 3 + r];
        }
        u[n] = v[0]; u[nn + n] = v[1]; u[2 * nn + n] = v[2];
      }
}

static void inv3(const double* S, double* I) {
  double a = S[0], b = S[1], c = S[2], d = S[3], e = S[4], f = S[5], g = S[6], h = S[7], k = S[8];
  double A = e * k - f * h, B = -(d * k - f * g), C = d * h - e * g;
  double det = a * A + b * B + c * C;
  double id = 1.0 / det;
  I[0] = A * id; I[1] = -(b * k - c * h) * id; I[2] = (b * f - c * e) * id;
  I[3] = B * id; I[4] = (a * k - c * g) * id; I[5] = -(a * f - c * d) * id;
  I[6] = C * id; I[7] = -(a * h - b * g) * id; I[8] = (a * e - b * d) * id;
}

// damped block-Jacobi (build feature): u += omega * D^-1 (f - K u), D = 3x3 diagonal block.
static void jacobi_sweep(const or_problem* p, int level, double* u, const double* f, double omega) {
  const Level& l = p->L[level];
  const long nn = l.nn;
  std::vector<double> r(3 * nn);
  if (level == 0) fine_apply(p, u, f, r.data(), 1);
  else coarse_apply(l, u, f, r.data());
#pragma omp parallel for collapse(2)
  for (int z = 0; z < l.nz; z++)
    for (int y = 0; y < l.ny; y++)
      for (int x = 0; x < l.nx; x++) {
        long n = l.nidx(x, y, z);
        if (!l.vmask[n]) continue;
        double S[9] = {0};
        if (level == 0) {
          if (p->support[n]) { u[n] = u[nn + n] = u[2 * nn + n] = 0; continue; }
          for (int k = 0; k < 8; k++) {
            int exx = x - 1 + k % 2, eyy = y - 1 + k / 2 % 2, ezz = z - 1 + k / 4;
            if (exx < 0 || eyy < 0 || ezz < 0 || exx >= l.ex || eyy >= l.ey || ezz >= l.ez) continue;
            long e = l.eidx(exx, eyy, ezz);
            if (!l.emask[e]) continue;
            int vi = 7 - k;
            for (int i = 0; i < 9; i++) S[i] += p->rhop[e] * p->K0[(vi * 3 + i / 3) * 24 + vi * 3 + i % 3];
          }
        } else {
          for (int i = 0; i < 9; i++) S[i] = l.stencil[(13 * 9 + i) * nn + n];
        }
        double I[9];
        inv3(S, I);
        double rr[3] = {r[n], r[nn + n], r[2 * nn + n]};
        for (int i = 0; i < 3; i++) u[i * nn + n] += omega * (I[i * 3] * rr[0] + I[i * 3 + 1] * rr[1] + I[i * 3 + 2] * rr[2]);
      }
}

extern "C" void or_smooth(const or_problem* p, int level, double* u, const double* f, int kind,
                          double omega, int sweeps, int reverse) {
  for (int s = 0; s < sweeps; s++) {
    if (kind == 1) { jacobi_sweep(p, level, u, f, omega); continue; }
    for (int ci = 0; ci < 8; ci++) {
      int c = reverse ? 7 - ci : ci;
      if (level == 0) fine_gs_colour(p, u, f, c, reverse != 0);
      else coarse_gs_colour(p->L[level], u, f, c, reverse != 0);
    }
  }
}

// ---------------------------------------------------------------- transfers
// restriction R = P^T (restrict_residual_kernel Grid.cu:2499-2550 and the
// non-dyadic variant :2552-2613); prolongation u_f += P u_c (:2637-2714).
extern "C" void or_restrict(const or_problem* p, int cl, const double* rf, double* fc) {
  const Level& c = p->L[cl];
  const Level& f = p->L[cl - 1];
  const int F = c.factor;
#pragma omp parallel for collapse(2)
  for (int Z = 0; Z < c.nz; Z++)
    for (int Y = 0; Y < c.ny; Y++)
      for (int X = 0; X < c.nx; X++) {
        long nC = c.nidx(X, Y, Z);
        double s[3] = {0, 0, 0};
        if (c.vmask[nC]) {
          for (int dz = -F + 1; dz < F; dz++)
            for (int dy = -F + 1; dy < F; dy++)
              for (int dx = -F + 1; dx < F; dx++) {
                int x = F * X + dx, y = F * Y + dy, z = F * Z + dz;
                if (x < 0 || y < 0 || z < 0 || x >= f.nx || y >= f.ny || z >= f.nz) continue;
                long n = f.nidx(x, y, z);
                if (!f.vmask[n]) continue;
                double w = double(F - std::abs(dx)) * (F - std::abs(dy)) * (F - std::abs(dz)) / (double(F) * F * F);
                for (int i = 0; i < 3; i++) s[i] += w * rf[i * f.nn + n];
              }
        }
        for (int i = 0; i < 3; i++) fc[i * c.nn + nC] = s[i];
      }
}

extern "C" void or_prolong(const or_problem* p, int cl, const double* uc, double* uf) {
  const Level& c = p->L[cl];
  const Level& f = p->L[cl - 1];
  const int F = c.factor;
#pragma omp parallel for collapse(2)
  for (int z = 0; z < f.nz; z++)
    for (int y = 0; y < f.ny; y++)
      for (int x = 0; x < f.nx; x++) {
        long n = f.nidx(x, y, z);
        if (!f.vmask[n]) continue;
        int X0 = x / F, Y0 = y / F, Z0 = z / F;
        double s[3] = {0, 0, 0};
        for (int A = 0; A < 8; A++) {
          int X = X0 + A % 2, Y = Y0 + A / 2 % 2, Z = Z0 + A / 4;
          if (X >= c.nx || Y >= c.ny || Z >= c.nz) continue;
          int ax = std::abs(x - F * X), ay = std::abs(y - F * Y), az = std::abs(z - F * Z);
          if (ax >= F || ay >= F || az >= F) continue;
          double w = double(F - ax) * (F - ay) * (F - az) / (double(F) * F * F);
          long nC = c.nidx(X, Y, Z);
          for (int i = 0; i < 3; i++) s[i] += w * uc[i * c.nn + nC];
        }
        for (int i = 0; i < 3; i++) uf[i * f.nn + n] += s[i];
      }
}

// ---------------------------------------------------------------- coarsest
// Dense FP64 factorisation of the coarsest stencil (the reference builds the
// same dense matrix, buildCoarsestSystem Grid.cpp:3697-3752, and solves it
// with a BDCSVD pseudo-inverse; with supports the matrix is SPD and the
// inverse coincides).  Cholesky-based explicit inverse.
void orc::coarsest_factor(or_problem* p) {
  const Level& c = p->L.back();
  p->cnode.clear();
  p->crow.assign(c.nn, -1);
  for (long n = 0; n < c.nn; n++)
    if (c.vmask[n]) { p->crow[n] = (long)p->cnode.size(); p->cnode.push_back(n); }
  int nc = (int)p->cnode.size();
  p->nc = nc;
  int N = 3 * nc;
  std::vector<double> K((size_t)N * N, 0.0);
  if (p->L.size() == 1) return;
  for (int i = 0; i < nc; i++) {
    long n = p->cnode[i];
    int x = n % c.nx, y = n / c.nx % c.ny, z = n / ((long)c.nx * c.ny);
    for (int d = 0; d < 27; d++) {
      int xx = x + d % 3 - 1, yy = y + d / 3 % 3 - 1, zz = z + d / 9 - 1;
      if (xx < 0 || yy < 0 || zz < 0 || xx >= c.nx || yy >= c.ny || zz >= c.nz) continue;
      long j = c.nidx(xx, yy, zz);
      long cj = p->crow[j];
      if (cj < 0) continue;
      for (int r = 0; r < 3; r++)
        for (int cc = 0; cc < 3; cc++)
          K[(size_t)(3 * i + r) * N + 3 * cj + cc] = c.stencil[(d * 9 + r * 3 + cc) * c.nn + n];
    }
  }
  // symmetrise (the Galerkin product is symmetric up to rounding)
  for (int i = 0; i < N; i++)
    for (int j = i + 1; j < N; j++) {
      double v = 0.5 * (K[(size_t)i * N + j] + K[(size_t)j * N + i]);
      K[(size_t)i * N + j] = K[(size_t)j * N + i] = v;
    }
  // without supports K is singular, its null space the rigid motions R of the
  // coarsest nodes (trilinear prolongation reproduces them): factor
  // K + a R R^T, a the mean diagonal, and K^+ = (K + a R R^T)^-1 - R R^T / a
  // (the reference's BDCSVD pseudo-inverse, Grid.cpp:4123-4185)
  double a_rig = 0;
  int k_rig = 0;
  if (!p->has_support) {
    std::vector<double> pos;
    for (int i = 0; i < nc; i++) {
      long n = p->cnode[i];
      pos.push_back((double)(n % c.nx));
      pos.push_back((double)(n / c.nx % c.ny));
      pos.push_back((double)(n / ((long)c.nx * c.ny)));
    }
    k_rig = rigid_basis(pos, nullptr, p->rigid_coarse, false);
    for (int i = 0; i < N; i++) a_rig += K[(size_t)i * N + i];
    a_rig /= N;
    for (int i = 0; i < N; i++)
      for (int j = 0; j < N; j++) {
        double s = 0;
        for (int q = 0; q < k_rig; q++) s += p->rigid_coarse[(size_t)q * N + i] * p->rigid_coarse[(size_t)q * N + j];
        K[(size_t)i * N + j] += a_rig * s;
      }
  }
  // Cholesky
  std::vector<double> Lc((size_t)N * N, 0.0);
  for (int j = 0; j < N; j++) {
    double s = K[(size_t)j * N + j];
    for (int k = 0; k < j; k++) s -= Lc[(size_t)j * N + k] * Lc[(size_t)j * N + k];
    if (s <= 0) { std::fprintf(stderr, "oracle: coarsest matrix not SPD\n"); s = 1e-300; }
    double d = std::sqrt(s);
    Lc[(size_t)j * N + j] = d;
    for (int i = j + 1; i < N; i++) {
      double t = K[(size_t)i * N + j];
      for (int k = 0; k < j; k++) t -= Lc[(size_t)i * N + k] * Lc[(size_t)j * N + k];
      Lc[(size_t)i * N + j] = t / d;
    }
  }
  // explicit inverse: solve L L^T X = I
  p->Kinv.assign((size_t)N * N, 0.0);
  std::vector<double> col(N);
  for (int c2 = 0; c2 < N; c2++) {
    for (int i = 0; i < N; i++) {
      double t = (i == c2) ? 1.0 : 0.0;
      for (int k = 0; k < i; k++) t -= Lc[(size_t)i * N + k] * col[k];
      col[i] = t / Lc[(size_t)i * N + i];
    }
    for (int i = N - 1; i >= 0; i--) {
      double t = col[i];
      for (int k = i + 1; k < N; k++) t -= Lc[(size_t)k * N + i] * col[k];
      col[i] = t / Lc[(size_t)i * N + i];
    }
    for (int i = 0; i < N; i++) p->Kinv[(size_t)i * N + c2] = col[i];
  }
  if (k_rig)
    for (int i = 0; i < N; i++)
      for (int j = 0; j < N; j++) {
        double s = 0;
        for (int q = 0; q < k_rig; q++) s += p->rigid_coarse[(size_t)q * N + i] * p->rigid_coarse[(size_t)q * N + j];
        p->Kinv[(size_t)i * N + j] -= s / a_rig;
      }
}

extern "C" void or_coarsest_solve(const or_problem* p, const double* f, double* u) {
  const Level& c = p->L.back();
  int N = 3 * p->nc;
  std::vector<double> fb(N), ub(N, 0.0);
  for (int i = 0; i < p->nc; i++)
    for (int r = 0; r < 3; r++) fb[3 * i + r] = f[r * c.nn + p->cnode[i]];
  for (int i = 0; i < N; i++) {
    double s = 0;
    for (int j = 0; j < N; j++) s += p->Kinv[(size_t)i * N + j] * fb[j];
    ub[i] = s;
  }
  for (long i = 0; i < 3 * c.nn; i++) u[i] = 0;
  for (int i = 0; i < p->nc; i++)
    for (int r = 0; r < 3; r++) u[r * c.nn + p->cnode[i]] = ub[3 * i + r];
}

// ---------------------------------------------------------------- V-cycle
struct Work {
  std::vector<std::vector<double>> u, f, r;
};

static void level_residual(const or_problem* p, int l, const double* u, const double* f, double* r) {
  if (l == 0) fine_apply(p, u, f, r, 1);
  else coarse_apply(p->L[l], u, f, r);
}

// HierarchyGrid::v_cycle (Grid.cpp:2431-2476): down-sweep residual ->
// restrict -> zero u -> pre-smooth; coarsest dense solve; up-sweep
// prolongate -> post-smooth; final fine residual.
extern "C" double or_vcycle(or_problem* p, double* u, const double* f, int pre, int post, int kind,
                            double omega, int symmetric) {
  int nl = (int)p->L.size();
  Work w;
  w.u.resize(nl); w.f.resize(nl); w.r.resize(nl);
  for (int l = 0; l < nl; l++) {
    long nn = p->L[l].nn;
    w.u[l].assign(3 * nn, 0.0); w.f[l].assign(3 * nn, 0.0); w.r[l].assign(3 * nn, 0.0);
  }
  const long nn0 = p->L[0].nn;
  std::copy(u, u + 3 * nn0, w.u[0].begin());
  std::copy(f, f + 3 * nn0, w.f[0].begin());
  for (int l = 0; l < nl; l++) {
    if (l > 0) {
      level_residual(p, l - 1, w.u[l - 1].data(), w.f[l - 1].data(), w.r[l - 1].data());
      or_restrict(p, l, w.r[l - 1].data(), w.f[l].data());
      std::fill(w.u[l].begin(), w.u[l].end(), 0.0);
    }
    double om = kind == 1 ? omega * 2.0 / p->lam[l] : omega;
    if (l < nl - 1) or_smooth(p, l, w.u[l].data(), w.f[l].data(), kind, om, pre, 0);
    else if (nl > 1) or_coarsest_solve(p, w.f[l].data(), w.u[l].data());
    else {  // single level: smoothing only, kept symmetric
      or_smooth(p, l, w.u[l].data(), w.f[l].data(), kind, om, pre, 0);
      or_smooth(p, l, w.u[l].data(), w.f[l].data(), kind, om, post, symmetric ? 1 : 0);
    }
  }
  for (int l = nl - 2; l >= 0; l--) {
    or_prolong(p, l + 1, w.u[l + 1].data(), w.u[l].data());
    double om = kind == 1 ? omega * 2.0 / p->lam[l] : omega;
    or_smooth(p, l, w.u[l].data(), w.f[l].data(), kind, om, post, symmetric ? 1 : 0);
  }
  level_residual(p, 0, w.u[0].data(), w.f[0].data(), w.r[0].data());
  std::copy(w.u[0].begin(), w.u[0].end(), u);
  double rn = std::sqrt(dot3(w.r[0].data(), w.r[0].data(), nn0));
  double fn = std::sqrt(dot3(f, f, nn0));
  return fn > 0 ? rn / fn : rn;
}

extern "C" int or_solve(or_problem* p, double* u, const double* f, double tol, int max_iter, int method,
                        int pre, int post, int kind, double omega, double* rel_res) {
  const long nn = p->L[0].nn;
  double fn = std::sqrt(dot3(f, f, nn));
  if (fn == 0) { for (long i = 0; i < 3 * nn; i++) u[i] = 0; if (rel_res) *rel_res = 0; return 0; }
  if (method == 0) {
    double rr = 1;
    int it = 0;
    while (it < max_iter) {
      rr = or_vcycle(p, u, f, pre, post, kind, omega, 0);
      it++;
      if (rr < tol) break;
    }
    p->solve_iters += it;
    displacement_project(p, u);
    if (rel_res) *rel_res = rr;
    return it;
  }
  std::vector<double> r(3 * nn), z(3 * nn), pp(3 * nn), q(3 * nn);
  or_residual(p, u, f, r.data());
  for (long i = 0; i < nn; i++)
    if (p->support[i]) r[i] = r[nn + i] = r[2 * nn + i] = 0;
  double rn = std::sqrt(dot3(r.data(), r.data(), nn));
  if (rn / fn < tol) { if (rel_res) *rel_res = rn / fn; return 0; }
  std::fill(z.begin(), z.end(), 0.0);
  or_vcycle(p, z.data(), r.data(), pre, post, kind, omega, 1);
  pp = z;
  double rz = dot3(r.data(), z.data(), nn);
  int it = 0;
  while (it < max_iter) {
    or_apply_K(p, pp.data(), q.data());
    for (long i = 0; i < nn; i++)
      if (p->support[i]) q[i] = q[nn + i] = q[2 * nn + i] = 0;
    double alpha = rz / dot3(pp.data(), q.data(), nn);
    for (long i = 0; i < 3 * nn; i++) { u[i] += alpha * pp[i]; r[i] -= alpha * q[i]; }
    it++;
    rn = std::sqrt(dot3(r.data(), r.data(), nn));
    if (rn / fn < tol) break;
    std::fill(z.begin(), z.end(), 0.0);
    or_vcycle(p, z.data(), r.data(), pre, post, kind, omega, 1);
    double rz2 = dot3(r.data(), z.data(), nn);
    double beta = rz2 / rz;
    rz = rz2;
    for (long i = 0; i < 3 * nn; i++) pp[i] = z[i] + beta * pp[i];
  }
  p->solve_iters += it;
  // support-free problems: the solution without rigid motion (displacementProject)
  displacement_project(p, u);
  // true residual
  or_residual(p, u, f, r.data());
  for (long i = 0; i < nn; i++)
    if (p->support[i]) r[i] = r[nn + i] = r[2 * nn + i] = 0;
  if (rel_res) *rel_res = std::sqrt(dot3(r.data(), r.data(), nn)) / fn;
  return it;
}
