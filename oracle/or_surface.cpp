// Surface-point self-support: FP64 CPU restatement (test infrastructure only).
//
// The reference samples the design's iso-surface rho = 0.5 and evaluates the
// overhang constraint at those points (deal_surface_points,
// optimization/optimization.cpp:1185-1221):
//   - background values: the spline minus 0.5 at the (mc + 2)^3 cell centres
//     of the model box enlarged by one cell, 0 outside the box
//     (Grid::compute_background_mcPoints_value, grid/Grid.cu:4066-4175);
//   - marching cubes at iso value 0, a corner counting as inside when its
//     value is <= 0, crossing points by linear interpolation
//     (marchingcube/MarchingCube.cpp:23-31, :58-113);
//   - an equal-distance pick of 3 n points when there are more than 2 n per
//     requested point, the points inside the model, and a final pick of n,
//     padded with the first point when fewer remain and placed at the origin
//     when none remain (Grid::compute_surface_nodes_in_model,
//     grid/Grid.cpp:3861-4060; generateEquidistantIntegers :3831-3847);
//   - normals = the spline gradient, turned outward by a probe 1e-3 along it
//     (grid/Grid.cu:5709-5943); flags (:5945-6040); the per-point constraint
//     (:6198-6283), its mean (:6285-6328) and its coefficient gradient divided
//     by the count (:6330-6505; grid/Grid.cpp:4263-4280).
//
// Deliberate differences, shared with the CUDA path:
//   - one sample per grid-edge crossing, ordered by edge (grid point x fastest,
//     then y, z; then the edge axis x, y, z), interpolated from the lower
//     corner to the upper one.  The reference lists the first corner of every
//     marching-cubes triangle in table order, so a crossing appears once per
//     triangle it starts;
//   - "inside the model" is "inside an active element".  The reference casts a
//     ray against the input mesh with a CGAL AABB tree from an OpenMP loop
//     whose critical section fixes the order of the kept points run by run;
//   - picks are clamped to the list (the reference's last pick can index one
//     past its end) and a pick of the whole list keeps it;
//   - the spline sums and the constraint run in double (float in the
//     reference); a point whose normal is zero contributes nothing (the
//     reference divides 0 by 0 there).
#include "or_internal.h"

// spline basis values and first derivatives at coordinate u (Cox-de Boor,
// Piegl-Tiller A2.2/A2.3: the recursion of SplineBasisDeriX, Grid.cu:514-610).
// The span index is formed in float as the reference does.
static bool basis_d(const or_problem* p, int a, double u, int* I, double* N, double* dN) {
  const int o = p->order, pdeg = o - 1;
  const float pf = (float)u;
  const int i = (int)((pf - p->bmin[a]) / p->step[a]) + o;
  *I = i;
  if (i < o || i > p->nb[a]) return false;
  const int span = i - 1;
  const auto& K = p->knots[a];
  double ndu[6][6], left[6], right[6];
  ndu[0][0] = 1.0;
  for (int j = 1; j <= pdeg; j++) {
    left[j] = u - (double)K[span + 1 - j];
    right[j] = (double)K[span + j] - u;
    double saved = 0.0;
    for (int r = 0; r < j; r++) {
      ndu[j][r] = right[r + 1] + left[j - r];
      const double temp = ndu[r][j - 1] / ndu[j][r];
      ndu[r][j] = saved + right[r + 1] * temp;
      saved = left[j - r] * temp;
    }
    ndu[j][j] = saved;
  }
  for (int j = 0; j <= pdeg; j++) N[j] = ndu[j][pdeg];
  for (int r = 0; r <= pdeg; r++) {
    double d = 0;
    if (pdeg >= 1) {
      if (r >= 1) d = ndu[r - 1][pdeg - 1] / ndu[pdeg][r - 1];
      if (r <= pdeg - 1) d -= ndu[r][pdeg - 1] / ndu[pdeg][r];
      d *= pdeg;
    }
    dN[r] = d;
  }
  return true;
}

// spline value and gradient at a point; false outside the knot support
static bool spline_vg(const or_problem* p, const double* c, const double pt[3], double* v, double g[3]) {
  const int o = p->order, nbx = p->nb[0], nby = p->nb[1];
  int I[3];
  double N[3][6], D[3][6];
  for (int a = 0; a < 3; a++)
    if (!basis_d(p, a, pt[a], &I[a], N[a], D[a])) return false;
  double s = 0, g0 = 0, g1 = 0, g2 = 0;
  for (int q = 0; q < o; q++)
    for (int b = 0; b < o; b++)
      for (int a = 0; a < o; a++) {
        const double cc = c[(I[0] - o + a) + (long)(I[1] - o + b) * nbx + (long)(I[2] - o + q) * nbx * nby];
        s += cc * N[0][a] * N[1][b] * N[2][q];
        g0 += cc * D[0][a] * N[1][b] * N[2][q];
        g1 += cc * N[0][a] * D[1][b] * N[2][q];
        g2 += cc * N[0][a] * N[1][b] * D[2][q];
      }
  *v = s;
  g[0] = g0; g[1] = g1; g[2] = g2;
  return true;
}

// cell-centre coordinate of background point index x along one axis:
// boxOrispan + x * eh + 0.5 * eh, float then double as the reference writes it
static float mc_coord(float lo, float eh, int x) {
  const float span = lo - eh;
  return (float)((double)(span + (float)x * eh) + 0.5 * (double)eh);
}

extern "C" void or_mc_values(const or_problem* p, const double* c, int mc, const float* box, float* val, float* pos3) {
  const int n = mc + 2;
  float eh[3];
  for (int a = 0; a < 3; a++) eh[a] = (box[3 + a] - box[a]) / (float)mc;
  for (int z = 0; z < n; z++)
    for (int y = 0; y < n; y++)
      for (int x = 0; x < n; x++) {
        const int id[3] = {x, y, z};
        float pos[3];
        bool outside_box = false;
        for (int a = 0; a < 3; a++) {
          pos[a] = mc_coord(box[a], eh[a], id[a]);
          if (pos[a] < box[a] || pos[a] > box[3 + a]) outside_box = true;
        }
        const double pt[3] = {pos[0], pos[1], pos[2]};
        double v, g[3];
        float vf = spline_vg(p, c, pt, &v, g) ? (float)v : -0.2f;
        if (outside_box) vf = 0.f;
        const long id3 = x + (long)n * (y + (long)n * z);
        val[id3] = (float)((double)vf - 0.5);
        if (pos3)
          for (int a = 0; a < 3; a++) pos3[(long)a * n * n * n + id3] = pos[a];
      }
}

// generateEquidistantIntegers (grid/Grid.cpp:3831-3847): int(i * range / (m - 1)),
// clamped to the list; m >= range keeps every index
extern "C" long or_equidistant(long range, long m, long* out) {
  if (m >= range) {
    for (long i = 0; i < range; i++) out[i] = i;
    return range;
  }
  const double step = m > 1 ? (double)range / (double)(m - 1) : 0.0;
  for (long i = 0; i < m; i++) out[i] = std::min((long)(i * step), range - 1);
  return m;
}

namespace {
struct Crossing {
  float p[3];
  bool in_model;
};
}

// the crossing of the edge from background point g (x, y, z) along axis a
static Crossing crossing_at(const or_problem* p, const float* val, int n, const float* box, const float* eh, int x,
                            int y, int z, int a) {
  const int id[3] = {x, y, z};
  int id2[3] = {x, y, z};
  id2[a] += 1;
  const float v1 = val[x + (long)n * (y + (long)n * z)];
  const float v2 = val[id2[0] + (long)n * (id2[1] + (long)n * id2[2])];
  Crossing cr;
  for (int b = 0; b < 3; b++) cr.p[b] = mc_coord(box[b], eh[b], id[b]);
  if (std::fabs(v1 - v2) > 0.00001f) {
    const float p2 = mc_coord(box[a], eh[a], id2[a]);
    const float t = (p2 - cr.p[a]) / (v2 - v1);
    cr.p[a] = cr.p[a] + t * (0.f - v1);
  }
  const orc::Level& l = p->L[0];
  const int dims[3] = {l.ex, l.ey, l.ez};
  int e[3];
  bool in = true;
  for (int b = 0; b < 3; b++) {
    const float f = std::floor(cr.p[b]);
    if (!(f >= 0.f && f < (float)dims[b])) { in = false; break; }
    e[b] = (int)f;
  }
  cr.in_model = in && l.emask[l.eidx(e[0], e[1], e[2])];
  return cr;
}

// info[0] crossings, info[1] after the first pick, info[2] inside the model,
// info[3] points written (npts, or 0 when npts <= 0)
extern "C" int or_surface_points(const or_problem* p, const double* c, int mc, int npts, const float* box,
                                 float* xyz, long* info) {
  const int n = mc + 2;
  std::vector<float> val((size_t)n * n * n);
  or_mc_values(p, c, mc, box, val.data(), nullptr);
  float eh[3];
  for (int a = 0; a < 3; a++) eh[a] = (box[3 + a] - box[a]) / (float)mc;
  std::vector<long> edges;
  for (int z = 0; z < n; z++)
    for (int y = 0; y < n; y++)
      for (int x = 0; x < n; x++) {
        const long g = x + (long)n * (y + (long)n * z);
        const bool in0 = val[g] <= 0.f;
        const int id[3] = {x, y, z};
        const long st[3] = {1, n, (long)n * n};
        for (int a = 0; a < 3; a++) {
          if (id[a] + 1 >= n) continue;
          if ((val[g + st[a]] <= 0.f) != in0) edges.push_back(3 * g + a);
        }
      }
  const long num = (long)edges.size();
  std::vector<long> picked;
  if (npts > 0 && num / npts > 2) {
    std::vector<long> idx(3 * (long)npts);
    const long m = or_equidistant(num, 3 * (long)npts, idx.data());
    for (long j = 0; j < m; j++) picked.push_back(edges[idx[j]]);
  } else {
    picked = edges;
  }
  std::vector<Crossing> kept;
  for (long e : picked) {
    const long g = e / 3;
    const int a = (int)(e % 3);
    const int x = (int)(g % n), y = (int)(g / n % n), z = (int)(g / ((long)n * n));
    Crossing cr = crossing_at(p, val.data(), n, box, eh, x, y, z, a);
    if (cr.in_model) kept.push_back(cr);
  }
  if (info) {
    info[0] = num;
    info[1] = (long)picked.size();
    info[2] = (long)kept.size();
    info[3] = npts > 0 ? npts : 0;
  }
  if (npts <= 0) return 0;
  const long nk = (long)kept.size();
  std::vector<long> src(npts, 0);
  if (nk >= npts) or_equidistant(nk, npts, src.data());
  else
    for (long j = 0; j < nk; j++) src[j] = j;
  for (long j = 0; j < npts; j++)
    for (int b = 0; b < 3; b++) xyz[(long)b * npts + j] = nk > 0 ? kept[src[j]].p[b] : 0.f;
  return npts;
}

static double Hs(double s, double beta) {
  const double eta = 0.5;
  return (std::tanh(beta * eta) + std::tanh(beta * (s - eta))) / (std::tanh(beta * eta) + std::tanh(beta * (1 - eta)));
}

// per-point penalty f(inner) and f'(inner) of mode m (grid/Grid.cu:123-155;
// p_norm 8, hfunction_c 10, sigmoid_c 0.09, grid/Grid.h:371-375)
static void surf_pen(int m, double inner, double* f, double* df) {
  if (m <= 1) {
    *f = std::pow(inner, 8.0);
    *df = 8.0 * std::pow(inner, 7.0);
  } else if (m <= 3) {
    *f = inner >= 1 ? 10.0 * (inner - 1) * (inner - 1) : 0;
    *df = inner >= 1 ? 20.0 * (inner - 1) : 0;
  } else {
    const double c = 0.09, e = std::exp(-(inner - 1.5) / c);
    *f = 1 / (1 + e);
    *df = 1 / (1 + e) / (1 + e) / c * e;
  }
}

// normals[3n] (SoA, outward), per[n], flags[2n] (actual, virtual), dc[n_coeff]
// (divided by the count) may be NULL.  Returns the constraint value.
extern "C" double or_surface_selfsupport(const or_problem* p, const double* c, const float* xyz, long n, double beta,
                                         int mode, double opt_angle, double default_angle, double* normals,
                                         double* per, uint8_t* flags, double* dc, double* count_out,
                                         double* dirsum_out) {
  const int o = p->order, nbx = p->nb[0], nby = p->nb[1];
  const long ncoef = (long)p->nb[0] * p->nb[1] * p->nb[2];
  std::vector<double> nv(3 * n, 0.0);
  std::vector<uint8_t> ins(n, 0);
  double dirsum = 0;
  for (long k = 0; k < n; k++) {
    const double pt[3] = {xyz[k], xyz[n + k], xyz[2 * n + k]};
    double v, g[3] = {0, 0, 0};
    ins[k] = spline_vg(p, c, pt, &v, g);
    if (!ins[k]) g[0] = g[1] = g[2] = 0;
    for (int a = 0; a < 3; a++) nv[3 * k + a] = g[a];
    // orientation probe 1e-3 along the (unnormalised) gradient
    const double pd[3] = {pt[0] + 1e-3 * g[0], pt[1] + 1e-3 * g[1], pt[2] + 1e-3 * g[2]};
    double vd, gd[3];
    if (!spline_vg(p, c, pd, &vd, gd)) vd = -0.1;
    dirsum += Hs(vd, beta) < 0.5 ? 1.0 : -1.0;
  }
  if (dirsum_out) *dirsum_out = dirsum;
  const double flip = dirsum < 0 ? -1.0 : 1.0;
  const double direction = dirsum > 0 ? 1.0 : -1.0;
  const double cosang = std::cos(opt_angle), cosdef = std::cos(default_angle);
  double sum = 0, down_cnt = 0;
  for (long k = 0; k < n; k++) {
    double* q = &nv[3 * k];
    for (int a = 0; a < 3; a++) q[a] *= flip;
    const double nn = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
    const bool down = q[2] < 0;
    if (down) down_cnt += 1;
    double f = 0, df = 0;
    if (nn > 0 && (mode % 2 == 1 || down)) surf_pen(mode, q[2] / nn / cosang, &f, &df);
    if (per) per[k] = f;
    sum += f;
    if (flags) {
      flags[k] = (down && nn > 0 && q[2] / nn / cosdef > 1) ? 1 : 0;
      flags[n + k] = (down && nn > 0 && q[2] / nn / cosang > 1) ? 1 : 0;
    }
    if (normals)
      for (int a = 0; a < 3; a++) normals[(long)a * n + k] = q[a];
  }
  const double cnt = (mode % 2 == 0) ? down_cnt : (double)n;
  if (count_out) *count_out = cnt;
  double value = 0;
  if (cnt != 0) value = mode <= 1 ? std::pow(sum / cnt, 1 / 8.0) - 1 : sum / cnt;
  if (dc) {
    for (long i = 0; i < ncoef; i++) dc[i] = 0;
    for (long k = 0; k < n; k++) {
      const double* q = &nv[3 * k];
      const double nn = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
      const bool down = q[2] < 0;
      if (!ins[k] || nn == 0 || !(mode % 2 == 1 || down)) continue;
      const double inner = q[2] / nn / cosang;
      double f, df;
      surf_pen(mode, inner, &f, &df);
      const double pt[3] = {xyz[k], xyz[n + k], xyz[2 * n + k]};
      int I[3];
      double N[3][6], D[3][6];
      for (int a = 0; a < 3; a++) basis_d(p, a, pt[a], &I[a], N[a], D[a]);
      const double den = nn * nn * cosang;
      for (int qz = 0; qz < o; qz++)
        for (int b = 0; b < o; b++)
          for (int a = 0; a < o; a++) {
            const double nd[3] = {direction * D[0][a] * N[1][b] * N[2][qz], direction * N[0][a] * D[1][b] * N[2][qz],
                                  direction * N[0][a] * N[1][b] * D[2][qz]};
            const double normdc = (q[0] * nd[0] + q[1] * nd[1] + q[2] * nd[2]) / nn;
            const double dinner = (nd[2] * nn - q[2] * normdc) / den;
            dc[(I[0] - o + a) + (long)(I[1] - o + b) * nbx + (long)(I[2] - o + qz) * nbx * nby] += df * dinner;
          }
    }
    const double scale = cnt == 0 ? 0.0 : 1.0 / cnt;
    for (long i = 0; i < ncoef; i++) dc[i] *= scale;
  }
  return value;
}
