// FP64 CPU oracle: compliance sensitivity, Heaviside projection, filters,
// B-spline density map and its adjoint, self-support constraint.
// TEST INFRASTRUCTURE ONLY (see oracle.h).
#include "or_internal.h"

using namespace orc;

// u_e^T K0 u_e per active element (elementCompliance_kernel Grid.cu:5569-5610,
// without the rho^p factor)
static double elem_quad(const or_problem* p, const double* u, int x, int y, int z) {
  const Level& l = p->L[0];
  double ue[24];
  for (int a = 0; a < 8; a++) {
    long n = l.nidx(x + a % 2, y + a / 2 % 2, z + a / 4);
    for (int c = 0; c < 3; c++) ue[3 * a + c] = u[c * l.nn + n];
  }
  double s = 0;
  for (int i = 0; i < 24; i++) {
    double t = 0;
    for (int j = 0; j < 24; j++) t += p->K0[i * 24 + j] * ue[j];
    s += ue[i] * t;
  }
  return s;
}

// dC/drho_e = -p rho_e^(p-1) u_e^T K0 u_e  (computeSensitivity_kernel,
// optimization/optimization.cu:102-165)
extern "C" void or_sensitivity(const or_problem* p, const double* u, double* sens) {
  const Level& l = p->L[0];
#pragma omp parallel for collapse(2)
  for (int z = 0; z < l.ez; z++)
    for (int y = 0; y < l.ey; y++)
      for (int x = 0; x < l.ex; x++) {
        long e = l.eidx(x, y, z);
        if (!l.emask[e]) { sens[e] = 0; continue; }
        double q = elem_quad(p, u, x, y, z);
        sens[e] = -p->penal * std::pow(p->rho[e], p->penal - 1) * q;
      }
}

extern "C" void or_element_energy(const or_problem* p, const double* u, double* energy) {
  const Level& l = p->L[0];
#pragma omp parallel for collapse(2)
  for (int z = 0; z < l.ez; z++)
    for (int y = 0; y < l.ey; y++)
      for (int x = 0; x < l.ex; x++) {
        long e = l.eidx(x, y, z);
        energy[e] = l.emask[e] ? p->rhop[e] * elem_quad(p, u, x, y, z) : 0.0;
      }
}

// Heaviside projection, eta = 0.5 (computeProjection_kernel optimization.cu:324-348)
extern "C" void or_heaviside(int n, const double* rin, double beta, double rhomin, const uint8_t* shell,
                             double* rout) {
  const double eta = 0.5;
  double den = std::tanh(beta * eta) + std::tanh(beta * (1 - eta));
  for (int i = 0; i < n; i++) {
    double v = (std::tanh(beta * eta) + std::tanh(beta * (rin[i] - eta))) / den;
    v = std::min(std::max(v, rhomin), 1.0);
    if (shell && shell[i]) v = 1;
    rout[i] = v;
  }
}

// chain with H'(rho) (computeProjectionSensitivity_kernel optimization.cu:167-189)
extern "C" void or_heaviside_chain(int n, const double* rin, double beta, const double* gin, double* gout) {
  const double eta = 0.5;
  double den = std::tanh(beta * eta) + std::tanh(beta * (1 - eta));
  for (int i = 0; i < n; i++) {
    double t = std::tanh(beta * (rin[i] - eta));
    gout[i] = gin[i] * beta * (1 - t * t) / den;
  }
}

// sensitivity filter (filterSensitivity_kernel Grid.cu:4210-4296): integer
// reach R = int(Rf + 0.5), neighbours with |d|^2 <= Rf^2, weight
// w(r) = 1 - 6r^2 + 8r^3 - 3r^4 with r = |d|/Rf, inactive neighbours skipped.
static inline double fweight(double r2, double R2) {
  double r = std::sqrt(r2 / R2);
  double rr = r * r;
  return 1 - 6 * rr + 8 * rr * r - 3 * rr * rr;
}

extern "C" void or_filter(const or_problem* p, double Rf, const double* in, double* out) {
  const Level& l = p->L[0];
  int R = (int)(Rf + 0.5);
  double R2 = Rf * Rf;
#pragma omp parallel for collapse(2)
  for (int z = 0; z < l.ez; z++)
    for (int y = 0; y < l.ey; y++)
      for (int x = 0; x < l.ex; x++) {
        long e = l.eidx(x, y, z);
        if (!l.emask[e]) { out[e] = 0; continue; }
        double gs = 0, ws = 0;
        for (int dx = -R; dx <= R; dx++)
          for (int dy = -R; dy <= R; dy++)
            for (int dz = -R; dz <= R; dz++) {
              int xx = x + dx, yy = y + dy, zz = z + dz;
              if (xx < 0 || yy < 0 || zz < 0 || xx >= l.ex || yy >= l.ey || zz >= l.ez) continue;
              double r2 = dx * dx + dy * dy + dz * dz;
              if (r2 > R2) continue;
              long n = l.eidx(xx, yy, zz);
              if (!l.emask[n]) continue;
              double w = fweight(r2, R2);
              gs += w * in[n];
              ws += w;
            }
        out[e] = gs / ws;
      }
}

// consistent density filter (build mode): out_e = sum_n w_en in_n / W_e
extern "C" void or_density_filter(const or_problem* p, double Rf, const double* in, double* out) {
  or_filter(p, Rf, in, out);
}

// its adjoint: out_n = sum_e w_en in_e / W_e
extern "C" void or_density_filter_adjoint(const or_problem* p, double Rf, const double* in, double* out) {
  const Level& l = p->L[0];
  int R = (int)(Rf + 0.5);
  double R2 = Rf * Rf;
  std::vector<double> scaled(l.ne, 0.0);
  for (int z = 0; z < l.ez; z++)
    for (int y = 0; y < l.ey; y++)
      for (int x = 0; x < l.ex; x++) {
        long e = l.eidx(x, y, z);
        if (!l.emask[e]) continue;
        double ws = 0;
        for (int dx = -R; dx <= R; dx++)
          for (int dy = -R; dy <= R; dy++)
            for (int dz = -R; dz <= R; dz++) {
              int xx = x + dx, yy = y + dy, zz = z + dz;
              if (xx < 0 || yy < 0 || zz < 0 || xx >= l.ex || yy >= l.ey || zz >= l.ez) continue;
              double r2 = dx * dx + dy * dy + dz * dz;
              if (r2 > R2 || !l.emask[l.eidx(xx, yy, zz)]) continue;
              ws += fweight(r2, R2);
            }
        scaled[e] = in[e] / ws;
      }
  // the weights are symmetric, so the adjoint is a gather of scaled inputs
  for (int z = 0; z < l.ez; z++)
    for (int y = 0; y < l.ey; y++)
      for (int x = 0; x < l.ex; x++) {
        long e = l.eidx(x, y, z);
        if (!l.emask[e]) { out[e] = 0; continue; }
        double s = 0;
        for (int dx = -R; dx <= R; dx++)
          for (int dy = -R; dy <= R; dy++)
            for (int dz = -R; dz <= R; dz++) {
              int xx = x + dx, yy = y + dy, zz = z + dz;
              if (xx < 0 || yy < 0 || zz < 0 || xx >= l.ex || yy >= l.ey || zz >= l.ez) continue;
              double r2 = dx * dx + dy * dy + dz * dz;
              long n = l.eidx(xx, yy, zz);
              if (r2 > R2 || !l.emask[n]) continue;
              s += fweight(r2, R2) * scaled[n];
            }
        out[e] = s;
      }
}

// ---------------------------------------------------------------- spline
// knot series (Grid.cpp:3307-3431): domain [0, e] enlarged by 2 spans' worth
// of the box on each side, step = (max-min)/(P+1), 'order' repeated end knots.
// All in float, as the reference.
extern "C" int or_spline_setup(or_problem* p, int order, int px, int py, int pz) {
  p->order = order;
  p->part[0] = px; p->part[1] = py; p->part[2] = pz;
  const Level& l = p->L[0];
  int edim[3] = {l.ex, l.ey, l.ez};
  for (int a = 0; a < 3; a++) {
    int P = p->part[a];
    p->nb[a] = order + P;
    float mn = 0.0f, mx = (float)edim[a];
    float delta = mx - mn;
    float scale_bound = 2.0f;
    mx += scale_bound * delta / (float)(P + 1);
    mn -= scale_bound * delta / (float)(P + 1);
    p->bmin[a] = mn; p->bmax[a] = mx;
    p->step[a] = (mx - mn) / (float)(P + 1);
    auto& K = p->knots[a];
    K.clear();
    float tmp = mn;
    for (int i = 0; i < order; i++) K.push_back(mn);
    for (int i = order; i < order + P; i++) { tmp += p->step[a]; K.push_back(tmp); }
    for (int i = order + P; i < 2 * order + P; i++) K.push_back(mx);
    // per element-coordinate tables
    p->sidx[a].assign(edim[a], 0);
    p->sN[a].assign((size_t)edim[a] * order, 0.0);
    p->sdN[a].assign((size_t)edim[a] * order, 0.0);
    p->sinside[a].assign(edim[a], 0);
    for (int x = 0; x < edim[a]; x++) {
      float eh = 1.0f, org = 0.0f;
      float pos = (float)((double)(org + x * eh) + 0.5 * eh);
      int i = (int)((pos - p->bmin[a]) / p->step[a]) + order;
      p->sidx[a][x] = i;
      bool inside = !(i < order || i > p->nb[a]);
      p->sinside[a][x] = inside;
      if (!inside) continue;
      // Cox-de Boor values and first derivatives (Piegl-Tiller A2.2/A2.3,
      // the recursion of SplineBasisX / SplineBasisDeriX Grid.cu:427-857)
      int span = i - 1;
      int pdeg = order - 1;
      double u = pos;
      std::vector<std::vector<double>> ndu(order, std::vector<double>(order, 0.0));
      std::vector<double> left(order, 0.0), right(order, 0.0);
      ndu[0][0] = 1.0;
      for (int j = 1; j <= pdeg; j++) {
        left[j] = u - (double)K[span + 1 - j];
        right[j] = (double)K[span + j] - u;
        double saved = 0.0;
        for (int r = 0; r < j; r++) {
          ndu[j][r] = right[r + 1] + left[j - r];
          double temp = ndu[r][j - 1] / ndu[j][r];
          ndu[r][j] = saved + right[r + 1] * temp;
          saved = left[j - r] * temp;
        }
        ndu[j][j] = saved;
      }
      for (int j = 0; j <= pdeg; j++) p->sN[a][(size_t)x * order + j] = ndu[j][pdeg];
      // first derivative
      for (int r = 0; r <= pdeg; r++) {
        double d = 0.0;
        int k = 1, rk = r - k, pk = pdeg - k;
        double a0 = 1.0, a1[2] = {0, 0};
        if (pdeg >= 1) {
          if (r >= k) { a1[0] = a0 / ndu[pk + 1][rk]; d = a1[0] * ndu[rk][pk]; }
          if (r <= pk) { a1[1] = -a0 / ndu[pk + 1][r]; d += a1[1] * ndu[r][pk]; }
          d *= pdeg;
        }
        p->sdN[a][(size_t)x * order + r] = d;
      }
    }
  }
  return p->nb[0] * p->nb[1] * p->nb[2];
}

extern "C" void or_spline_info(const or_problem* p, int* nbasis, float* bmin, float* step) {
  for (int a = 0; a < 3; a++) { nbasis[a] = p->nb[a]; bmin[a] = p->bmin[a]; step[a] = p->step[a]; }
}

extern "C" void or_spline_axis(const or_problem* p, int axis, int* idx, double* N, double* dN) {
  size_t n = p->sidx[axis].size();
  for (size_t i = 0; i < n; i++) idx[i] = p->sinside[axis][i] ? p->sidx[axis][i] : -1;
  std::copy(p->sN[axis].begin(), p->sN[axis].end(), N);
  std::copy(p->sdN[axis].begin(), p->sdN[axis].end(), dN);
}

// rho_hat_e = clamp(sum_ijk c N_i N_j N_k, rhomin, 1); outside -> -0.2; shell -> 1
// (coeff2density Grid.cu:3405-3536)
extern "C" void or_coeff2density(const or_problem* p, const double* c, double rhomin, const uint8_t* shell,
                                 double* rho_hat) {
  const Level& l = p->L[0];
  const int o = p->order;
  const int nbx = p->nb[0], nby = p->nb[1];
#pragma omp parallel for collapse(2)
  for (int z = 0; z < l.ez; z++)
    for (int y = 0; y < l.ey; y++)
      for (int x = 0; x < l.ex; x++) {
        long e = l.eidx(x, y, z);
        if (!l.emask[e]) { rho_hat[e] = 0; continue; }
        double v;
        if (!p->sinside[0][x] || !p->sinside[1][y] || !p->sinside[2][z]) v = -0.2;
        else {
          int i = p->sidx[0][x], j = p->sidx[1][y], k = p->sidx[2][z];
          v = 0;
          for (int ir = i - o; ir < i; ir++)
            for (int is = j - o; is < j; is++)
              for (int it = k - o; it < k; it++)
                v += c[ir + (long)is * nbx + (long)it * nbx * nby] * p->sN[0][(size_t)x * o + ir - i + o] *
                     p->sN[1][(size_t)y * o + is - j + o] * p->sN[2][(size_t)z * o + it - k + o];
        }
        v = std::min(std::max(v, rhomin), 1.0);
        if (shell && shell[e]) v = 1;
        rho_hat[e] = v;
      }
}

// race-free adjoint dC/dc_k = sum_e g_e N_k(x_e) over active non-shell
// elements inside the spline domain (ddensity2dcoeff Grid.cu:3566-3721)
extern "C" void or_density2coeff_adjoint(const or_problem* p, const double* g, const uint8_t* shell, double* dc) {
  const Level& l = p->L[0];
  const int o = p->order;
  const int nbx = p->nb[0], nby = p->nb[1];
  long nc = (long)p->nb[0] * p->nb[1] * p->nb[2];
  for (long i = 0; i < nc; i++) dc[i] = 0;
  for (int z = 0; z < l.ez; z++)
    for (int y = 0; y < l.ey; y++)
      for (int x = 0; x < l.ex; x++) {
        long e = l.eidx(x, y, z);
        if (!l.emask[e] || (shell && shell[e])) continue;
        if (!p->sinside[0][x] || !p->sinside[1][y] || !p->sinside[2][z]) continue;
        int i = p->sidx[0][x], j = p->sidx[1][y], k = p->sidx[2][z];
        for (int ir = i - o; ir < i; ir++)
          for (int is = j - o; is < j; is++)
            for (int it = k - o; it < k; it++)
              dc[ir + (long)is * nbx + (long)it * nbx * nby] +=
                  g[e] * p->sN[0][(size_t)x * o + ir - i + o] * p->sN[1][(size_t)y * o + is - j + o] *
                  p->sN[2][(size_t)z * o + it - k + o];
      }
}

// ---------------------------------------------------------------- self-support
// penalty pieces (Grid.cu:123-190, 3161-3185)
static double Hs(double s, double beta) {
  double eta = 0.5;
  return (std::tanh(beta * eta) + std::tanh(beta * (s - eta))) / (std::tanh(beta * eta) + std::tanh(beta * (1 - eta)));
}
static double hfun(double x, double c) { return x >= 1 ? c * (x - 1) * (x - 1) : 0; }
static double dhfun(double x, double c) { return x >= 1 ? 2 * c * (x - 1) : 0; }
static double overhang(double x, double mid, double c) { return 2 / (1 + std::exp(-(x - mid) / c)); }
static double doverhang(double x, double mid, double c) {
  double e = std::exp(-(x - mid) / c);
  return 2 / (1 + e) / (1 + e) / c * e;
}
static double ndist(double x, double a) { return std::exp(-a * (x - 0.5) * (x - 0.5)); }
static double dndist(double x, double a) { return -2 * a * (x - 0.5) * std::exp(-a * (x - 0.5) * (x - 0.5)); }
static double inner_(double x, double a) { return x > 1 ? a * (x - 1) + 1 : 1; }
static double dinner_(double x, double a) { return x > 1 ? a : 1; }

// the pieces above at given points, for the golden fixtures of the
// reference's own functions (Heaviside, Dirac Grid.cu:76-121; h, dh, inner_,
// dinner_, overhang, doverhang, normal_distri, dnormal_distri :123-190):
// out[k * n + i], k in that order
extern "C" void or_ss_funcs(int n, const double* x, double beta, double a, double mid, double c, double* out) {
  const double eta = 0.5;
  const double den = std::tanh(beta * eta) + std::tanh(beta * (1 - eta));
  for (int i = 0; i < n; i++) {
    const double t = std::tanh(beta * (x[i] - eta));
    out[0 * (size_t)n + i] = Hs(x[i], beta);
    out[1 * (size_t)n + i] = beta * (1 - t * t) / den;
    out[2 * (size_t)n + i] = hfun(x[i], a);
    out[3 * (size_t)n + i] = dhfun(x[i], a);
    out[4 * (size_t)n + i] = inner_(x[i], a);
    out[5 * (size_t)n + i] = dinner_(x[i], a);
    out[6 * (size_t)n + i] = overhang(x[i], mid, c);
    out[7 * (size_t)n + i] = doverhang(x[i], mid, c);
    out[8 * (size_t)n + i] = ndist(x[i], a);
    out[9 * (size_t)n + i] = dndist(x[i], a);
  }
}

// spline value at an arbitrary point (SplineBasisX + coefficient sum)
static double spline_value_at(const or_problem* p, const double* c, const double pt[3], bool* inside) {
  const int o = p->order;
  int I[3];
  std::vector<double> Nv[3];
  for (int a = 0; a < 3; a++) {
    float pf = (float)pt[a];
    int i = (int)((pf - p->bmin[a]) / p->step[a]) + o;
    I[a] = i;
    if (i < o || i > p->nb[a]) { *inside = false; return 0; }
    int span = i - 1, pdeg = o - 1;
    const auto& K = p->knots[a];
    std::vector<double> N(o, 0.0), left(o, 0.0), right(o, 0.0);
    N[0] = 1.0;
    double u = pt[a];
    for (int j = 1; j <= pdeg; j++) {
      left[j] = u - (double)K[span + 1 - j];
      right[j] = (double)K[span + j] - u;
      double saved = 0;
      for (int r = 0; r < j; r++) {
        double temp = N[r] / (right[r + 1] + left[j - r]);
        N[r] = saved + right[r + 1] * temp;
        saved = left[j - r] * temp;
      }
      N[j] = saved;
    }
    Nv[a] = N;
  }
  *inside = true;
  double v = 0;
  const int nbx = p->nb[0], nby = p->nb[1];
  for (int ir = I[0] - o; ir < I[0]; ir++)
    for (int is = I[1] - o; is < I[1]; is++)
      for (int it = I[2] - o; it < I[2]; it++)
        v += c[ir + (long)is * nbx + (long)it * nbx * nby] * Nv[0][ir - I[0] + o] * Nv[1][is - I[1] + o] *
             Nv[2][it - I[2] + o];
  return v;
}

// deal_background_points (optimization.cpp:1223-1242) -> Grid.cu:7449-8250.
extern "C" double or_selfsupport(const or_problem* p, const double* c, double beta, int mode, double opt_angle,
                                 double default_angle, double* per_element, double* dc, double* count_out,
                                 double* direction_sum) {
  const Level& l = p->L[0];
  const int o = p->order;
  const int nbx = p->nb[0], nby = p->nb[1];
  long ncoef = (long)p->nb[0] * p->nb[1] * p->nb[2];
  double mid = std::cos(M_PI) / std::cos(default_angle);
  double sc = (mid - 1) / std::log(1 / 0.004 - 1);
  const double p_norm = 8.0, hfc = 10.0, na = 200.0, ia = 15.0;  // Grid.h:371-378
  double fpara = (mode <= 1) ? p_norm : (mode <= 3 ? hfc : sc);
  double cosang = std::cos(opt_angle);
  // 1) value and gradient at element centres
  std::vector<long> elist;
  for (long e = 0; e < l.ne; e++) if (l.emask[e]) elist.push_back(e);
  long n = (long)elist.size();
  std::vector<double> fv(n), gr(3 * n), dir(n);
  for (long k = 0; k < n; k++) {
    long e = elist[k];
    int x = e % l.ex, y = e / l.ex % l.ey, z = e / ((long)l.ex * l.ey);
    double v = 0, g[3] = {0, 0, 0};
    if (p->sinside[0][x] && p->sinside[1][y] && p->sinside[2][z]) {
      int I[3] = {p->sidx[0][x], p->sidx[1][y], p->sidx[2][z]};
      const double* N0 = &p->sN[0][(size_t)x * o];
      const double* N1 = &p->sN[1][(size_t)y * o];
      const double* N2 = &p->sN[2][(size_t)z * o];
      const double* D0 = &p->sdN[0][(size_t)x * o];
      const double* D1 = &p->sdN[1][(size_t)y * o];
      const double* D2 = &p->sdN[2][(size_t)z * o];
      for (int a = 0; a < o; a++)
        for (int b = 0; b < o; b++)
          for (int q = 0; q < o; q++) {
            double cc = c[(I[0] - o + a) + (long)(I[1] - o + b) * nbx + (long)(I[2] - o + q) * nbx * nby];
            v += cc * N0[a] * N1[b] * N2[q];
            g[0] += cc * D0[a] * N1[b] * N2[q];
            g[1] += cc * N0[a] * D1[b] * N2[q];
            g[2] += cc * N0[a] * N1[b] * D2[q];
          }
    }
    fv[k] = v;
    for (int a = 0; a < 3; a++) gr[3 * k + a] = g[a];
    // 2) orientation probe (correct_spline_background_ele_normal_direction)
    double pt[3] = {x + 0.5 + 0.01 * g[0], y + 0.5 + 0.01 * g[1], z + 0.5 + 0.01 * g[2]};
    bool ins;
    double vd = spline_value_at(p, c, pt, &ins);
    if (!ins) vd = -0.1;
    double vv = (p->sinside[0][x] && p->sinside[1][y] && p->sinside[2][z]) ? v : -0.1;
    double s = Hs(vv, beta) - Hs(vd, beta);
    dir[k] = s > 0 ? 1 : -1;
  }
  double count = 0;
  for (long k = 0; k < n; k++) count += dir[k];
  if (direction_sum) *direction_sum = count;
  if (count < 0)
    for (long k = 0; k < 3 * n; k++) gr[k] = -gr[k];
  double direction = count > 0 ? 1.0 : -1.0;
  // 3) per-element constraint and count
  double sum = 0, cnt = 0;
  for (long k = 0; k < n; k++) {
    double* nv = &gr[3 * k];
    double nn = std::sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
    double inner = nv[2] / nn / cosang;
    double val = 0;
    bool down = nv[2] < 0;
    if (down) cnt += 1;
    switch (mode) {
      case 0: if (down) val = std::pow(inner, fpara); break;
      case 1: val = std::pow(inner, fpara); break;
      case 2: if (down) val = hfun(inner, fpara); break;
      case 3: val = hfun(inner, fpara); break;
      case 4: if (down) val = ndist(fv[k], na) * overhang(inner, mid, fpara) * inner_(inner, ia); break;
      case 5: val = ndist(fv[k], na) * overhang(inner, mid, fpara) * inner_(inner, ia); break;
    }
    if (per_element) per_element[elist[k]] = val;
    sum += val;
  }
  double count2 = (mode % 2 == 0) ? cnt : (double)n;
  if (count_out) *count_out = count2;
  double value = 0;
  if (count2 != 0) {
    if (mode <= 1) value = std::pow(sum / count2, 1 / fpara) - 1;
    else value = sum / count2;
  }
  // 4) gradient w.r.t. coefficients (compute_spline_bg_selfsupp_constraint_dcoeff)
  if (dc) {
    for (long i = 0; i < ncoef; i++) dc[i] = 0;
    for (long k = 0; k < n; k++) {
      long e = elist[k];
      int x = e % l.ex, y = e / l.ex % l.ey, z = e / ((long)l.ex * l.ey);
      if (!(p->sinside[0][x] && p->sinside[1][y] && p->sinside[2][z])) continue;
      double* nv = &gr[3 * k];
      double nn = std::sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
      double inner = nv[2] / nn / cosang;
      bool down = nv[2] < 0;
      int I[3] = {p->sidx[0][x], p->sidx[1][y], p->sidx[2][z]};
      const double* N0 = &p->sN[0][(size_t)x * o];
      const double* N1 = &p->sN[1][(size_t)y * o];
      const double* N2 = &p->sN[2][(size_t)z * o];
      const double* D0 = &p->sdN[0][(size_t)x * o];
      const double* D1 = &p->sdN[1][(size_t)y * o];
      const double* D2 = &p->sdN[2][(size_t)z * o];
      double fvk = fv[k];
      for (int a = 0; a < o; a++)
        for (int b = 0; b < o; b++)
          for (int q = 0; q < o; q++) {
            double dfv = N0[a] * N1[b] * N2[q];
            double nd[3] = {direction * D0[a] * N1[b] * N2[q], direction * N0[a] * D1[b] * N2[q],
                            direction * N0[a] * N1[b] * D2[q]};
            double normdc = (nv[0] * nd[0] + nv[1] * nd[1] + nv[2] * nd[2]) / nn;
            double up = nd[2] * nn - nv[2] * normdc;
            double down_ = nn * nn * cosang;
            double dinner = up / down_;
            double val = 0;
            switch (mode) {
              case 0: if (down) val = fpara * std::pow(inner, fpara - 1) * dinner; break;
              case 1: val = fpara * std::pow(inner, fpara - 1) * dinner; break;
              case 2: if (down) val = dhfun(inner, fpara) * dinner; break;
              case 3: val = dhfun(inner, fpara) * dinner; break;
              case 4:
              case 5:
                if (mode == 5 || down)
                  val = dndist(fvk, na) * dfv * overhang(inner, mid, fpara) * inner_(inner, ia) +
                        ndist(fvk, na) * doverhang(inner, mid, fpara) * dinner * inner_(inner, ia) +
                        ndist(fvk, na) * overhang(inner, mid, fpara) * dinner * dinner_(inner, ia);
                break;
            }
            dc[(I[0] - o + a) + (long)(I[1] - o + b) * nbx + (long)(I[2] - o + q) * nbx * nby] += val;
          }
    }
    double scale = count2 == 0 ? 0.0 : 1.0 / count2;
    for (long i = 0; i < ncoef; i++) dc[i] *= scale;
  }
  return value;
}
