// FP64 CPU oracle: admissible-load projection, worst-case eigenproblem
// (dense aggregated, Lanczos, modified power method).
// TEST INFRASTRUCTURE ONLY (see oracle.h).
#include "or_internal.h"
#include <cstdio>

using namespace orc;

// deterministic uniform [-1,1) stream shared with the CUDA path
static inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
static inline double urand(uint64_t seed, uint64_t i) {
  uint64_t h = splitmix64(seed * 0x100000001B3ull ^ splitmix64(i));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}

// ---------------------------------------------------------------- rigid motions
int orc::rigid_basis(const std::vector<double>& pos, const double* nrm, std::vector<double>& Q, bool drop) {
  const size_t m = pos.size();  // 3 per node
  std::vector<std::vector<double>> col(6, std::vector<double>(m, 0.0));
  for (size_t k = 0; k < m / 3; k++) {
    const double* p = &pos[3 * k];
    // rows c of [I | p^], p^ = [[0, -z, y], [z, 0, -x], [-y, x, 0]]
    const double ph[3][3] = {{0, -p[2], p[1]}, {p[2], 0, -p[0]}, {-p[1], p[0], 0}};
    for (int c = 0; c < 3; c++) {
      col[c][3 * k + c] = 1.0;
      for (int j = 0; j < 3; j++) col[3 + j][3 * k + c] = ph[c][j];
    }
    if (nrm) {
      const double* nv = &nrm[3 * k];
      for (int j = 0; j < 6; j++) {
        double* b = &col[j][3 * k];
        const double s = b[0] * nv[0] + b[1] * nv[1] + b[2] * nv[2];
        for (int c = 0; c < 3; c++) b[c] = s * nv[c];
      }
    }
  }
  auto dotv = [&](const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0;
    for (size_t i = 0; i < m; i++) s += a[i] * b[i];
    return s;
  };
  bool invalid[6] = {false, false, false, false, false, false};
  for (int i = 0; i < 6; i++) {
    const double oldres = std::sqrt(dotv(col[i], col[i]));
    for (int j = 0; j < i; j++) {
      if (drop && invalid[j]) continue;
      const double w = dotv(col[i], col[j]);
      for (size_t t = 0; t < m; t++) col[i][t] -= w * col[j][t];
    }
    const double res = std::sqrt(dotv(col[i], col[i]));
    if (drop && (res / oldres < 1e-6 || oldres < 1e-6)) invalid[i] = true;
    for (size_t t = 0; t < m; t++) col[i][t] /= res;
  }
  Q.clear();
  int k = 0;
  for (int i = 0; i < 6; i++) {
    if (drop && invalid[i]) continue;
    Q.insert(Q.end(), col[i].begin(), col[i].end());
    k++;
  }
  return k;
}

// setNodes / setLoadNodes (projection.cpp:47-110, :129-269) for problems
// without supports: the rigid motions of all active fine nodes (for
// displacementProject), of the load nodes (for forceProject; normal-projected
// in constrained-direction modes) and of the coarsest nodes (pseudo-inverse)
void orc::rigid_setup(or_problem* p) {
  const Level& f = p->L[0];
  std::vector<double> pos;
  std::vector<long> act;
  for (long n = 0; n < f.nn; n++) {
    if (!f.vmask[n]) continue;
    act.push_back(n);
    pos.push_back((double)(n % f.nx));
    pos.push_back((double)(n / f.nx % f.ny));
    pos.push_back((double)(n / ((long)f.nx * f.ny)));
  }
  std::vector<double> Q;
  const int k = rigid_basis(pos, nullptr, Q, false);
  const size_t m = pos.size();
  p->rigid_full.assign((size_t)3 * f.nn * 6, 0.0);
  for (int j = 0; j < k; j++)
    for (size_t a = 0; a < act.size(); a++)
      for (int c = 0; c < 3; c++) p->rigid_full[(size_t)j * 3 * f.nn + c * f.nn + act[a]] = Q[j * m + 3 * a + c];
  std::vector<double> lpos, lnrm;
  for (int n : p->load_nodes) {
    lpos.push_back((double)(n % f.nx));
    lpos.push_back((double)(n / f.nx % f.ny));
    lpos.push_back((double)(n / ((long)f.nx * f.ny)));
    for (int c = 0; c < 3; c++) lnrm.push_back(p->normals[3 * (size_t)n + c]);
  }
  p->rigid_k[0] = rigid_basis(lpos, nullptr, p->rigid_load[0], true);
  p->rigid_k[1] = rigid_basis(lpos, lnrm.data(), p->rigid_load[1], true);
}

// displacementProject (projection.cpp:374-411): u -= R R^T u over the
// orthonormal rigid motions of the active fine nodes
void orc::displacement_project(const or_problem* p, double* u) {
  if (p->has_support) return;
  const long n3 = 3 * p->L[0].nn;
  for (int j = 0; j < 6; j++) {
    const double* r = &p->rigid_full[(size_t)j * n3];
    double s = 0;
    for (long i = 0; i < n3; i++) s += r[i] * u[i];
    for (long i = 0; i < n3; i++) u[i] -= s * r[i];
  }
}

extern "C" void or_displacement_project(const or_problem* p, double* u) { displacement_project(p, u); }

// forceProject (projection.cpp:289-360 / projection.cu:165-231): forces kept
// only on load nodes; in constrained-direction modes only the component
// along the load normal survives (f -= Nd^T Nd f); without supports the
// rigid motions of the load set are removed as well (f -= Rd Rd^T f).
extern "C" void or_force_project(const or_problem* p, double* f, int cf) {
  const long nn = p->L[0].nn;
  std::vector<double> keep(3 * p->load_nodes.size());
  for (size_t k = 0; k < p->load_nodes.size(); k++) {
    long n = p->load_nodes[k];
    double v[3] = {f[n], f[nn + n], f[2 * nn + n]};
    if (cf) {
      const double* nr = &p->normals[3 * n];
      double s = v[0] * nr[0] + v[1] * nr[1] + v[2] * nr[2];
      for (int c = 0; c < 3; c++) v[c] = s * nr[c];
    }
    for (int c = 0; c < 3; c++) keep[3 * k + c] = v[c];
  }
  if (!p->has_support) {
    const int ci = cf ? 1 : 0;
    const size_t m = keep.size();
    const std::vector<double>& Q = p->rigid_load[ci];
    std::vector<double> w(p->rigid_k[ci], 0.0);
    for (int j = 0; j < p->rigid_k[ci]; j++)
      for (size_t i = 0; i < m; i++) w[j] += Q[j * m + i] * keep[i];
    for (int j = 0; j < p->rigid_k[ci]; j++)
      for (size_t i = 0; i < m; i++) keep[i] -= w[j] * Q[j * m + i];
  }
  for (long i = 0; i < 3 * nn; i++) f[i] = 0;
  for (size_t k = 0; k < p->load_nodes.size(); k++) {
    long n = p->load_nodes[k];
    for (int c = 0; c < 3; c++) f[c * nn + n] = keep[3 * k + c];
  }
}

// cyclic Jacobi eigen-decomposition of a symmetric n x n matrix (row-major);
// eigenvalues in w, eigenvectors in columns of V.
static void jacobi_eig(int n, std::vector<double> A, std::vector<double>& w, std::vector<double>& V) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) V[(size_t)i * n + i] = 1;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0;
    for (int i = 0; i < n; i++)
      for (int j = i + 1; j < n; j++) off += A[(size_t)i * n + j] * A[(size_t)i * n + j];
    if (off < 1e-30) break;
    for (int pi = 0; pi < n; pi++)
      for (int q = pi + 1; q < n; q++) {
        double apq = A[(size_t)pi * n + q];
        if (std::fabs(apq) < 1e-300) continue;
        double app = A[(size_t)pi * n + pi], aqq = A[(size_t)q * n + q];
        double theta = (aqq - app) / (2 * apq);
        double t = (theta >= 0 ? 1 : -1) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
        double c = 1 / std::sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < n; k++) {
          double akp = A[(size_t)k * n + pi], akq = A[(size_t)k * n + q];
          A[(size_t)k * n + pi] = c * akp - s * akq;
          A[(size_t)k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; k++) {
          double apk = A[(size_t)pi * n + k], aqk = A[(size_t)q * n + k];
          A[(size_t)pi * n + k] = c * apk - s * aqk;
          A[(size_t)q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; k++) {
          double vkp = V[(size_t)k * n + pi], vkq = V[(size_t)k * n + q];
          V[(size_t)k * n + pi] = c * vkp - s * vkq;
          V[(size_t)k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  w.resize(n);
  for (int i = 0; i < n; i++) w[i] = A[(size_t)i * n + i];
}

static int solve_tight(or_problem* p, double* u, const double* f, double tol) {
  double rr;
  std::fill(u, u + 3 * p->L[0].nn, 0.0);
  return or_solve(p, u, f, tol, 500, 1, 1, 1, 0, 1.0, &rr);  // projected when support-free
}

// dense aggregated worst case (TestSuit::verifyModifiedPM / aggregatedSystem,
// utils/test_utils.cpp:2598-2645, 2859-2928)
extern "C" double or_dense_worst(or_problem* p, int cf, double tol, double* f_worst, double* u_worst) {
  const long nn = p->L[0].nn;
  int nl = (int)p->load_nodes.size();
  int per = cf ? 1 : 3;
  int m = nl * per;
  std::vector<std::vector<double>> U(m, std::vector<double>(3 * nn));
  std::vector<double> b(3 * nn), C((size_t)m * m);
  auto basis = [&](int col, double* v) {
    std::fill(v, v + 3 * nn, 0.0);
    int k = col / per;
    long n = p->load_nodes[k];
    if (cf) for (int c = 0; c < 3; c++) v[c * nn + n] = p->normals[3 * n + c];
    else v[(col % 3) * nn + n] = 1.0;
  };
  // basis vectors of the admissible loads (forceProject also removes the
  // rigid motions of support-free problems; a no-op on the basis otherwise)
  for (int col = 0; col < m; col++) {
    basis(col, b.data());
    or_force_project(p, b.data(), cf);
    solve_tight(p, U[col].data(), b.data(), tol);
  }
  for (int i = 0; i < m; i++) {
    basis(i, b.data());
    or_force_project(p, b.data(), cf);
    for (int j = 0; j < m; j++) C[(size_t)i * m + j] = dot3(b.data(), U[j].data(), nn);
  }
  for (int i = 0; i < m; i++)
    for (int j = i + 1; j < m; j++) {
      double v = 0.5 * (C[(size_t)i * m + j] + C[(size_t)j * m + i]);
      C[(size_t)i * m + j] = C[(size_t)j * m + i] = v;
    }
  std::vector<double> w, V;
  jacobi_eig(m, C, w, V);
  int best = 0;
  for (int i = 1; i < m; i++) if (w[i] > w[best]) best = i;
  if (f_worst) std::fill(f_worst, f_worst + 3 * nn, 0.0);
  if (u_worst) std::fill(u_worst, u_worst + 3 * nn, 0.0);
  for (int col = 0; col < m; col++) {
    double y = V[(size_t)col * m + best];
    basis(col, b.data());
    or_force_project(p, b.data(), cf);
    for (long i = 0; i < 3 * nn; i++) {
      if (f_worst) f_worst[i] += y * b[i];
      if (u_worst) u_worst[i] += y * U[col][i];
    }
  }
  return w[best];
}

// Lanczos on P K^-1 P with full reorthogonalisation (build feature; the
// reference iterates a modified power method instead).
extern "C" double or_lanczos(or_problem* p, int steps, int cf, double tol, uint64_t seed, double* f_worst,
                             double* u_worst, double* ritz) {
  const long nn = p->L[0].nn;
  int nl = (int)p->load_nodes.size();
  std::vector<std::vector<double>> Vb, Ub;
  std::vector<double> v(3 * nn, 0.0), w(3 * nn), u(3 * nn);
  for (int k = 0; k < nl; k++) {
    long n = p->load_nodes[k];
    for (int c = 0; c < 3; c++) v[c * nn + n] = urand(seed, 3ull * k + c);
  }
  or_force_project(p, v.data(), cf);
  double nv = std::sqrt(dot3(v.data(), v.data(), nn));
  for (auto& x : v) x /= nv;
  std::vector<double> alpha, beta;
  for (int it = 0; it < steps; it++) {
    Vb.push_back(v);
    solve_tight(p, u.data(), v.data(), tol);
    Ub.push_back(u);
    w = u;
    or_force_project(p, w.data(), cf);
    double a = dot3(v.data(), w.data(), nn);
    alpha.push_back(a);
    for (int pass = 0; pass < 2; pass++)
      for (auto& vj : Vb) {
        double s = dot3(vj.data(), w.data(), nn);
        for (long i = 0; i < 3 * nn; i++) w[i] -= s * vj[i];
      }
    double b = std::sqrt(dot3(w.data(), w.data(), nn));
    if (it == steps - 1 || b < 1e-14 * std::fabs(a)) break;
    beta.push_back(b);
    for (long i = 0; i < 3 * nn; i++) v[i] = w[i] / b;
  }
  int m = (int)alpha.size();
  std::vector<double> T((size_t)m * m, 0.0);
  for (int i = 0; i < m; i++) {
    T[(size_t)i * m + i] = alpha[i];
    if (i + 1 < m) T[(size_t)i * m + i + 1] = T[(size_t)(i + 1) * m + i] = beta[i];
  }
  std::vector<double> ev, EV;
  jacobi_eig(m, T, ev, EV);
  int best = 0;
  for (int i = 1; i < m; i++) if (ev[i] > ev[best]) best = i;
  if (ritz) for (int i = 0; i < m; i++) ritz[i] = ev[i];
  if (f_worst) std::fill(f_worst, f_worst + 3 * nn, 0.0);
  if (u_worst) std::fill(u_worst, u_worst + 3 * nn, 0.0);
  for (int k = 0; k < m; k++) {
    double y = EV[(size_t)k * m + best];
    for (long i = 0; i < 3 * nn; i++) {
      if (f_worst) f_worst[i] += y * Vb[k][i];
      if (u_worst) u_worst[i] += y * Ub[k][i];
    }
  }
  return ev[best];
}

// modifiedPM (optimization.cpp:215-353): random admissible unit force, one
// V-cycle(1,1) per step warm-started from the previous displacement,
// f <- P u / |P u|, until the load-node force change <= 1e-4 and r_rel <= 1e-2.
extern "C" double or_modified_pm(or_problem* p, int cf, uint64_t seed, int max_itn, double* f_out, double* u_out,
                                 int* itn_out) {
  const long nn = p->L[0].nn;
  int nl = (int)p->load_nodes.size();
  std::vector<double> f(3 * nn, 0.0), u(3 * nn, 0.0), fs_old(3 * nl), fs(3 * nl);
  for (int k = 0; k < nl; k++) {
    long n = p->load_nodes[k];
    for (int c = 0; c < 3; c++) f[c * nn + n] = urand(seed, 3ull * k + c);
  }
  or_force_project(p, f.data(), cf);
  double fn = std::sqrt(dot3(f.data(), f.data(), nn));
  for (auto& x : f) x /= fn;
  auto gather = [&](std::vector<double>& dst) {
    for (int k = 0; k < nl; k++)
      for (int c = 0; c < 3; c++) dst[3 * k + c] = f[c * nn + p->load_nodes[k]];
  };
  gather(fs_old);
  double fch = 1, rr = 1;
  int itn = 0;
  while (itn++ < max_itn && (fch > 1e-4 || rr > 1e-2)) {
    rr = or_vcycle(p, u.data(), f.data(), 1, 1, 0, 1.0, 0);
    displacement_project(p, u.data());
    f = u;
    or_force_project(p, f.data(), cf);
    fn = std::sqrt(dot3(f.data(), f.data(), nn));
    for (auto& x : f) x /= fn;
    gather(fs);
    double d = 0, s = 0;
    for (int i = 0; i < 3 * nl; i++) { d += (fs[i] - fs_old[i]) * (fs[i] - fs_old[i]); s += fs_old[i] * fs_old[i]; }
    fch = std::sqrt(d) / std::sqrt(s);
    fs_old = fs;
  }
  if (itn_out) *itn_out = itn;
  if (f_out) std::copy(f.begin(), f.end(), f_out);
  if (u_out) std::copy(u.begin(), u.end(), u_out);
  return dot3(f.data(), u.data(), nn);
}
