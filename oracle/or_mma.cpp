// FP64 CPU oracle: the reference's MMA (optimization/mma_t.h, mma_t.cpp,
// mma_t.cu) restated in double precision.  TEST INFRASTRUCTURE ONLY.
#include "or_internal.h"

typedef std::vector<double> vec;

struct or_mma {
  int n, m;
  vec x, xmin, xmax, L, U, alpha, beta, lastdx;
  vec xi, eta, y, lambda, mu, s, a, c, d;
  double z = 1, zeta = 1, a0 = 1, eps = 1;
  int stop_counter = 0;
  std::vector<vec> p, q;
  vec b, plambda, qlambda;
};

// clamp_asymptotes (mma_t.cu:747-761)
static void clamp_asym(or_mma* s) {
  for (int i = 0; i < s->n; i++) {
    double st = s->xmax[i] - s->xmin[i], x = s->x[i];
    s->L[i] = std::min(std::max(s->L[i], x - 10 * st), x - 0.01 * st);
    s->U[i] = std::min(std::max(s->U[i], x + 0.01 * st), x + 10 * st);
    s->alpha[i] = std::max(s->xmin[i], std::max(s->L[i] + 0.1 * (x - s->L[i]), x - 0.5 * st));
    s->beta[i] = std::min(s->xmax[i], std::min(s->U[i] - 0.1 * (s->U[i] - x), x + 0.5 * st));
  }
}

extern "C" or_mma* or_mma_create(int n, int m, const double* xmin, const double* xmax) {
  or_mma* s = new or_mma();
  s->n = n; s->m = m;
  s->xmin.assign(xmin, xmin + n); s->xmax.assign(xmax, xmax + n);
  // set_bound (mma_t.cu:809-819)
  s->alpha = s->xmin; s->beta = s->xmax; s->L = s->alpha; s->U = s->beta;
  s->x.resize(n);
  for (int i = 0; i < n; i++) s->x[i] = (s->alpha[i] + s->beta[i]) / 2;
  clamp_asym(s);
  s->lastdx.assign(n, 0.0);
  s->y.assign(m, 1.0); s->lambda.assign(m, 1.0); s->s.assign(m, 1.0); s->mu.assign(m, 0.0);
  s->a.assign(m, 0.0); s->c.assign(m, 10.0); s->d.assign(m, 1.0);
  // init_subproblem_variable (mma_t.cu:797-807)
  s->xi.resize(n); s->eta.resize(n);
  for (int i = 0; i < n; i++) {
    s->x[i] = (s->alpha[i] + s->beta[i]) / 2;
    s->xi[i] = std::max(1 / (s->x[i] - s->alpha[i]), 1.0);
    s->eta[i] = std::max(1 / (s->beta[i] - s->x[i]), 1.0);
  }
  for (int j = 0; j < m; j++) s->mu[j] = std::max(s->c[j] / 2, 1.0);
  return s;
}

// build extension: start from a given design instead of the box midpoint
extern "C" void or_mma_set_x(or_mma* s, const double* x) {
  for (int i = 0; i < s->n; i++) s->x[i] = x[i];
  clamp_asym(s);
}

extern "C" void or_mma_get(or_mma* s, double* x, double* L, double* U, double* al, double* be) {
  for (int i = 0; i < s->n; i++) {
    if (x) x[i] = s->x[i];
    if (L) L[i] = s->L[i];
    if (U) U[i] = s->U[i];
    if (al) al[i] = s->alpha[i];
    if (be) be[i] = s->beta[i];
  }
}

extern "C" void or_mma_destroy(or_mma* s) { delete s; }

static void update_pql(or_mma* s, const vec& lam) {
  s->plambda = s->p[0];
  s->qlambda = s->q[0];
  for (int j = 0; j < s->m; j++)
    for (int i = 0; i < s->n; i++) {
      s->plambda[i] += lam[j] * s->p[j + 1][i];
      s->qlambda[i] += lam[j] * s->q[j + 1][i];
    }
}

struct W {
  vec x, y, lambda, xi, eta, mu, s;
  double z, zeta;
};

// kkt_err (mma_t.cu:574-678): returns (2-norm, inf-norm)
static std::pair<double, double> kkt(or_mma* S, const W& w, double damp) {
  update_pql(S, w.lambda);
  double sum = 0, mx = -10;
  auto acc = [&](double v) { sum += v * v; mx = std::max(mx, std::fabs(v)); };
  int n = S->n, m = S->m;
  for (int i = 0; i < n; i++) {
    double ux = S->U[i] - w.x[i], xl = w.x[i] - S->L[i];
    acc(S->plambda[i] / (ux * ux) - S->qlambda[i] / (xl * xl) - w.xi[i] + w.eta[i]);
  }
  for (int j = 0; j < m; j++) acc(S->c[j] + S->d[j] * w.y[j] - w.lambda[j] - w.mu[j]);
  double la = 0;
  for (int j = 0; j < m; j++) la += w.lambda[j] * S->a[j];
  acc(S->a0 - w.zeta - la);
  for (int j = 0; j < m; j++) {
    double g = 0;
    for (int i = 0; i < n; i++) g += S->p[j + 1][i] / (S->U[i] - w.x[i]) + S->q[j + 1][i] / (w.x[i] - S->L[i]);
    double r = (g - S->a[j] * w.z - w.y[j] + w.s[j] - S->b[j]) / damp;
    acc(r);
  }
  for (int i = 0; i < n; i++) acc(w.xi[i] * (w.x[i] - S->alpha[i]) - S->eps);
  for (int i = 0; i < n; i++) acc(w.eta[i] * (S->beta[i] - w.x[i]) - S->eps);
  for (int j = 0; j < m; j++) acc(w.mu[j] * w.y[j] - S->eps);
  acc(w.zeta * w.z - S->eps);
  for (int j = 0; j < m; j++) acc(w.lambda[j] * w.s[j] - S->eps);
  return {std::sqrt(sum), mx};
}

// dense (m+1)^2 solve with partial pivoting (stand-in for Eigen colPivHouseholderQr)
static void dense_solve(int N, std::vector<double> A, std::vector<double> b, std::vector<double>& x) {
  for (int k = 0; k < N; k++) {
    int piv = k;
    for (int i = k + 1; i < N; i++) if (std::fabs(A[i * N + k]) > std::fabs(A[piv * N + k])) piv = i;
    if (piv != k) { for (int j = 0; j < N; j++) std::swap(A[k * N + j], A[piv * N + j]); std::swap(b[k], b[piv]); }
    for (int i = k + 1; i < N; i++) {
      double f = A[i * N + k] / A[k * N + k];
      for (int j = k; j < N; j++) A[i * N + j] -= f * A[k * N + j];
      b[i] -= f * b[k];
    }
  }
  x.assign(N, 0.0);
  for (int i = N - 1; i >= 0; i--) {
    double t = b[i];
    for (int j = i + 1; j < N; j++) t -= A[i * N + j] * x[j];
    x[i] = t / A[i * N + i];
  }
}

// mma_t::update (mma_t.cpp:18-51) -> subproblem.solve (mma_t.cu:330-499)
extern "C" int or_mma_update(or_mma* S, const double* df, const double* dg, const double* g, double* info) {
  const int n = S->n, m = S->m;
  vec curx = S->x;
  // init (mma_t.cu:69-106)
  S->p.assign(m + 1, vec(n));
  S->q.assign(m + 1, vec(n));
  for (int j = 0; j <= m; j++) {
    const double* d = (j == 0) ? df : dg + (size_t)(j - 1) * n;
    for (int i = 0; i < n; i++) {
      double ux = S->U[i] - S->x[i], xl = S->x[i] - S->L[i];
      double pos = std::max(d[i], 0.0), neg = std::max(-d[i], 0.0);
      double raa = 1e-5 / (S->xmax[i] - S->xmin[i]);
      S->p[j][i] = ux * ux * (1.001 * pos + 0.001 * neg + raa);
      S->q[j][i] = xl * xl * (0.001 * pos + 1.001 * neg + raa);
    }
  }
  S->b.assign(m, 0.0);
  for (int j = 0; j < m; j++) {
    double gp = 0;
    for (int i = 0; i < n; i++) gp += S->p[j + 1][i] / (S->U[i] - S->x[i]) + S->q[j + 1][i] / (S->x[i] - S->L[i]);
    S->b[j] = gp - g[j];
  }
  // reset (mma_t.cu:702-713)
  for (int i = 0; i < n; i++) S->x[i] = (S->alpha[i] + S->beta[i]) / 2;
  S->eps = 1; S->zeta = S->z = 1;
  for (int j = 0; j < m; j++) { S->y[j] = 1; S->lambda[j] = 1; S->s[j] = 1; S->mu[j] = std::max(S->c[j] / 2, 1.0); }
  for (int i = 0; i < n; i++) {
    S->xi[i] = std::max(1 / (S->x[i] - S->alpha[i]), 1.0);
    S->eta[i] = std::max(1 / (S->beta[i] - S->x[i]), 1.0);
  }
  update_pql(S, S->lambda);

  double err = 1e30, lasterr = 0;
  int nsub = 0;
  bool overflow = false;
  double step_used = 0;
  while (S->eps > 1e-6) {
    err = 1e30;
    double damp = 1;
    int stays = 0;
    while (err > 0.9 * S->eps) {
      vec Dx(n), hdx(n), G((size_t)m * n), Dy(m), Dl(m), hdy(m), hdl(m);
      for (int i = 0; i < n; i++) {
        double ux = S->U[i] - S->x[i], xl = S->x[i] - S->L[i];
        double psi = 2 * S->plambda[i] / (ux * ux * ux) + 2 * S->qlambda[i] / (xl * xl * xl);
        Dx[i] = psi + S->xi[i] / (S->x[i] - S->alpha[i]) + S->eta[i] / (S->beta[i] - S->x[i]);
        double varphi = S->plambda[i] / (ux * ux) - S->qlambda[i] / (xl * xl);
        hdx[i] = -(S->eps / (S->x[i] - S->alpha[i]) - S->eps / (S->beta[i] - S->x[i]) - varphi);
        for (int j = 0; j < m; j++) G[(size_t)j * n + i] = S->p[j + 1][i] / (ux * ux) - S->q[j + 1][i] / (xl * xl);
      }
      double la = 0;
      for (int j = 0; j < m; j++) {
        Dy[j] = S->d[j] + S->mu[j] / S->y[j];
        Dl[j] = S->s[j] / S->lambda[j];
        hdy[j] = -(S->lambda[j] + S->eps / S->y[j] - S->c[j] - S->d[j] * S->y[j]);
        double gp = 0;
        for (int i = 0; i < n; i++) gp += S->p[j + 1][i] / (S->U[i] - S->x[i]) + S->q[j + 1][i] / (S->x[i] - S->L[i]);
        hdl[j] = -(S->z * S->a[j] + S->y[j] + S->b[j] - S->eps / S->lambda[j] - gp);
        la += S->lambda[j] * S->a[j];
      }
      double hdz = -(la + S->eps / S->z - S->a0);
      // solveLinearSystem (mma_t.cu:228-328)
      int N = m + 1;
      std::vector<double> A((size_t)N * N, 0.0), rhs(N, 0.0), sol;
      for (int j = 0; j < m; j++) {
        A[j * N + j] += Dl[j] + 1 / Dy[j];
        for (int k = 0; k < m; k++) {
          double s = 0;
          for (int i = 0; i < n; i++) s += G[(size_t)j * n + i] * (G[(size_t)k * n + i] / Dx[i]);
          A[j * N + k] += s;
        }
        double s = 0;
        for (int i = 0; i < n; i++) s += G[(size_t)j * n + i] * (hdx[i] / Dx[i]);
        rhs[j] = hdl[j] + hdy[j] / Dy[j] - s;
        A[j * N + m] = S->a[j];
        A[m * N + j] = S->a[j];
      }
      A[m * N + m] = -S->zeta / S->z;
      rhs[m] = hdz;
      dense_solve(N, A, rhs, sol);
      vec dx(n), dy(m), dl(m);
      double dz = sol[m];
      for (int i = 0; i < n; i++) {
        double t = -hdx[i] / Dx[i];
        for (int j = 0; j < m; j++) t -= sol[j] * G[(size_t)j * n + i] / Dx[i];
        dx[i] = t;
      }
      for (int j = 0; j < m; j++) { dl[j] = sol[j]; dy[j] = dl[j] / Dy[j] - hdy[j] / Dy[j]; }
      vec dxi(n), deta(n), dmu(m), ds(m);
      for (int i = 0; i < n; i++) {
        dxi[i] = S->eps / (S->x[i] - S->alpha[i]) - dx[i] / (S->x[i] - S->alpha[i]) * S->xi[i] - S->xi[i];
        deta[i] = S->eps / (S->beta[i] - S->x[i]) + S->eta[i] / (S->beta[i] - S->x[i]) * dx[i] - S->eta[i];
      }
      for (int j = 0; j < m; j++) {
        dmu[j] = S->eps / S->y[j] - dy[j] * S->mu[j] / S->y[j] - S->mu[j];
        ds[j] = S->eps / S->lambda[j] - S->s[j] / S->lambda[j] * dl[j] - S->s[j];
      }
      double dzeta = S->eps / S->z - S->zeta - (S->zeta / S->z) * dz;
      // step bound (mma_t.cu:412-415), clamp factor 0.99
      const double cf = 0.99;
      double t1 = -1e300, t2 = -1e300, t3 = -1e300;
      for (int i = 0; i < n; i++) {
        t1 = std::max(t1, (-1 / cf) * (dx[i] / (S->x[i] - S->alpha[i])));
        t2 = std::max(t2, (1 / cf) * (dx[i] / (S->beta[i] - S->x[i])));
      }
      auto art = [&](double dv, double v) { t3 = std::max(t3, (-1 / cf) * dv / v); };
      for (int j = 0; j < m; j++) art(dy[j], S->y[j]);
      art(dz, S->z);
      for (int j = 0; j < m; j++) art(dl[j], S->lambda[j]);
      for (int i = 0; i < n; i++) art(dxi[i], S->xi[i]);
      for (int i = 0; i < n; i++) art(deta[i], S->eta[i]);
      for (int j = 0; j < m; j++) art(dmu[j], S->mu[j]);
      art(dzeta, S->zeta);
      for (int j = 0; j < m; j++) art(ds[j], S->s[j]);
      double max_t = 1 / std::max(std::max(t1, t2), std::max(t3, 1.0));
      // search_step (mma_t.cu:501-571)
      W cur{S->x, S->y, S->lambda, S->xi, S->eta, S->mu, S->s, S->z, S->zeta};
      double old_err = kkt(S, cur, 1).first;
      double step = max_t, new_err = 1e30, new_inf = 1e30;
      while (step > 1e-12 && new_err > old_err) {
        W nw = cur;
        for (int i = 0; i < n; i++) {
          nw.x[i] += dx[i] * step; nw.xi[i] += dxi[i] * step; nw.eta[i] += deta[i] * step;
        }
        for (int j = 0; j < m; j++) {
          nw.y[j] += dy[j] * step; nw.lambda[j] += dl[j] * step; nw.mu[j] += dmu[j] * step; nw.s[j] += ds[j] * step;
        }
        nw.z += dz * step; nw.zeta += dzeta * step;
        auto e2 = kkt(S, nw, damp);
        new_err = e2.first; new_inf = e2.second;
        if (new_err < old_err) {
          S->x = nw.x; S->y = nw.y; S->z = nw.z; S->lambda = nw.lambda; S->xi = nw.xi; S->eta = nw.eta;
          S->mu = nw.mu; S->zeta = nw.zeta; S->s = nw.s;
          break;
        }
        step /= 2;
      }
      step_used = step;
      err = new_inf;
      if ((err - lasterr) / err < 1e-5) stays++;
      else stays = 0;
      lasterr = err;
      if (stays > 6) { damp *= 10; stays = 0; }
      if (nsub++ > 80) { overflow = true; break; }
    }
    if (overflow) break;
    S->eps *= 0.1;
  }
  // adjust_asym (mma_t.cu:164-226) with this step and the previous one
  vec cur_dx(n);
  for (int i = 0; i < n; i++) cur_dx[i] = S->x[i] - curx[i];
  for (int i = 0; i < n; i++) {
    double gamma = 1, d1 = cur_dx[i], d2 = S->lastdx[i];
    if (d1 * d2 > 0) gamma = 1.2;
    if (d1 * d2 < 0) gamma = 0.7;
    double xv = S->x[i], st = S->xmax[i] - S->xmin[i];
    double nl = xv - gamma * (xv - d1 - S->L[i]);
    double nu = xv + gamma * (S->U[i] - xv + d1);
    nl = std::min(std::max(nl, xv - 10 * st), xv - 0.01 * st);
    nu = std::min(std::max(nu, xv + 0.01 * st), xv + 10 * st);
    S->L[i] = nl; S->U[i] = nu;
    double na = S->xmin[i];
    na = std::max(na, nl + 0.1 * (xv - nl));
    na = std::max(na, xv - 0.5 * st);
    double nb = S->xmax[i];
    nb = std::min(nb, nu - 0.1 * (nu - xv));
    nb = std::min(nb, xv + 0.5 * st);
    S->alpha[i] = na; S->beta[i] = nb;
  }
  S->lastdx = cur_dx;
  double nrm = 0;
  for (int i = 0; i < n; i++) nrm += cur_dx[i] * cur_dx[i];
  if (std::sqrt(nrm) < 1e-3) S->stop_counter++;
  if (info) { info[0] = err; info[1] = step_used; info[2] = nsub; info[3] = overflow; }
  return S->stop_counter > 10 ? 1 : 0;
}
