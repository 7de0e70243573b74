// CPU FP64 oracle for the thermal property update (table cubic splines).
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA property kernels; the
// product never links or calls it.  Restates (paths relative to the
// CHAPSim1WW project root):
//   CUBIC_SPLINE       src/Flow_State.f90:1693-1787  (Forsythe, Malcolm &
//                      Moler, "Computer Methods for Mathematical
//                      Computations", 1977: end conditions from third
//                      divided differences)
//   NIST_SLEVAL_*      src/Flow_State.f90:1015-1070, 1420-1581 (binary
//                      search, cubic evaluation, out-of-range = error,
//                      |T - 1| < 1e-10 -> 1 for the T-based splines)
//   THERM_PROP_UPDATE  src/THERM_PROP_UPDATE.f90:129-205 (|h| < 1e-10 leaves
//                      the cell's properties unchanged; otherwise h -> T, then
//                      T -> mu, k, rho)
// and the synthetic table of the heated IO configuration: 4096 points over
// h in [-1, 1], cp = 1 + 8 exp(-(h/0.1)^2), T = int_{-1}^h dh/cp,
// rho = 1/(1+2T), mu = k = rho^-1/2.
#include <cmath>
#include <cstdint>
#include <vector>

extern "C" {

// Forsythe-Malcolm-Moler cubic spline coefficients.
void oracle_cubic_spline(int n, const double *x, const double *y, double *b, double *c, double *d) {
  if (n < 2) return;
  if (n < 3) {
    b[0] = (y[1] - y[0]) / (x[1] - x[0]);
    c[0] = d[0] = 0.0;
    b[1] = b[0];
    c[1] = d[1] = 0.0;
    return;
  }
  const int nm1 = n - 1;
  // tridiagonal system: b diagonal, d off-diagonal, c right-hand side
  d[0] = x[1] - x[0];
  c[1] = (y[1] - y[0]) / d[0];
  for (int i = 1; i < nm1; ++i) {
    d[i] = x[i + 1] - x[i];
    b[i] = 2.0 * (d[i - 1] + d[i]);
    c[i + 1] = (y[i + 1] - y[i]) / d[i];
    c[i] = c[i + 1] - c[i];
  }
  // end conditions: third derivatives from divided differences
  b[0] = -d[0];
  b[n - 1] = -d[n - 2];
  c[0] = 0.0;
  c[n - 1] = 0.0;
  if (n > 3) {
    c[0] = c[2] / (x[3] - x[1]) - c[1] / (x[2] - x[0]);
    c[n - 1] = c[n - 2] / (x[n - 1] - x[n - 3]) - c[n - 3] / (x[n - 2] - x[n - 4]);
    c[0] = c[0] * d[0] * d[0] / (x[3] - x[0]);
    c[n - 1] = -c[n - 1] * d[n - 2] * d[n - 2] / (x[n - 1] - x[n - 4]);
  }
  for (int i = 1; i < n; ++i) {  // forward elimination
    const double t = d[i - 1] / b[i - 1];
    b[i] = b[i] - t * d[i - 1];
    c[i] = c[i] - t * c[i - 1];
  }
  c[n - 1] = c[n - 1] / b[n - 1];  // back substitution
  for (int l = 1; l <= nm1; ++l) {
    const int i = n - 1 - l;
    c[i] = (c[i] - d[i] * c[i + 1]) / b[i];
  }
  // coefficients of the cubic on each interval
  b[n - 1] = (y[n - 1] - y[nm1 - 1]) / d[nm1 - 1] + d[nm1 - 1] * (c[nm1 - 1] + 2.0 * c[n - 1]);
  for (int i = 0; i < nm1; ++i) {
    b[i] = (y[i + 1] - y[i]) / d[i] - d[i] * (c[i + 1] + 2.0 * c[i]);
    d[i] = (c[i + 1] - c[i]) / d[i];
    c[i] = 3.0 * c[i];
  }
  c[n - 1] = 3.0 * c[n - 1];
  d[n - 1] = d[n - 2];
}

// Spline evaluation; returns 0, or -1 when u is outside (x[0], x[n-1])
// (the reference STOPs there).
int oracle_spline_eval(int n, const double *x, const double *y, const double *b, const double *c,
                       const double *d, double u, double *out) {
  if (u <= x[0] || u >= x[n - 1]) return -1;
  int i = 0, j = n;  // binary search for x[i] <= u < x[i+1] (0-based)
  while (j > i + 1) {
    const int k = (i + j) / 2;
    if (u < x[k]) j = k; else i = k;
  }
  const double dx = u - x[i];
  *out = y[i] + dx * (b[i] + dx * (c[i] + dx * d[i]));
  return 0;
}

// Synthetic property table (non-dimensional columns H, T, D, M, K, CP, B).
// T is integrated from the table's lower end (T(-1) = 0) by composite
// Simpson, 64 panels per table interval, accumulated interval by interval.
void oracle_synth_table(int n, double *H, double *T, double *D, double *M, double *K, double *CP, double *B) {
  auto cp = [](double h) { return 1.0 + 8.0 * std::exp(-(h / 0.1) * (h / 0.1)); };
  auto invcp = [&](double h) { return 1.0 / cp(h); };
  for (int i = 0; i < n; ++i) H[i] = -1.0 + 2.0 * (double)i / (double)(n - 1);
  T[0] = 0.0;
  for (int i = 1; i < n; ++i) {
    const int m = 64;
    const double a = H[i - 1], hh = (H[i] - H[i - 1]) / m;
    double s = invcp(a) + invcp(H[i]);
    for (int q = 1; q < m; ++q) s += invcp(a + q * hh) * (q % 2 ? 4.0 : 2.0);
    T[i] = T[i - 1] + s * hh / 3.0;
  }
  for (int i = 0; i < n; ++i) {
    D[i] = 1.0 / (1.0 + 2.0 * T[i]);
    M[i] = 1.0 / std::sqrt(D[i]);
    K[i] = M[i];
    CP[i] = cp(H[i]);
    B[i] = 2.0 / (1.0 + 2.0 * T[i]);
  }
}

// THERM_PROP_UPDATE over ncell cells.  tab = columns H, T, D, M, K of length
// n; the splines are built here (NIST_SPLINE_H/T).  Returns the number of
// cells whose h or T fell outside the table (left unchanged).
int64_t oracle_therm_prop_update(int n, const double *H, const double *Tt, const double *Dt, const double *Mt,
                                 const double *Kt, int64_t ncell, const double *h, double *T, double *rho,
                                 double *mu, double *k) {
  std::vector<double> bht(n), cht(n), dht(n);
  std::vector<double> btd(n), ctd(n), dtd(n), btm(n), ctm(n), dtm(n), btk(n), ctk(n), dtk(n);
  oracle_cubic_spline(n, H, Tt, bht.data(), cht.data(), dht.data());
  oracle_cubic_spline(n, Tt, Dt, btd.data(), ctd.data(), dtd.data());
  oracle_cubic_spline(n, Tt, Mt, btm.data(), ctm.data(), dtm.data());
  oracle_cubic_spline(n, Tt, Kt, btk.data(), ctk.data(), dtk.data());
  int64_t bad = 0;
  for (int64_t c = 0; c < ncell; ++c) {
    const double hv = h[c];
    if (std::fabs(hv) < 1.0e-10) continue;  // properties left unchanged
    double tv, mv, kv, dv;
    if (oracle_spline_eval(n, H, Tt, bht.data(), cht.data(), dht.data(), hv, &tv)) { ++bad; continue; }
    if (oracle_spline_eval(n, Tt, Mt, btm.data(), ctm.data(), dtm.data(), tv, &mv) ||
        oracle_spline_eval(n, Tt, Kt, btk.data(), ctk.data(), dtk.data(), tv, &kv) ||
        oracle_spline_eval(n, Tt, Dt, btd.data(), ctd.data(), dtd.data(), tv, &dv)) {
      ++bad;
      continue;
    }
    if (std::fabs(tv - 1.0) < 1.0e-10) { mv = 1.0; kv = 1.0; dv = 1.0; }
    T[c] = tv;
    mu[c] = mv;
    k[c] = kv;
    rho[c] = dv;
  }
  return bad;
}

}  // extern "C"
