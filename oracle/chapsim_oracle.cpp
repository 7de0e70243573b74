// CPU FP64 oracle for the CHAPSim TG RK3 fractional-step substep.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA library.  Nothing in the
// product (libchapsim, the chapsim1ww_b200 host package) links, loads or calls
// this file.  Parity against reference outputs is unpinned (the Fortran
// reference cannot be built here and ships no golden data); the oracle is
// pinned by the reference's own self-checks and by an independent numpy
// restatement (tests/golden/).
//
// Every routine cites the reference file:line it restates (paths relative to
// the CHAPSim1WW project root).  Channel geometry only (icase = ICHANL), so the
// cylindrical metric factors RCCI1/RCCI2/RNDI1/RNDI2 are identically 1
// (src/COORDJR.f90:20-23) and are dropped from every formula below.
#include "chapsim_oracle.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cplx;

namespace {

// ---------------------------------------------------------------- utilities
inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Uniform draw in [-1, 1) keyed by (seed, component, i, j, k); identical to
// the product library's initial-field generator (same published splitmix64).
inline double rnd_pm1(uint64_t seed, int comp, int i, int j, int k) {
  uint64_t ctr = ((uint64_t)comp << 60) ^ ((uint64_t)k << 40) ^
                 ((uint64_t)j << 20) ^ (uint64_t)i;
  uint64_t x = splitmix64(splitmix64(seed) ^ ctr);
  double u = (double)(x >> 11) * (1.0 / 9007199254740992.0);
  return -1.0 + 2.0 * u;
}

// Mixed-radix recursive complex DFT (decimation in time, generic radix
// butterflies).  Semantics follow the CFFT99 definition
// (libs/fft99/CFFT99.f90:171-196): sign=-1 gives C(k)=sum g(j) e^{-2 pi i jk/N},
// sign=+1 the unnormalised inverse.  Lengths with any prime factor are allowed.
struct Dft {
  int n = 0;
  std::vector<cplx> tw[2];  // tw[s][m] = exp(sign*2 pi i m/n)
  void init(int n_) {
    n = n_;
    for (int s = 0; s < 2; ++s) {
      tw[s].resize(n);
      double sg = s == 0 ? -1.0 : 1.0;
      for (int m = 0; m < n; ++m) {
        double a = 2.0 * M_PI * (double)m / (double)n;
        tw[s][m] = cplx(std::cos(a), sg * std::sin(a));
      }
    }
  }
  static int smallest_factor(int m) {
    for (int p = 2; p * p <= m; ++p)
      if (m % p == 0) return p;
    return m;
  }
  // x: input with stride, y: output contiguous length m (m divides n);
  // tmp: scratch of length >= m, reused by every recursion level because a
  // level touches it only after its sub-transforms have returned.
  void rec(const cplx *x, int stride, cplx *y, int m, const std::vector<cplx> &w,
           cplx *tmp) const {
    if (m == 1) { y[0] = x[0]; return; }
    int p = smallest_factor(m);
    int q = m / p;
    for (int r = 0; r < p; ++r) rec(x + r * stride, stride * p, y + r * q, q, w, tmp);
    int tstep = n / m;  // exp(sign 2 pi i / m) = w[tstep]
    if (p == 2) {
      for (int k = 0; k < q; ++k) {
        cplx t = w[(size_t)k * tstep] * y[q + k];
        tmp[k] = y[k] + t;
        tmp[k + q] = y[k] - t;
      }
    } else {
      for (int k = 0; k < q; ++k)
        for (int s = 0; s < p; ++s) {
          int kk = k + s * q;
          cplx acc = 0.0;
          long e = 0;
          for (int r = 0; r < p; ++r) {
            acc += w[(size_t)e * tstep] * y[r * q + k];
            e += kk;
            if (e >= m) e %= m;
          }
          tmp[kk] = acc;
        }
    }
    for (int kk = 0; kk < m; ++kk) y[kk] = tmp[kk];
  }
  void run(const cplx *in, cplx *out, int sign, cplx *tmp) const {
    rec(in, 1, out, n, tw[sign < 0 ? 0 : 1], tmp);
  }
};

// Cyclic tridiagonal solve, TDMAIJI_CYC (src/TDMAIJI_CYC.f90:67-154):
// two-sweep elimination carrying a second right-hand side for the corner
// coupling.  a/b/c/r indexed 0..n-1, r overwritten by the solution.
void tdma_cyc(const double *a, const double *b, const double *c, double *r, int n,
              double *h0, double *g1, double *g2) {
  h0[0] = c[0] / b[0];
  g1[0] = r[0] / b[0];
  g2[0] = -a[0] / b[0];
  for (int i = 1; i <= n - 3; ++i) {
    double pp = 1.0 / (b[i] - h0[i - 1] * a[i]);
    h0[i] = c[i] * pp;
    g1[i] = (r[i] - g1[i - 1] * a[i]) * pp;
    g2[i] = -(g2[i - 1] * a[i]) * pp;
  }
  {
    int i = n - 2;
    double pp = 1.0 / (b[i] - h0[i - 1] * a[i]);
    g1[i] = (r[i] - g1[i - 1] * a[i]) * pp;
    g2[i] = (-c[i] - g2[i - 1] * a[i]) * pp;
  }
  for (int i = n - 3; i >= 0; --i) {
    g1[i] = -h0[i] * g1[i + 1] + g1[i];
    g2[i] = -h0[i] * g2[i + 1] + g2[i];
  }
  {
    int i = n - 1;
    double pp = r[i] - c[i] * g1[0] - a[i] * g1[i - 1];
    double qq = b[i] + c[i] * g2[0] + a[i] * g2[i - 1];
    r[i] = pp / qq;
  }
  for (int i = n - 2; i >= 0; --i) r[i] = g1[i] + g2[i] * r[n - 1];
}

// Non-cyclic Thomas solve with zero boundary vector, TDMAIJJ_nonCYC
// (src/TDMAIJJ_nonCYC.f90:67-120).
void tdma_noncyc(const double *a, const double *b, const double *c, double *r, int n,
                 double *h, double *g) {
  h[0] = c[0] / b[0];
  g[0] = r[0] / b[0];
  for (int j = 1; j <= n - 2; ++j) {
    double pp = 1.0 / (b[j] - h[j - 1] * a[j]);
    h[j] = c[j] * pp;
    g[j] = (r[j] - a[j] * g[j - 1]) * pp;
  }
  {
    int j = n - 1;
    double pp = 1.0 / (b[j] - h[j - 1] * a[j]);
    g[j] = (r[j] - a[j] * g[j - 1]) * pp;
    r[j] = g[j];
  }
  for (int j = n - 2; j >= 0; --j) r[j] = g[j] - h[j] * r[j + 1];
}

}  // namespace

static int g_threads = 0;

struct oracle_tg {
  int nx, ny, nz;
  double lx, lz, str2, ren, dt, cfgv;
  int istr2, flowdrvtp;
  double dx, dxi, dxqi, dz, dzi, dzqi, cvisc, volm, area_inlet;
  // 1-based y arrays, allocated ny+2 (index 0..ny+1).
  std::vector<double> ynd, ycc, dyfi, dyci, wff, wfb, amph, acph, apph;
  std::vector<double> amvr[4], acvr[4], apvr[4];  // idr 1..3
  std::vector<double> ak1, ak3;                   // modified wavenumbers
  double tgam[4], troh[4], talp[4];
  // fields, Fortran layout (nx, 0:ny+1, nz)
  std::vector<double> q[4];      // 1..3
  std::vector<double> pr, dph, rhsllphi, qtmp, rhs;
  std::vector<double> convh0[4];  // 1..3
  Dft dftx, dftz;

  int64_t len() const { return (int64_t)nx * (ny + 2) * nz; }
  inline int64_t id(int i, int j, int k) const {  // i,k 1-based; j 0..ny+1
    return (int64_t)(i - 1) + (int64_t)nx * ((int64_t)j + (int64_t)(ny + 2) * (k - 1));
  }
  inline int ip(int i) const { return i == nx ? 1 : i + 1; }  // IPV_tg, INDEXSET.f90:16-21
  inline int im(int i) const { return i == 1 ? nx : i - 1; }  // IMV_tg
  inline int kp(int k) const { return k == nz ? 1 : k + 1; }  // KPV, INDEXSET.f90:42-47
  inline int km(int k) const { return k == 1 ? nz : k - 1; }  // KMV
};

#define Q(n, i, j, k) o->q[n][o->id(i, j, k)]

extern "C" {

void oracle_set_threads(int n) { g_threads = n; }
int oracle_get_threads(void) {
#ifdef _OPENMP
  return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
  return 1;
#endif
}

static void setup_mesh(oracle_tg *o) {
  const int ny = o->ny, nnd2 = ny + 1;
  // CONSPARA.f90:41-73 (TG only).
  o->dx = o->lx / (double)o->nx;
  o->dxi = 1.0 / o->dx;
  o->dxqi = o->dxi * o->dxi;
  o->dz = o->lz / (double)o->nz;
  o->dzi = 1.0 / o->dz;
  o->dzqi = o->dzi * o->dzi;
  o->cvisc = 1.0 / o->ren;
  o->ynd.assign(ny + 2, 0.0);
  o->ycc.assign(ny + 2, 0.0);
  o->dyfi.assign(ny + 2, 0.0);
  o->dyci.assign(ny + 2, 0.0);
  o->wff.assign(ny + 2, 0.0);
  o->wfb.assign(ny + 2, 0.0);
  // COORDJR.f90:27-48: tanh stretching (istr2=1) or uniform (istr2=0),
  // y in [-1, 1]; cell centres are mapped (not averaged) when stretched.
  for (int j = 1; j <= nnd2; ++j) {
    if (o->istr2 == 1) {
      double x2 = (double)(j - 1) / (double)(nnd2 - 1);
      o->ynd[j] = std::tanh(o->str2 * (x2 - 0.5)) / std::tanh(o->str2 * 0.5);
    } else {
      o->ynd[j] = -1.0 + (double)(j - 1) * (2.0 / (double)ny);
    }
  }
  for (int j = 1; j <= ny; ++j) {
    if (o->istr2 == 1) {
      double x2 = ((double)(j - 1) + 0.5) / (double)(nnd2 - 1);
      o->ycc[j] = std::tanh(o->str2 * (x2 - 0.5)) / std::tanh(o->str2 * 0.5);
    } else {
      o->ycc[j] = 0.5 * (o->ynd[j] + o->ynd[j + 1]);
    }
  }
  // COORDJR.f90:130-143: inverse spacings; wall DYCI is a half cell.
  for (int j = 1; j <= ny; ++j) o->dyfi[j] = 1.0 / (o->ynd[j + 1] - o->ynd[j]);
  for (int j = 2; j <= nnd2 - 1; ++j) o->dyci[j] = 1.0 / ((o->ynd[j + 1] - o->ynd[j - 1]) * 0.5);
  o->dyci[1] = 2.0 / (o->ynd[2] - o->ynd[1]);
  o->dyci[nnd2] = 2.0 / (o->ynd[nnd2] - o->ynd[ny]);
  // MESH_YWEIGHT_FACTORS, COORDJR.f90:427-450.
  for (int jc = 2; jc <= ny; ++jc) {
    int jm = jc - 1;
    o->wff[jc] = (o->ynd[jc] - o->ycc[jm]) / (o->ycc[jc] - o->ycc[jm]);
    o->wfb[jc] = (o->ycc[jc] - o->ynd[jc]) / (o->ycc[jc] - o->ycc[jm]);
  }
  o->wfb[1] = 1.0; o->wff[1] = 0.0;
  o->wfb[nnd2] = 0.0; o->wff[nnd2] = 1.0;
  // AREA_INOUTLET, COORDJR.f90:495-520 (channel, RCCI1 = 1).
  o->area_inlet = 0.0;
  for (int j = 1; j <= ny; ++j)
    for (int k = 1; k <= o->nz; ++k) o->area_inlet += 1.0 / o->dyfi[j] / o->dzi;
  o->volm = 0.0;
  for (int k = 1; k <= o->nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= o->nx; ++i) o->volm += 1.0 / o->dyfi[j];
  // TDMA_COEF, src/TDMA_COEF.f90:53-119 (ICHANL branch).
  o->amph.assign(ny + 2, 0.0);
  o->acph.assign(ny + 2, 0.0);
  o->apph.assign(ny + 2, 0.0);
  for (int jc = 1; jc <= ny; ++jc) {
    int jp = jc + 1;
    o->amph[jc] = o->dyfi[jc] * o->dyci[jc];
    o->apph[jc] = o->dyfi[jc] * o->dyci[jp];
    if (jc == 1) o->amph[jc] = o->dyfi[jc] * o->dyci[jc] * 0.5;
    if (jp == nnd2) o->apph[jc] = o->dyfi[jc] * o->dyci[jp] * 0.5;
  }
  for (int jc = 1; jc <= ny; ++jc) o->acph[jc] = -(o->amph[jc] + o->apph[jc]);
  o->acph[1] = o->amph[1] + o->acph[1];
  o->amph[1] = 0.0;
  o->acph[ny] = o->apph[ny] + o->acph[ny];
  o->apph[ny] = 0.0;
  for (int idr = 1; idr <= 3; ++idr) {
    o->amvr[idr].assign(ny + 2, 0.0);
    o->acvr[idr].assign(ny + 2, 0.0);
    o->apvr[idr].assign(ny + 2, 0.0);
    if (idr == 1 || idr == 3) {
      for (int jc = 2; jc <= ny - 1; ++jc) {
        int jp = jc + 1;
        o->amvr[idr][jc] = o->dyfi[jc] * o->dyci[jc];
        o->apvr[idr][jc] = o->dyfi[jc] * o->dyci[jp];
        o->acvr[idr][jc] = -(o->amvr[idr][jc] + o->apvr[idr][jc]);
      }
      double ucaj = 4.0 / (2.0 / o->dyci[2] + 1.0 / o->dyfi[1]);
      o->amvr[idr][1] = 0.0;
      o->apvr[idr][1] = ucaj * o->dyci[2];
      o->acvr[idr][1] = -ucaj * (o->dyci[2] + 2.0 * o->dyfi[1]);
      ucaj = 4.0 / (2.0 / o->dyci[ny] + 1.0 / o->dyfi[ny]);
      o->amvr[idr][ny] = ucaj * o->dyci[ny];
      o->apvr[idr][ny] = 0.0;
      o->acvr[idr][ny] = -ucaj * (2.0 * o->dyfi[ny] + o->dyci[ny]);
    } else {
      for (int jc = 2; jc <= ny; ++jc) {
        int jm = jc - 1;
        o->amvr[idr][jc] = o->dyfi[jm] * o->dyci[jc];
        o->apvr[idr][jc] = o->dyfi[jc] * o->dyci[jc];
        o->acvr[idr][jc] = -(o->amvr[idr][jc] + o->apvr[idr][jc]);
      }
      o->amvr[idr][1] = 0.0; o->apvr[idr][1] = 0.0; o->acvr[idr][1] = 1.0;
      o->amvr[idr][nnd2] = 0.0; o->apvr[idr][nnd2] = 0.0; o->acvr[idr][nnd2] = 1.0;
    }
  }
  // FFT99_ROOT modified wavenumbers, src/possion3d_FFT99.f90:155-179.
  o->ak1.assign(o->nx, 0.0);
  o->ak3.assign(o->nz, 0.0);
  for (int i = 1; i <= o->nx; ++i) {
    double ap = (i <= o->nx / 2) ? (double)(i - 1) * 2.0 * M_PI
                                 : -(double)(o->nx - i + 1) * 2.0 * M_PI;
    o->ak1[i - 1] = 2.0 * (1.0 - std::cos(ap / o->nx)) * o->dxqi;
  }
  for (int k = 1; k <= o->nz; ++k) {
    double an = (k <= o->nz / 2) ? (double)(k - 1) * 2.0 * M_PI
                                 : -(double)(o->nz - k + 1) * 2.0 * M_PI;
    o->ak3[k - 1] = 2.0 * (1.0 - std::cos(an / o->nz)) * o->dzqi;
  }
  // CONS_RKCOEF, src/CONS_RKCOEF.f90:24-54.
  o->tgam[0] = 1.0; o->tgam[1] = 8.0 / 15.0; o->tgam[2] = 5.0 / 12.0; o->tgam[3] = 3.0 / 4.0;
  o->troh[0] = 0.0; o->troh[1] = 0.0; o->troh[2] = -17.0 / 60.0; o->troh[3] = -5.0 / 12.0;
  for (int n = 0; n < 4; ++n) o->talp[n] = o->tgam[n] + o->troh[n];
}

oracle_tg *oracle_tg_create(int nx, int ny, int nz, double lx, double lz, double str2,
                            int istr2, double ren, double dt, int flowdrvtp, double cfgv) {
  if (nx < 4 || ny < 4 || nz < 4 || (nx % 2) || (nz % 2)) return nullptr;
  oracle_tg *o = new oracle_tg();
  o->nx = nx; o->ny = ny; o->nz = nz;
  o->lx = lx; o->lz = lz; o->str2 = str2; o->istr2 = istr2;
  o->ren = ren; o->dt = dt; o->flowdrvtp = flowdrvtp; o->cfgv = cfgv;
  setup_mesh(o);
  int64_t n = o->len();
  for (int c = 1; c <= 3; ++c) { o->q[c].assign(n, 0.0); o->convh0[c].assign(n, 0.0); }
  o->pr.assign(n, 0.0); o->dph.assign(n, 0.0); o->rhsllphi.assign(n, 0.0);
  o->qtmp.assign(n, 0.0); o->rhs.assign(n, 0.0);
  o->dftx.init(nx);
  o->dftz.init(nz);
  return o;
}

void oracle_tg_destroy(oracle_tg *o) { delete o; }

// The complex DFT above, shared with the IO-section oracle.
struct oracle_dft {
  Dft d;
};
oracle_dft *oracle_dft_create(int n) {
  if (n < 1) return nullptr;
  oracle_dft *f = new oracle_dft();
  f->d.init(n);
  return f;
}
void oracle_dft_destroy(oracle_dft *f) { delete f; }
void oracle_dft_run(const oracle_dft *f, const double *in, double *out, int sign, double *tmp) {
  f->d.run(reinterpret_cast<const cplx *>(in), reinterpret_cast<cplx *>(out), sign, reinterpret_cast<cplx *>(tmp));
}
int64_t oracle_tg_field_len(const oracle_tg *o) { return o->len(); }

static std::vector<double> *field_ptr(oracle_tg *o, int id) {
  switch (id) {
    case ORC_U: return &o->q[1];
    case ORC_V: return &o->q[2];
    case ORC_W: return &o->q[3];
    case ORC_P: return &o->pr;
    case ORC_PHI: return &o->dph;
    case ORC_RHSPHI: return &o->rhsllphi;
    case ORC_H0U: return &o->convh0[1];
    case ORC_H0V: return &o->convh0[2];
    case ORC_H0W: return &o->convh0[3];
  }
  return nullptr;
}

int oracle_tg_get_field(const oracle_tg *o, int id, double *out) {
  auto *f = field_ptr(const_cast<oracle_tg *>(o), id);
  if (!f) return -1;
  std::memcpy(out, f->data(), sizeof(double) * f->size());
  return 0;
}
int oracle_tg_set_field(oracle_tg *o, int id, const double *in) {
  auto *f = field_ptr(o, id);
  if (!f) return -1;
  std::memcpy(f->data(), in, sizeof(double) * f->size());
  return 0;
}

int oracle_tg_get_coef(const oracle_tg *o, int what, double *out) {
  const int ny = o->ny;
  const std::vector<double> *v = nullptr;
  int lo = 1, hi = ny;
  switch (what) {
    case 0: v = &o->ynd; hi = ny + 1; break;
    case 1: v = &o->ycc; break;
    case 2: v = &o->dyfi; break;
    case 3: v = &o->dyci; hi = ny + 1; break;
    case 4: v = &o->wff; hi = ny + 1; break;
    case 5: v = &o->wfb; hi = ny + 1; break;
    case 6: v = &o->amph; break;
    case 7: v = &o->acph; break;
    case 8: v = &o->apph; break;
    default:
      if (what >= 9 && what <= 17) {
        int idr = (what - 9) / 3 + 1, t = (what - 9) % 3;
        v = t == 0 ? &o->amvr[idr] : (t == 1 ? &o->acvr[idr] : &o->apvr[idr]);
        hi = ny + 1;
      } else {
        return -1;
      }
  }
  for (int j = lo; j <= hi; ++j) out[j - lo] = (*v)[j];
  return hi - lo + 1;
}

double oracle_tg_volm(const oracle_tg *o) { return o->volm; }

// BC_WALL_Q (src/BC_WALL.f90:204-230): no-slip ghosts and v on the walls.
static void bc_wall_q(oracle_tg *o) {
  const int ny = o->ny;
  for (int k = 1; k <= o->nz; ++k)
    for (int i = 1; i <= o->nx; ++i) {
      Q(1, i, 0, k) = 0.0; Q(3, i, 0, k) = 0.0; Q(2, i, 1, k) = 0.0; Q(2, i, 0, k) = 0.0;
      Q(1, i, ny + 1, k) = 0.0; Q(3, i, ny + 1, k) = 0.0; Q(2, i, ny + 1, k) = 0.0;
    }
}
// BC_WALL_PR / BC_WALL_DPH (src/BC_WALL.f90:268-408): zero normal gradient.
static void bc_wall_copy(oracle_tg *o, std::vector<double> &f) {
  const int ny = o->ny;
  for (int k = 1; k <= o->nz; ++k)
    for (int i = 1; i <= o->nx; ++i) {
      f[o->id(i, 0, k)] = f[o->id(i, 1, k)];
      f[o->id(i, ny + 1, k)] = f[o->id(i, ny, k)];
    }
}

// CONVECTION_X_tg / _Y_tg / _Z_tg (src/CONVECTION_X.f90:23-74,
// src/CONVECTION_Y.f90:22-91, src/CONVECTION_Z.f90:22-75), channel branch.
static void convection(oracle_tg *o) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  const double xnd2cl = 0.5, ynd2cl = 0.5, znd2cl = 0.5;
  std::fill(o->qtmp.begin(), o->qtmp.end(), 0.0);
  std::fill(o->dph.begin(), o->dph.end(), 0.0);
  std::fill(o->rhsllphi.begin(), o->rhsllphi.end(), 0.0);
#pragma omp parallel for num_threads(oracle_get_threads()) schedule(static)
  for (int jc = 1; jc <= ny; ++jc) {
    const int jm = jc - 1, jp = jc + 1, jj = jc, jjp = jj + 1, jjm = jj - 1;
    const double *wff = o->wff.data(), *wfb = o->wfb.data();
    // x-momentum
    double coe1 = xnd2cl * xnd2cl * o->dxi;
    double coe2 = o->dyfi[jj] * xnd2cl;
    double coe3 = xnd2cl * znd2cl * o->dzi;
    for (int kc = 1; kc <= nz; ++kc) {
      int km = o->km(kc), kp = o->kp(kc);
      for (int ic = 1; ic <= nx; ++ic) {
        int ip = o->ip(ic), im = o->im(ic);
        double h11 = ((Q(1, ip, jc, kc) + Q(1, ic, jc, kc)) * (Q(1, ip, jc, kc) + Q(1, ic, jc, kc)) -
                      (Q(1, im, jc, kc) + Q(1, ic, jc, kc)) * (Q(1, im, jc, kc) + Q(1, ic, jc, kc))) * coe1;
        double h12 = ((Q(2, ic, jp, kc) + Q(2, im, jp, kc)) *
                          (wff[jjp] * Q(1, ic, jp, kc) + wfb[jjp] * Q(1, ic, jc, kc)) -
                      (Q(2, ic, jc, kc) + Q(2, im, jc, kc)) *
                          (wff[jj] * Q(1, ic, jc, kc) + wfb[jj] * Q(1, ic, jm, kc))) * coe2;
        double h13 = ((Q(3, ic, jc, kp) + Q(3, im, jc, kp)) * (Q(1, ic, jc, kp) + Q(1, ic, jc, kc)) -
                      (Q(3, ic, jc, kc) + Q(3, im, jc, kc)) * (Q(1, ic, jc, kc) + Q(1, ic, jc, km))) * coe3;
        o->qtmp[o->id(ic, jc, kc)] = -(h11 + h12 + h13);
      }
    }
    // y-momentum: skips the wall face jc = 1 (NYI = 2 on the bottom rank).
    if (jc >= 2) {
      double c1 = o->dxi * xnd2cl;
      double c2 = o->dyci[jj] * ynd2cl * ynd2cl;
      double c31 = o->dzi * znd2cl;
      for (int kc = 1; kc <= nz; ++kc) {
        int km = o->km(kc), kp = o->kp(kc);
        for (int ic = 1; ic <= nx; ++ic) {
          int ip = o->ip(ic), im = o->im(ic);
          double h21 = ((wff[jj] * Q(1, ip, jc, kc) + wfb[jj] * Q(1, ip, jm, kc)) *
                            (Q(2, ip, jc, kc) + Q(2, ic, jc, kc)) -
                        (wff[jj] * Q(1, ic, jc, kc) + wfb[jj] * Q(1, ic, jm, kc)) *
                            (Q(2, ic, jc, kc) + Q(2, im, jc, kc))) * c1;
          double h22 = ((Q(2, ic, jp, kc) + Q(2, ic, jc, kc)) * (Q(2, ic, jp, kc) + Q(2, ic, jc, kc)) -
                        (Q(2, ic, jc, kc) + Q(2, ic, jm, kc)) * (Q(2, ic, jc, kc) + Q(2, ic, jm, kc))) * c2;
          double h23 = ((wff[jj] * Q(3, ic, jc, kp) + wfb[jj] * Q(3, ic, jm, kp)) *
                            (Q(2, ic, jc, kp) + Q(2, ic, jc, kc)) -
                        (wff[jj] * Q(3, ic, jc, kc) + wfb[jj] * Q(3, ic, jm, kc)) *
                            (Q(2, ic, jc, kc) + Q(2, ic, jc, km))) * c31;
          o->dph[o->id(ic, jc, kc)] = -(h21 + h22 + h23);
        }
      }
    }
    (void)jjm;
    // z-momentum
    double z1 = xnd2cl * znd2cl * o->dxi;
    double z2 = o->dyfi[jj] * znd2cl;
    double z3 = znd2cl * znd2cl * o->dzi;
    for (int kc = 1; kc <= nz; ++kc) {
      int km = o->km(kc), kp = o->kp(kc);
      for (int ic = 1; ic <= nx; ++ic) {
        int ip = o->ip(ic), im = o->im(ic);
        double h31 = ((Q(1, ip, jc, kc) + Q(1, ip, jc, km)) * (Q(3, ip, jc, kc) + Q(3, ic, jc, kc)) -
                      (Q(1, ic, jc, kc) + Q(1, ic, jc, km)) * (Q(3, ic, jc, kc) + Q(3, im, jc, kc))) * z1;
        double h32 = ((Q(2, ic, jp, kc) + Q(2, ic, jp, km)) *
                          (wff[jjp] * Q(3, ic, jp, kc) + wfb[jjp] * Q(3, ic, jc, kc)) -
                      (Q(2, ic, jc, kc) + Q(2, ic, jc, km)) *
                          (wff[jj] * Q(3, ic, jc, kc) + wfb[jj] * Q(3, ic, jm, kc))) * z2;
        double h33 = ((Q(3, ic, jc, kp) + Q(3, ic, jc, kc)) * (Q(3, ic, jc, kp) + Q(3, ic, jc, kc)) -
                      (Q(3, ic, jc, kc) + Q(3, ic, jc, km)) * (Q(3, ic, jc, kc) + Q(3, ic, jc, km))) * z3;
        o->rhsllphi[o->id(ic, jc, kc)] = -(h31 + h32 + h33);
      }
    }
  }
}

// RHS_CvLpGpS_tg (src/RHS_CvLpGpS_tg.f90:29-213) for component idr.
static void rhs_cvlpgps(oracle_tg *o, int ns, int idr) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  const int nii = (idr == 2) ? 2 : 1;
  const std::vector<double> &conv = idr == 1 ? o->qtmp : (idr == 2 ? o->dph : o->rhsllphi);
  const double coe1 = o->talp[ns] * o->cvisc;
  const double coe2 = o->talp[ns] * o->dt;
  std::vector<double> &h0 = o->convh0[idr];
#pragma omp parallel for num_threads(oracle_get_threads()) schedule(static)
  for (int kc = 1; kc <= nz; ++kc) {
    int km = o->km(kc), kp = o->kp(kc);
    for (int jc = nii; jc <= ny; ++jc) {
      int jm = jc - 1, jp = jc + 1, jj = jc;
      for (int ic = 1; ic <= nx; ++ic) {
        int ip = o->ip(ic), im = o->im(ic);
        int64_t c = o->id(ic, jc, kc);
        double rhsc = o->tgam[ns] * conv[c] + o->troh[ns] * h0[c];
        double rhsl = coe1 * ((Q(idr, ip, jc, kc) - 2.0 * Q(idr, ic, jc, kc) + Q(idr, im, jc, kc)) * o->dxqi +
                              (Q(idr, ic, jc, kp) - 2.0 * Q(idr, ic, jc, kc) + Q(idr, ic, jc, km)) * o->dzqi +
                              (Q(idr, ic, jp, kc) * o->apvr[idr][jj] + Q(idr, ic, jc, kc) * o->acvr[idr][jj] +
                               Q(idr, ic, jm, kc) * o->amvr[idr][jj]));
        h0[c] = conv[c];
        double pgm;
        if (idr == 1)
          pgm = (o->pr[c] - o->pr[o->id(im, jc, kc)]) * o->dxi * coe2;
        else if (idr == 2)
          pgm = (o->pr[c] - o->pr[o->id(ic, jm, kc)]) * o->dyci[jj] * coe2;
        else
          pgm = (o->pr[c] - o->pr[o->id(ic, jc, km)]) * o->dzi * coe2;
        o->rhs[c] = (rhsc + rhsl) * o->dt - pgm;
      }
    }
  }
  // Flow drive (NFLOW = 1, streamwise x), src/RHS_CvLpGpS_tg.f90:179-213.
  if (idr == 1) {
    double dpgrns = 0.0;
    if (o->flowdrvtp == 1) {
      // Same summation order as the reference: I outer, J, K inner.
      double s = 0.0;
      for (int ic = 1; ic <= nx; ++ic)
        for (int jc = 1; jc <= ny; ++jc)
          for (int kc = 1; kc <= nz; ++kc) s += o->rhs[o->id(ic, jc, kc)] / o->dyfi[jc];
      dpgrns = s / o->volm;
    } else if (o->flowdrvtp == 2) {
      dpgrns = -0.5 * o->cfgv * coe2;
    }
    for (int kc = 1; kc <= nz; ++kc)
      for (int jc = nii; jc <= ny; ++jc)
        for (int ic = 1; ic <= nx; ++ic) o->rhs[o->id(ic, jc, kc)] -= dpgrns;
  }
}

// MOMFA_tg (src/MOMFA_tg.f90:17-240): x cyclic, z cyclic, y non-cyclic
// Crank-Nicolson factors, then q += dq.  For idr = 2 the y-solve spans
// j = 1..ny although row 1 was not rebuilt for v: it still holds the u
// increment at j = 1 (reference behaviour, kept as is).
static void momfa(oracle_tg *o, int ns, int idr) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  const double facoe = 0.5 * o->talp[ns] * o->dt * o->cvisc;
  const int n2i = (idr == 2) ? 2 : 1;
  // x (MOMFA1_X_tg)
  {
    const double coe = -facoe * o->dxqi;
#pragma omp parallel num_threads(oracle_get_threads())
    {
      std::vector<double> a(nx, coe), b(nx, 1.0 - 2.0 * coe), c(nx, coe), r(nx), h0(nx), g1(nx), g2(nx);
#pragma omp for schedule(static) collapse(2)
      for (int k = 1; k <= nz; ++k)
        for (int j = n2i; j <= ny; ++j) {
          for (int i = 1; i <= nx; ++i) r[i - 1] = o->rhs[o->id(i, j, k)];
          tdma_cyc(a.data(), b.data(), c.data(), r.data(), nx, h0.data(), g1.data(), g2.data());
          for (int i = 1; i <= nx; ++i) o->rhs[o->id(i, j, k)] = r[i - 1];
        }
    }
  }
  // z (MOMFA2_Z_tg)
  {
    const double rmc2 = -facoe * o->dzqi;
#pragma omp parallel num_threads(oracle_get_threads())
    {
      std::vector<double> a(nz, rmc2), b(nz, 1.0 - 2.0 * rmc2), c(nz, rmc2), r(nz), h0(nz), g1(nz), g2(nz);
#pragma omp for schedule(static) collapse(2)
      for (int j = n2i; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
          for (int k = 1; k <= nz; ++k) r[k - 1] = o->rhs[o->id(i, j, k)];
          tdma_cyc(a.data(), b.data(), c.data(), r.data(), nz, h0.data(), g1.data(), g2.data());
          for (int k = 1; k <= nz; ++k) o->rhs[o->id(i, j, k)] = r[k - 1];
        }
    }
  }
  // y (MOMFA3_Y_tg), all rows j = 1..ny
  {
#pragma omp parallel num_threads(oracle_get_threads())
    {
      std::vector<double> a(ny), b(ny), c(ny), r(ny), h(ny), g(ny);
      for (int j = 1; j <= ny; ++j) {
        a[j - 1] = -facoe * o->amvr[idr][j];
        b[j - 1] = 1.0 - facoe * o->acvr[idr][j];
        c[j - 1] = -facoe * o->apvr[idr][j];
      }
#pragma omp for schedule(static) collapse(2)
      for (int k = 1; k <= nz; ++k)
        for (int i = 1; i <= nx; ++i) {
          for (int j = 1; j <= ny; ++j) r[j - 1] = o->rhs[o->id(i, j, k)];
          tdma_noncyc(a.data(), b.data(), c.data(), r.data(), ny, h.data(), g.data());
          for (int j = 1; j <= ny; ++j) o->rhs[o->id(i, j, k)] = r[j - 1];
        }
    }
  }
  for (int k = 1; k <= nz; ++k)
    for (int j = n2i; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) Q(idr, i, j, k) += o->rhs[o->id(i, j, k)];
}

int oracle_tg_divg(oracle_tg *o, int ns) {
  // DIVG_tg (src/DIVG.f90:21-57).
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  const double coe0 = 1.0 / (o->dt * o->talp[ns]);
  std::fill(o->rhsllphi.begin(), o->rhsllphi.end(), 0.0);
#pragma omp parallel for num_threads(oracle_get_threads()) schedule(static)
  for (int jc = 1; jc <= ny; ++jc) {
    int jp = jc + 1;
    double c1 = o->dxi, c2 = o->dyfi[jc];
    for (int kc = 1; kc <= nz; ++kc) {
      int kp = o->kp(kc);
      for (int ic = 1; ic <= nx; ++ic) {
        int ip = o->ip(ic);
        double d = (Q(1, ip, jc, kc) - Q(1, ic, jc, kc)) * c1 + (Q(2, ic, jp, kc) - Q(2, ic, jc, kc)) * c2 +
                   (Q(3, ic, jc, kp) - Q(3, ic, jc, kc)) * o->dzi;
        o->rhsllphi[o->id(ic, jc, kc)] = d * coe0;
      }
    }
  }
  return 0;
}

int oracle_tg_pois3d(oracle_tg *o) {
  // FFT99_POIS3D_periodicxz(ITG), src/possion3d_FFT99.f90:254-488, and the
  // coefficient set-up TDMA_PHI_COEF, :185-220.  Spectral data is (kx, j, kz)
  // with kx = 0..nx/2.
  const int nx = o->nx, ny = o->ny, nz = o->nz, lh = nx / 2 + 1;
  std::vector<cplx> spec((size_t)lh * ny * nz);
  auto S = [&](int kx, int j, int kz) -> cplx & { return spec[(size_t)kx + (size_t)lh * ((j - 1) + (size_t)ny * kz)]; };
  const double un1 = 1.0 / nx, un3 = 1.0 / nz;
#pragma omp parallel num_threads(oracle_get_threads())
  {
    std::vector<cplx> in(std::max(nx, nz)), out(std::max(nx, nz)), tmp(std::max(nx, nz));
    // forward x: (1/nx) sum x e^{-i...} for every (j, k) row (FFT99, ISIGN=-1)
#pragma omp for schedule(static) collapse(2)
    for (int j = 1; j <= ny; ++j)
      for (int k = 1; k <= nz; ++k) {
        for (int i = 1; i <= nx; ++i) in[i - 1] = cplx(o->rhsllphi[o->id(i, j, k)], 0.0);
        o->dftx.run(in.data(), out.data(), -1, tmp.data());
        for (int kx = 0; kx < lh; ++kx) S(kx, j, k - 1) = out[kx] * un1;
      }
    // forward z (CFFT99, ISIGN=-1) then scale 1/nz
#pragma omp for schedule(static) collapse(2)
    for (int j = 1; j <= ny; ++j)
      for (int kx = 0; kx < lh; ++kx) {
        for (int k = 0; k < nz; ++k) in[k] = S(kx, j, k);
        o->dftz.run(in.data(), out.data(), -1, tmp.data());
        for (int k = 0; k < nz; ++k) S(kx, j, k) = out[k] * un3;
      }
  }
  S(0, 1, 0) = 0.0;  // :324-327
  // y tridiagonal per (kx, kz); the real and imaginary parts are solved with
  // the same real coefficients (:334-443).
#pragma omp parallel num_threads(oracle_get_threads())
  {
    std::vector<double> a(ny), b(ny), c(ny), rr(ny), ri(ny), h(ny), g(ny);
#pragma omp for schedule(static) collapse(2)
    for (int kz = 0; kz < nz; ++kz)
      for (int kx = 0; kx < lh; ++kx) {
        for (int j = 1; j <= ny; ++j) {
          c[j - 1] = o->apph[j];
          a[j - 1] = o->amph[j];
          b[j - 1] = o->acph[j] + (-o->ak1[kx] - o->ak3[kz]);
        }
        if (kx == 0 && kz == 0) {  // mean mode: row 1 decoupled (:206-211)
          b[0] = o->acph[1] + (-o->ak1[0] - o->ak3[0]);
          c[0] = 0.0;
          a[0] = 0.0;
        }
        for (int j = 1; j <= ny; ++j) { rr[j - 1] = S(kx, j, kz).real(); ri[j - 1] = S(kx, j, kz).imag(); }
        if (kz == 0 && kx == 0) { rr[0] = 0.0; ri[0] = 0.0; }
        tdma_noncyc(a.data(), b.data(), c.data(), rr.data(), ny, h.data(), g.data());
        tdma_noncyc(a.data(), b.data(), c.data(), ri.data(), ny, h.data(), g.data());
        for (int j = 1; j <= ny; ++j) S(kx, j, kz) = cplx(rr[j - 1], ri[j - 1]);
      }
  }
  std::fill(o->dph.begin(), o->dph.end(), 0.0);
#pragma omp parallel num_threads(oracle_get_threads())
  {
    std::vector<cplx> in(std::max(nx, nz)), out(std::max(nx, nz)), tmp(std::max(nx, nz));
#pragma omp for schedule(static) collapse(2)
    for (int j = 1; j <= ny; ++j)
      for (int kx = 0; kx < lh; ++kx) {
        for (int k = 0; k < nz; ++k) in[k] = S(kx, j, k);
        o->dftz.run(in.data(), out.data(), +1, tmp.data());
        for (int k = 0; k < nz; ++k) S(kx, j, k) = out[k];
      }
    // inverse x (FFT99, ISIGN=+1): Hermitian extension; the imaginary parts of
    // the kx = 0 and kx = nx/2 coefficients are taken as zero.
#pragma omp for schedule(static) collapse(2)
    for (int j = 1; j <= ny; ++j)
      for (int k = 1; k <= nz; ++k) {
        for (int kx = 0; kx < lh; ++kx) in[kx] = S(kx, j, k - 1);
        in[0] = cplx(in[0].real(), 0.0);
        in[nx / 2] = cplx(in[nx / 2].real(), 0.0);
        for (int kx = lh; kx < nx; ++kx) in[kx] = std::conj(in[nx - kx]);
        o->dftx.run(in.data(), out.data(), +1, tmp.data());
        for (int i = 1; i <= nx; ++i) o->dph[o->id(i, j, k)] = out[i - 1].real();
      }
  }
  return 0;
}

int oracle_tg_velo_correction(oracle_tg *o, int ns) {
  // VELOUPDT_tg (src/VELO_CORRECTION.f90:19-105), then BC_WALL_Q_tg.
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  const double cx = o->dt * o->talp[ns] * o->dxi, cz = o->dt * o->talp[ns] * o->dzi;
#pragma omp parallel for num_threads(oracle_get_threads()) schedule(static)
  for (int kc = 1; kc <= nz; ++kc) {
    int km = o->km(kc);
    for (int jc = 1; jc <= ny; ++jc)
      for (int ic = 1; ic <= nx; ++ic) {
        int im = o->im(ic);
        Q(1, ic, jc, kc) -= (o->dph[o->id(ic, jc, kc)] - o->dph[o->id(im, jc, kc)]) * cx;
        Q(3, ic, jc, kc) -= (o->dph[o->id(ic, jc, kc)] - o->dph[o->id(ic, jc, km)]) * cz;
      }
    for (int jc = 2; jc <= ny; ++jc) {
      double cy = o->dt * o->talp[ns] * o->dyci[jc];
      for (int ic = 1; ic <= nx; ++ic)
        Q(2, ic, jc, kc) -= (o->dph[o->id(ic, jc, kc)] - o->dph[o->id(ic, jc - 1, kc)]) * cy;
    }
  }
  bc_wall_q(o);
  return 0;
}

int oracle_tg_prcalc(oracle_tg *o, int ns) {
  // PRCALC_tg (src/PRESSURE_CORRECTION.f90:1-24), then BC_WALL_PR_tg.
  const double be = 0.5 * o->talp[ns] * o->dt * o->cvisc;
  for (int k = 1; k <= o->nz; ++k)
    for (int j = 1; j <= o->ny; ++j)
      for (int i = 1; i <= o->nx; ++i) {
        int64_t c = o->id(i, j, k);
        o->pr[c] = o->pr[c] + o->dph[c] - be * o->rhsllphi[c];
      }
  bc_wall_copy(o, o->pr);
  return 0;
}

int oracle_tg_substep(oracle_tg *o, int ns) {
  // SOLVERRK3_MOM_tg (src/SOLVERRK3_MOM_tg.f90:28-57).
  if (ns < 0 || ns > 3) return -1;
  convection(o);
  for (int idr = 1; idr <= 3; ++idr) {
    rhs_cvlpgps(o, ns, idr);
    momfa(o, ns, idr);
  }
  bc_wall_q(o);
  oracle_tg_divg(o, ns);
  oracle_tg_pois3d(o);
  bc_wall_copy(o, o->dph);
  oracle_tg_velo_correction(o, ns);
  oracle_tg_prcalc(o, ns);
  return 0;
}

int oracle_tg_step(oracle_tg *o) {
  for (int ns = 1; ns <= 3; ++ns)
    if (oracle_tg_substep(o, ns)) return -1;
  return 0;
}

double oracle_tg_divmax(const oracle_tg *o) {
  // DIVGCK_tg (src/DIVGCK.f90:16-58).
  double dmax = 0.0;
  for (int k = 1; k <= o->nz; ++k) {
    int kp = o->kp(k);
    for (int j = 1; j <= o->ny; ++j)
      for (int i = 1; i <= o->nx; ++i) {
        int ip = o->ip(i);
        double d = (Q(1, ip, j, k) - Q(1, i, j, k)) * o->dxi + (Q(2, i, j + 1, k) - Q(2, i, j, k)) * o->dyfi[j] +
                   (Q(3, i, j, kp) - Q(3, i, j, k)) * o->dzi;
        dmax = std::max(dmax, std::fabs(d));
      }
  }
  return dmax;
}

// CFL_tg (src/CFL.f90:1-40).
double oracle_tg_cfl(const oracle_tg *o) {
  double m = 0.0;
  for (int k = 1; k <= o->nz; ++k)
    for (int j = 1; j <= o->ny; ++j)
      for (int i = 1; i <= o->nx; ++i) {
        const double q = (std::fabs((Q(1, i, j, k) + Q(1, o->ip(i), j, k)) * o->dxi) +
                          std::fabs((Q(2, i, j, k) + Q(2, i, j + 1, k)) * o->dyfi[j]) +
                          std::fabs((Q(3, i, j, k) + Q(3, i, j, o->kp(k))) * o->dzi)) * 0.5;
        m = std::fmax(m, q);
      }
  return m;
}

void oracle_tg_set_dt(oracle_tg *o, double dt) { o->dt = dt; }

// PP_MEAN_ZX_FLOW_TG (src/processing/PP_MEAN_ZX.f90:1-294), channel branch:
// per y-row U1 (4), UP (3), U2 (6), U3 (10), DVDL1 (9), DVDLP (9), DVDL2 (81),
// scaled by VL1313 = 1/(nx nz) and the cell-centring factors.  out holds
// ny * 122 values.
void oracle_tg_stats(const oracle_tg *o, double *out) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  const double vl = 1.0 / (double)(nx * nz);
  const double coe0 = vl, coe1 = vl * 0.5, coe2 = vl * (0.5 * 0.5), coe3 = vl * (0.5 * 0.5 * 0.5);
  double cog1[3][3] = {{vl * o->dxi, vl * 0.25, vl * 0.25 * o->dzi},
                       {vl * 0.25 * o->dxi, vl, vl * 0.25 * o->dzi},
                       {vl * 0.25 * o->dxi, vl * 0.25, vl * o->dzi}};
#pragma omp parallel for schedule(static) num_threads(oracle_get_threads())
  for (int j = 1; j <= ny; ++j) {
    double u1[4] = {0, 0, 0, 0}, up[3] = {0, 0, 0}, u2[6] = {0}, u3[10] = {0}, d1[3][3] = {{0}}, dp[3][3] = {{0}};
    static thread_local double d2[9][9];
    for (auto &r : d2)
      for (double &x : r) x = 0.0;
    const int jp = j + 1, jm = j - 1;
    for (int i = 1; i <= nx; ++i) {
      const int ip = o->ip(i), im = o->im(i);
      for (int k = 1; k <= nz; ++k) {
        const int kp = o->kp(k), km = o->km(k);
        double U[3], Uip[3], Uim[3], Ujp[3], Ujm[3], Ukp[3], Ukm[3];
        U[0] = Q(1, i, j, k) + Q(1, ip, j, k);
        Ujp[0] = Q(1, i, jp, k) + Q(1, ip, jp, k);
        Ujm[0] = Q(1, i, jm, k) + Q(1, ip, jm, k);
        Ukp[0] = Q(1, i, j, kp) + Q(1, ip, j, kp);
        Ukm[0] = Q(1, i, j, km) + Q(1, ip, j, km);
        U[2] = Q(3, i, j, k) + Q(3, i, j, kp);
        Uip[2] = Q(3, ip, j, k) + Q(3, ip, j, kp);
        Uim[2] = Q(3, im, j, k) + Q(3, im, j, kp);
        Ujp[2] = Q(3, i, jp, k) + Q(3, i, jp, kp);
        Ujm[2] = Q(3, i, jm, k) + Q(3, i, jm, kp);
        U[1] = Q(2, i, j, k) + Q(2, i, jp, k);
        Uip[1] = Q(2, ip, j, k) + Q(2, ip, jp, k);
        Uim[1] = Q(2, im, j, k) + Q(2, im, jp, k);
        Ukp[1] = Q(2, i, j, kp) + Q(2, i, jp, kp);
        Ukm[1] = Q(2, i, j, km) + Q(2, i, jp, km);
        const double p = o->pr[o->id(i, j, k)];
        for (int m = 0; m < 3; ++m) {
          u1[m] += U[m];
          up[m] += U[m] * p;
        }
        u1[3] += p;
        int l = 0;
        for (int m = 0; m < 3; ++m)
          for (int n = m; n < 3; ++n) u2[l++] += U[m] * U[n];
        l = 0;
        for (int m = 0; m < 3; ++m)
          for (int n = m; n < 3; ++n)
            for (int h = n; h < 3; ++h) u3[l++] += U[m] * U[n] * U[h];
        double D[3][3];
        D[0][0] = Q(1, ip, j, k) - Q(1, i, j, k);
        D[0][1] = (Ujp[0] - U[0]) * o->dyci[jp] + (U[0] - Ujm[0]) * o->dyci[j];
        D[0][2] = Ukp[0] - Ukm[0];
        D[1][0] = Uip[1] - Uim[1];
        D[1][1] = (Q(2, i, jp, k) - Q(2, i, j, k)) * o->dyfi[j];
        D[1][2] = Ukp[1] - Ukm[1];
        D[2][0] = Uip[2] - Uim[2];
        D[2][1] = (Ujp[2] - U[2]) * o->dyci[jp] + (U[2] - Ujm[2]) * o->dyci[j];
        D[2][2] = Q(3, i, j, kp) - Q(3, i, j, k);
        for (int m = 0; m < 3; ++m)
          for (int n = 0; n < 3; ++n) {
            d1[m][n] += D[m][n];
            dp[m][n] += D[m][n] * p;
          }
        for (int a = 0; a < 9; ++a)
          for (int b = 0; b < 9; ++b) d2[a][b] += D[a / 3][a % 3] * D[b / 3][b % 3];
      }
    }
    double *r = out + (size_t)(j - 1) * 122;
    int q = 0;
    for (int m = 0; m < 3; ++m) r[q++] = u1[m] * coe1;
    r[q++] = u1[3] * coe0;
    for (int m = 0; m < 3; ++m) r[q++] = up[m] * coe1;
    for (int m = 0; m < 6; ++m) r[q++] = u2[m] * coe2;
    for (int m = 0; m < 10; ++m) r[q++] = u3[m] * coe3;
    for (int m = 0; m < 3; ++m)
      for (int n = 0; n < 3; ++n) r[q++] = d1[m][n] * cog1[m][n];
    for (int m = 0; m < 3; ++m)
      for (int n = 0; n < 3; ++n) r[q++] = dp[m][n] * cog1[m][n];
    for (int a = 0; a < 9; ++a)
      for (int b = 0; b < 9; ++b) r[q++] = d2[a][b] * (cog1[a / 3][a % 3] * cog1[b / 3][b % 3]);
  }
}

double oracle_tg_bulk(const oracle_tg *o) {
  // BULK_VELOCITY_TG (src/INITIAL_FL_FLD_TG.f90:122-149).
  double s = 0.0;
  for (int j = 1; j <= o->ny; ++j)
    for (int i = 1; i <= o->nx; ++i)
      for (int k = 1; k <= o->nz; ++k) s += Q(1, i, j, k) / o->dyfi[j];
  s = s / o->dzi;
  return s / (o->area_inlet * (double)o->nx);
}

double oracle_tg_pois_residual(const oracle_tg *o) {
  // CHECK_FFT_SOLVER (src/PRESSURE_CORRECTION.f90:159-202): apply the discrete
  // operator to phi and compare with the right-hand side.  The mean of the
  // rhs over each y-plane is removed from row 1's check because that row is
  // replaced by the pinning condition.
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  double rmax = 0.0;
  // mean-mode compatibility: row j=1 of the (0,0) mode is not solved; compare
  // instead the residual with the j=1 plane mean removed.
  std::vector<double> lres((size_t)nx * nz);
  double mean1 = 0.0, meanr1 = 0.0;
  for (int j = 1; j <= ny; ++j)
    for (int k = 1; k <= nz; ++k)
      for (int i = 1; i <= nx; ++i) {
        int64_t c = o->id(i, j, k);
        double lp = (o->dph[o->id(o->ip(i), j, k)] - 2.0 * o->dph[c] + o->dph[o->id(o->im(i), j, k)]) * o->dxqi +
                    (o->dph[o->id(i, j, o->kp(k))] - 2.0 * o->dph[c] + o->dph[o->id(i, j, o->km(k))]) * o->dzqi;
        double ly = o->acph[j] * o->dph[c];
        if (j > 1) ly += o->amph[j] * o->dph[o->id(i, j - 1, k)];
        if (j < ny) ly += o->apph[j] * o->dph[o->id(i, j + 1, k)];
        double r = lp + ly - o->rhsllphi[c];
        if (j == 1) { lres[(size_t)(i - 1) + (size_t)nx * (k - 1)] = r; mean1 += r; meanr1 += 1.0; }
        else rmax = std::max(rmax, std::fabs(r));
      }
  mean1 /= meanr1;
  for (double r : lres) rmax = std::max(rmax, std::fabs(r - mean1));
  return rmax;
}

static void init_common_tail(oracle_tg *o) {
  // v = 0 on the bottom wall face, bulk rescale of u (src/INITIAL_FL_FLD_TG.f90:48-72)
  for (int k = 1; k <= o->nz; ++k)
    for (int i = 1; i <= o->nx; ++i) Q(2, i, 1, k) = 0.0;
  double ub = oracle_tg_bulk(o);
  for (auto &x : o->q[1]) x /= ub;
  bc_wall_q(o);
  std::fill(o->pr.begin(), o->pr.end(), 0.0);
  for (int c = 1; c <= 3; ++c) std::fill(o->convh0[c].begin(), o->convh0[c].end(), 0.0);
}

void oracle_tg_init_random(oracle_tg *o, uint64_t seed, double amp) {
  // RANDOM_FL_FLD_TG sequence (src/INITIAL_FL_FLD_TG.f90:2-72) with a
  // counter-based generator: perturb, remove xz means, add the laminar
  // profile 1.5(1-y^2) (LAMPOISLPROF.f90:49-56), v = 0 at the wall, rescale
  // the bulk velocity to 1.
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  for (auto &f : o->q) std::fill(f.begin(), f.end(), 0.0);
  for (int j = 1; j <= ny; ++j)
    for (int k = 1; k <= nz; ++k)
      for (int i = 1; i <= nx; ++i)
        for (int c = 1; c <= 3; ++c) Q(c, i, j, k) = amp * rnd_pm1(seed, c, i, j, k);
  for (int k = 1; k <= nz; ++k)
    for (int i = 1; i <= nx; ++i) Q(2, i, 1, k) = 0.0;
  for (int c = 1; c <= 3; ++c)
    for (int j = 1; j <= ny; ++j) {
      double s = 0.0;
      for (int i = 1; i <= nx; ++i)
        for (int k = 1; k <= nz; ++k) s += Q(c, i, j, k);
      s /= (double)(nx * nz);
      for (int i = 1; i <= nx; ++i)
        for (int k = 1; k <= nz; ++k) Q(c, i, j, k) -= s;
    }
  for (int j = 1; j <= ny; ++j) {
    double vini = 1.5 * (1.0 - o->ycc[j] * o->ycc[j]);
    for (int k = 1; k <= nz; ++k)
      for (int i = 1; i <= nx; ++i) Q(1, i, j, k) += vini;
  }
  init_common_tail(o);
}

void oracle_tg_init_poiseuille(oracle_tg *o) {
  for (auto &f : o->q) std::fill(f.begin(), f.end(), 0.0);
  for (int j = 1; j <= o->ny; ++j) {
    double vini = 1.5 * (1.0 - o->ycc[j] * o->ycc[j]);
    for (int k = 1; k <= o->nz; ++k)
      for (int i = 1; i <= o->nx; ++i) Q(1, i, j, k) = vini;
  }
  init_common_tail(o);
}

}  // extern "C"
