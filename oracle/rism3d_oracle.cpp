// CPU FP64 restatement of the reference 3D-RISM solve path -- TEST
// INFRASTRUCTURE ONLY (checker and timed CPU baseline; never shipped, never
// called by the product).  Each function names the reference routine it
// restates (paths relative to the reference's src-cuda/).
//
// Build: g++ -O3 -fopenmp -shared -fPIC (see oracle/build.py).
#include "rism3d_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>
#include <omp.h>

namespace {

typedef std::complex<double> cd;

// physical.h:4-17 (same CODATA values)
const double kAvogadro = 6.02214076e23;
const double kBohr = 0.5291771500001;      // Angstrom
const double kBoltzmann = 1.380649e-23;    // J/K
const double kHartree = 4.359744722207185e-18;  // J

// ---------------------------------------------------------------------------
// Mixed-radix complex FFT (own code; the reference uses cuFFT Z2Z,
// fft3d.cu:16,31,35).  Unnormalised; sign -1 = exp(-2 pi i jk/n).
// ---------------------------------------------------------------------------
struct Fft1 {
  int n = 0;
  std::vector<int> fac;     // radix sequence
  std::vector<cd> twf, twb; // exp(-+2 pi i k / n)

  explicit Fft1(int n_) : n(n_) {
    int r = n;
    while (r % 4 == 0) { fac.push_back(4); r /= 4; }
    while (r % 2 == 0) { fac.push_back(2); r /= 2; }
    for (int p = 3; r > 1;) {
      while (r % p == 0) { fac.push_back(p); r /= p; }
      p += 2;
      if (p * p > r && r > 1) { fac.push_back(r); r = 1; }
    }
    if (fac.empty()) fac.push_back(1);
    twf.resize(n);
    twb.resize(n);
    for (int k = 0; k < n; ++k) {
      double a = -2.0 * M_PI * (double)k / (double)n;
      twf[k] = cd(std::cos(a), std::sin(a));
      twb[k] = std::conj(twf[k]);
    }
  }

  // out[k] = sum_j in[j*is] W^{jk}
  void run(const cd *in, int is, cd *out, int sign) const {
    const cd *tw = sign < 0 ? twf.data() : twb.data();
    if (n == 1) { out[0] = in[0]; return; }
    rec(out, in, 1, is, 0, n, tw);
  }

  void rec(cd *out, const cd *in, int fstride, int is, int stage, int len,
           const cd *tw) const {
    const int p = fac[stage];
    const int m = len / p;
    if (m == 1) {
      for (int q = 0; q < p; ++q) out[q] = in[(size_t)q * fstride * is];
    } else {
      for (int q = 0; q < p; ++q)
        rec(out + q * m, in + (size_t)q * fstride * is, fstride * p, is,
            stage + 1, m, tw);
    }
    // radix-p butterflies over the p sub-transforms of length m
    if (p == 2) {
      for (int u = 0; u < m; ++u) {
        cd a = out[u];
        cd b = out[u + m] * tw[(size_t)u * fstride];
        out[u] = a + b;
        out[u + m] = a - b;
      }
    } else if (p == 4) {
      const cd jrot = (tw == twf.data()) ? cd(0, -1) : cd(0, 1);
      for (int u = 0; u < m; ++u) {
        cd a0 = out[u];
        cd a1 = out[u + m] * tw[(size_t)u * fstride];
        cd a2 = out[u + 2 * m] * tw[(size_t)2 * u * fstride];
        cd a3 = out[u + 3 * m] * tw[(size_t)3 * u * fstride];
        cd s02 = a0 + a2, d02 = a0 - a2;
        cd s13 = a1 + a3, d13 = (a1 - a3) * jrot;
        out[u] = s02 + s13;
        out[u + m] = d02 + d13;
        out[u + 2 * m] = s02 - s13;
        out[u + 3 * m] = d02 - d13;
      }
    } else {
      std::vector<cd> scr(p);
      for (int u = 0; u < m; ++u) {
        for (int q = 0; q < p; ++q) scr[q] = out[u + q * m];
        for (int q1 = 0; q1 < p; ++q1) {
          size_t k = (size_t)u + (size_t)q1 * m;
          cd acc = 0.0;
          for (int q = 0; q < p; ++q)
            acc += scr[q] * tw[(k * (size_t)q * fstride) % (size_t)n];
          out[k] = acc;
        }
      }
    }
  }
};

// In-place unnormalised 3D FFT of a [nz][ny][nx] (x fastest) complex grid.
void fft3d_raw(int nx, int ny, int nz, cd *a, int sign) {
  Fft1 fx(nx), fy(ny), fz(nz);
  const size_t nxy = (size_t)nx * ny;
#pragma omp parallel
  {
    std::vector<cd> lin(std::max(nx, std::max(ny, nz)));
    std::vector<cd> lout(lin.size());
#pragma omp for schedule(static)
    for (long l = 0; l < (long)ny * nz; ++l) {
      cd *row = a + (size_t)l * nx;
      fx.run(row, 1, lout.data(), sign);
      std::copy(lout.begin(), lout.begin() + nx, row);
    }
#pragma omp for schedule(static)
    for (long l = 0; l < (long)nx * nz; ++l) {
      int ix = (int)(l % nx), iz = (int)(l / nx);
      cd *base = a + ix + nxy * iz;
      fy.run(base, nx, lout.data(), sign);
      for (int j = 0; j < ny; ++j) base[(size_t)j * nx] = lout[j];
    }
#pragma omp for schedule(static)
    for (long l = 0; l < (long)nxy; ++l) {
      cd *base = a + l;
      fz.run(base, (int)nxy, lout.data(), sign);
      for (int j = 0; j < nz; ++j) base[(size_t)j * nxy] = lout[j];
    }
  }
}

// fft3d.cu:4-94.  dkf = exp(-i pi sum_d x_d/n_d) with x_d = i_d - n_d/2
// (set_kf, :71-83); dir = (-1)^(ix+iy+iz) (set_ir, :86-94).
// Forward: a <- dv dir FFT(dir dkf a); inverse: a <- (1/V) conj(dkf) dir
// IFFT(dir a) (execute, :22-38; timekf :41-49, timekb :52-60,
// timeirvol :63-68).
struct Shifted3D {
  int nx, ny, nz;
  size_t n;
  double volf, volb;
  std::vector<cd> dkf;
  std::vector<signed char> dir;
  Shifted3D(int nx_, int ny_, int nz_, double bx, double by, double bz)
      : nx(nx_), ny(ny_), nz(nz_) {
    n = (size_t)nx * ny * nz;
    double vol = bx * by * bz;
    volf = vol / (double)n;
    volb = 1.0 / vol;
    dkf.resize(n);
    dir.resize(n);
    for (int iz = 0; iz < nz; ++iz)
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
          size_t ip = ix + (size_t)nx * (iy + (size_t)ny * iz);
          int x = ix - nx / 2, y = iy - ny / 2, z = iz - nz / 2;
          double dkr = M_PI / nx * x + M_PI / ny * y + M_PI / nz * z;
          dkf[ip] = cd(std::cos(dkr), -std::sin(dkr));
          dir[ip] = ((ix + iy + iz) % 2 == 0) ? 1 : -1;
        }
  }
  void forward(cd *a) const {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) a[i] = (a[i] * (double)dir[i]) * dkf[i];
    fft3d_raw(nx, ny, nz, a, -1);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) a[i] *= (double)dir[i] * volf;
  }
  void inverse(cd *a) const {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) a[i] *= (double)dir[i];
    fft3d_raw(nx, ny, nz, a, +1);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i)
      a[i] = (a[i] * ((double)dir[i] * volb)) * std::conj(dkf[i]);
  }
};

// spline.cc:4-43 (natural cubic spline, own tridiagonal sweep)
void spline_coe(int np, const double *xp, const double *yp,
                std::vector<double> &c0, std::vector<double> &c1,
                std::vector<double> &c2) {
  std::vector<double> a(np), b(np), c(np), d(np), s(np);
  int n = np - 2;
  for (int k = 1; k <= n; ++k) {
    double hl = xp[k] - xp[k - 1];
    double hr = xp[k + 1] - xp[k];
    a[k] = hl / (hl + hr);
    b[k] = 1 - a[k];
    double q1 = (yp[k + 1] - yp[k]) / hr;
    double q2 = (yp[k] - yp[k - 1]) / hl;
    c[k] = 6.0 * ((q1 - q2) / (hl + hr));
    d[k] = 2.0;
  }
  for (int k = 1; k < n; ++k) {
    b[k] = b[k] / d[k];
    c[k] = c[k] / d[k];
    d[k + 1] = d[k + 1] - a[k + 1] * b[k];
    c[k + 1] = c[k + 1] - a[k + 1] * c[k];
  }
  s[n] = c[n] / d[n];
  for (int k = n - 1; k >= 1; --k) s[k] = c[k] - b[k] * s[k + 1];
  s[0] = s[n + 1] = 0.0;
  c0.assign(np, 0.0);
  c1.assign(np, 0.0);
  c2.assign(np, 0.0);
  for (int k = 0; k <= n; ++k) {
    double h = xp[k + 1] - xp[k];
    c1[k] = s[k] / 2.0;
    c2[k] = (s[k + 1] - s[k]) / (6.0 * h);
    c0[k] = (yp[k + 1] - yp[k]) / h - c1[k] * h - c2[k] * h * h;
  }
}

// splint.cc:4-20 (bisection, then cubic in t = x - x_k)
double splint(int np, const double *xp, const double *yp,
              const std::vector<double> &c0, const std::vector<double> &c1,
              const std::vector<double> &c2, double x) {
  int klo = 0, khi = np - 1;
  while (khi - klo > 1) {
    int k = (khi + klo) >> 1;
    if (xp[k] > x) khi = k; else klo = k;
  }
  int k = klo;
  double t = x - xp[k];
  return ((c2[k] * t + c1[k]) * t + c0[k]) * t + yp[k];
}

struct Problem {
  const OracleInput *in;
  int nx, ny, nz, nv;
  size_t n;
  double dv, vol, drx, dry, drz;
  Problem(const OracleInput *p) : in(p) {
    nx = p->nx; ny = p->ny; nz = p->nz; nv = p->natv;
    n = (size_t)nx * ny * nz;
    vol = p->bx * p->by * p->bz;
    dv = vol / (double)n;                   // cell.cc:9-11
    drx = p->bx / nx; dry = p->by / ny; drz = p->bz / nz;  // cell.cc:12-14
  }
  double rx(int ix) const { return (ix - nx / 2) * drx; }  // cal_LJ.cu:54
  double ry(int iy) const { return (iy - ny / 2) * dry; }
  double rz(int iz) const { return (iz - nz / 2) * drz; }
  // set_g (initialize_g.cu:53-63)
  void kvec(size_t ip, double &kx, double &ky, double &kz) const {
    int ix = (int)(ip % nx), iy = (int)((ip / nx) % ny), iz = (int)(ip / ((size_t)nx * ny));
    kx = 2.0 * M_PI * (ix - nx / 2.0 + 0.5) / in->bx;
    ky = 2.0 * M_PI * (iy - ny / 2.0 + 0.5) / in->by;
    kz = 2.0 * M_PI * (iz - nz / 2.0 + 0.5) / in->bz;
  }
};

// cal_LJ.cu:4-72 and cal_Coulomb.cu:8-155; with an ESP cube the closure's
// e is the cube times hartree / (kB T) (cal_Coulomb.cu:88-90) while fr and fk
// stay the point-charge forms
void potentials(const Problem &P, double *u, double *e, double *fr, cd *fk) {
  const OracleInput *in = P.in;
  const int na = in->natom, nv = P.nv;
  std::vector<double> siguv((size_t)na * nv), epsuv((size_t)na * nv);
  for (int iv = 0; iv < nv; ++iv)
    for (int iu = 0; iu < na; ++iu) {
      siguv[iu + (size_t)na * iv] = (in->sig[iu] + in->sigv[iv]) * 0.5;
      epsuv[iu + (size_t)na * iv] = std::sqrt(in->eps[iu] * in->epsv[iv]);
    }
  const double cut2 = 1.0e-2 * 1.0e-2;
  const double ikbt = 1.0 / (kAvogadro * kBoltzmann * in->temper);
  const double ubeta = kHartree * kBohr / (kBoltzmann * in->temper);
#pragma omp parallel for schedule(static)
  for (long ip = 0; ip < (long)P.n; ++ip) {
    int ix = (int)(ip % P.nx), iy = (int)((ip / P.nx) % P.ny),
        iz = (int)(ip / ((size_t)P.nx * P.ny));
    double rx = P.rx(ix), ry = P.ry(iy), rz = P.rz(iz);
    for (int iv = 0; iv < nv; ++iv) {
      double acc = 0.0;
      for (int iu = 0; iu < na; ++iu) {
        size_t iuv = iu + (size_t)na * iv;
        double dx = rx - in->xyz[3 * iu], dy = ry - in->xyz[3 * iu + 1],
               dz = rz - in->xyz[3 * iu + 2];
        double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 < cut2) r2 = cut2;
        double irs2 = siguv[iuv] * siguv[iuv] / r2;
        double irs6 = irs2 * irs2 * irs2;
        acc += epsuv[iuv] * 4.0 * irs6 * (irs6 - 1.0);
      }
      u[(size_t)iv * P.n + ip] = acc * ikbt;
    }
    double de = 0.0, dfr = 0.0;
    for (int iu = 0; iu < na; ++iu) {
      double dx = rx - in->xyz[3 * iu], dy = ry - in->xyz[3 * iu + 1],
             dz = rz - in->xyz[3 * iu + 2];
      double ra = std::sqrt(dx * dx + dy * dy + dz * dz);
      if (ra >= 1.0e-5) {
        double qr = in->q[iu] / ra;
        de += qr;
        dfr += qr * (1 - std::exp(-ra));
      } else {
        dfr += in->q[iu];
      }
    }
    e[ip] = in->esp ? in->esp[ip] * (kHartree / (kBoltzmann * in->temper)) : de * ubeta;
    fr[ip] = dfr * ubeta;
    double kx, ky, kz;
    P.kvec(ip, kx, ky, kz);
    double rk2 = kx * kx + ky * ky + kz * kz;
    double rk4i = 1.0 / (rk2 * (rk2 + 1.0));
    double re = 0.0, im = 0.0;
    for (int iu = 0; iu < na; ++iu) {
      double ruk = kx * in->xyz[3 * iu] + ky * in->xyz[3 * iu + 1] + kz * in->xyz[3 * iu + 2];
      double tmp = 4.0 * M_PI * in->q[iu] * rk4i;
      re += tmp * std::cos(ruk);
      im -= tmp * std::sin(ruk);
    }
    fk[ip] = cd(re * ubeta, im * ubeta);
  }
}

// initialize_g.cu:7-50 (sorted unique |k|) + solvent_spline.cu:8-91
// (spline each X[a][b] at the unique |k|).  Returns 0 or -1 when the
// largest |k| exceeds the table (solvent_spline.cu:18-21).
int chi_table(const Problem &P, std::vector<int> &indga,
              std::vector<double> &xuniq /* [nv][nv][nga] */, int &nga,
              std::vector<double> *ga_out = nullptr) {
  const OracleInput *in = P.in;
  std::vector<double> g2(P.n);
  for (size_t ip = 0; ip < P.n; ++ip) {
    double kx, ky, kz;
    P.kvec(ip, kx, ky, kz);
    g2[ip] = kx * kx + ky * ky + kz * kz;
  }
  std::vector<int> ord(P.n);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(),
                   [&](int a, int b) { return g2[a] < g2[b]; });
  std::vector<double> ga;
  indga.assign(P.n, 0);
  double ga2o = -1.0;
  nga = 0;
  for (size_t i = 0; i < P.n; ++i) {
    int igs = ord[i];
    double ga2 = g2[igs];
    if (ga2 > ga2o) {
      ++nga;
      ga.push_back(std::sqrt(ga2));
      ga2o = ga2;
    }
    indga[igs] = nga - 1;
  }
  const int ntab = in->ntab;
  std::vector<double> ttab(ntab);
  double dk = M_PI / (in->dr * ntab);           // solvent_read.cc:82-86
  for (int i = 0; i < ntab; ++i) ttab[i] = dk * (i + 1);
  if (ga[nga - 1] > ttab[ntab - 1]) return -1;
  if (ga_out) *ga_out = ga;
  const int nv = P.nv;
  xuniq.assign((size_t)nv * nv * nga, 0.0);
  std::vector<double> c0, c1, c2;
  for (int a = 0; a < nv; ++a)
    for (int b = 0; b < nv; ++b) {
      const double *y = in->xvv + ((size_t)a * nv + b) * ntab;
      spline_coe(ntab, ttab.data(), y, c0, c1, c2);
      double *dst = xuniq.data() + ((size_t)a * nv + b) * nga;
#pragma omp parallel for schedule(static)
      for (int i = 0; i < nga; ++i)
        dst[i] = splint(ntab, ttab.data(), y, c0, c1, c2, ga[i]);
    }
  return 0;
}

// Row-blocked sum: one partial per x-row, then a sequential sum of the
// partials (the reference reduces each x-row in a block, then
// thrust::reduce over rows; the order here is fixed so the oracle is
// deterministic for any thread count).
template <class F>
double grid_sum(const Problem &P, F f) {
  const long rows = (long)P.ny * P.nz;
  std::vector<double> part(rows);
#pragma omp parallel for schedule(static)
  for (long r = 0; r < rows; ++r) {
    double s = 0.0;
    size_t base = (size_t)r * P.nx;
    for (int ix = 0; ix < P.nx; ++ix) s += f(base + ix);
    part[r] = s;
  }
  double s = 0.0;
  for (long r = 0; r < rows; ++r) s += part[r];
  return s;
}

// excp_fd.cc:1-6: derivative of the hard-sphere excess free-energy density
// at packing fraction pf and density dens
double excp_fd(double pf, double dens) {
  return (4.0 - 2.0 * pf) / ((1.0 - pf) * (1.0 - pf) * (1.0 - pf)) * (pf / dens);
}

// cal_rmdft.cu:5-115 with the tables of solvent_spline2.cu:7-103: the
// solvent c(k) (.cvk) and the hard-sphere chi and weight of site 0 splined
// at the unique |k|; cvva_vv -= chs_v rho_0 / rho_v; then
//   xmu1 = -sum rho_v h_v,  w_v = F^-1[sum_v' c_vv' rho_v' H_v'],
//   xmu2 = sum rho_v w_v,   xmu3 = sum rho_v w_v h_v,
//   n_v = rho_0 + F^-1[rho_0 w_v H_v],
//   f_v = rho_0 ((h_v + 1) excp_fd(a n_v, n_v) - excp_fd(pf_v, rho_0)), a = pf_v / rho_0,
//   eda = sum rho_v ((F^-1[w_v F f_v] + e_v)(h_v + 1) - e_v),
//         e_v = rho_0 excp_fd(pf_v, rho_0) w_v(0),
// returning (xmu1 + xmu2 + xmu3 / 2 - eda) dv.  The file supplies site 0's
// hard-sphere data only; the other sites' tables are zero (the reference
// leaves them uninitialised).  h is transformed in place forth and back
// as the reference does.  Returns 0, or -4 when the hard-sphere table does
// not reach the largest |k| (solvent_spline2.cu:16-19).
int rmdft(const Problem &P, const Shifted3D &fft, const std::vector<int> &indga,
          const std::vector<double> &ga, std::vector<cd> huv, double *result) {
  const OracleInput *in = P.in;
  const int nv = P.nv, nga = (int)ga.size(), ntab = in->ntab, nt2 = in->ntab2;
  const size_t n = P.n;
  if (ga[nga - 1] > in->ttab2[nt2 - 1]) return -4;
  std::vector<double> ttab(ntab);
  const double dk = M_PI / (in->dr * ntab);
  for (int i = 0; i < ntab; ++i) ttab[i] = dk * (i + 1);
  std::vector<double> c0, c1, c2;
  std::vector<double> cva((size_t)nv * nv * nga), chsa((size_t)nv * nga, 0.0),
      wfka((size_t)nv * nga, 0.0), pf(nv, 0.0), w0(nv, 0.0);
  for (int a = 0; a < nv; ++a)
    for (int b = 0; b < nv; ++b) {               // solvent_spline.cu:50-62
      const double *y = in->cvv + ((size_t)a * nv + b) * ntab;
      spline_coe(ntab, ttab.data(), y, c0, c1, c2);
      for (int i = 0; i < nga; ++i)
        cva[((size_t)a * nv + b) * nga + i] = splint(ntab, ttab.data(), y, c0, c1, c2, ga[i]);
    }
  spline_coe(nt2, in->ttab2, in->chs, c0, c1, c2);
  for (int i = 0; i < nga; ++i) chsa[i] = splint(nt2, in->ttab2, in->chs, c0, c1, c2, ga[i]);
  spline_coe(nt2, in->ttab2, in->wfk, c0, c1, c2);
  for (int i = 0; i < nga; ++i) wfka[i] = splint(nt2, in->ttab2, in->wfk, c0, c1, c2, ga[i]);
  pf[0] = in->pfhs;
  w0[0] = in->wfk0;
  const double rho0 = in->rhov[0];
  for (int v = 0; v < nv; ++v)                   // solvent_spline2.cu:65-70
    for (int i = 0; i < nga; ++i)
      cva[((size_t)v * nv + v) * nga + i] -= chsa[(size_t)v * nga + i] * rho0 / in->rhov[v];
  double xmu1 = 0.0;
  for (int v = 0; v < nv; ++v) {
    const cd *h = &huv[(size_t)v * n];
    xmu1 -= grid_sum(P, [&](size_t i) { return h[i].real(); }) * in->rhov[v];
  }
  for (int v = 0; v < nv; ++v) fft.forward(&huv[(size_t)v * n]);
  std::vector<cd> work((size_t)nv * n);
  for (int v = 0; v < nv; ++v) {                 // cal_dwork
#pragma omp parallel for schedule(static)
    for (long ip = 0; ip < (long)n; ++ip) {
      const int ig = indga[ip];
      cd s(0.0, 0.0);
      for (int b = 0; b < nv; ++b)
        s += huv[(size_t)b * n + ip] * (cva[((size_t)v * nv + b) * nga + ig] * in->rhov[b]);
      work[(size_t)v * n + ip] = s;
    }
  }
  for (int v = 0; v < nv; ++v) {
    fft.inverse(&huv[(size_t)v * n]);
    fft.inverse(&work[(size_t)v * n]);
  }
  double xmu2 = 0.0, xmu3 = 0.0;
  for (int v = 0; v < nv; ++v) {
    const cd *w = &work[(size_t)v * n];
    xmu2 += grid_sum(P, [&](size_t i) { return w[i].real(); }) * in->rhov[v];
  }
  for (int v = 0; v < nv; ++v) {
    const cd *w = &work[(size_t)v * n], *h = &huv[(size_t)v * n];
    xmu3 += grid_sum(P, [&](size_t i) { return w[i].real() * h[i].real(); }) * in->rhov[v];
  }
  for (int v = 0; v < nv; ++v) fft.forward(&huv[(size_t)v * n]);
  for (int v = 0; v < nv; ++v) {                 // rho0wfkhk
    cd *w = &work[(size_t)v * n];
    const cd *h = &huv[(size_t)v * n];
#pragma omp parallel for schedule(static)
    for (long ip = 0; ip < (long)n; ++ip) w[ip] = h[ip] * (rho0 * wfka[(size_t)v * nga + indga[ip]]);
  }
  for (int v = 0; v < nv; ++v) {
    fft.inverse(&huv[(size_t)v * n]);
    fft.inverse(&work[(size_t)v * n]);
  }
  for (int v = 0; v < nv; ++v) {                 // rho0, rho0guvfmbex
    cd *w = &work[(size_t)v * n];
    const cd *h = &huv[(size_t)v * n];
    const double bex = excp_fd(pf[v], rho0), a = pf[v] / rho0;
#pragma omp parallel for schedule(static)
    for (long ip = 0; ip < (long)n; ++ip) {
      const double dens = w[ip].real() + rho0;
      w[ip] = cd(rho0 * ((h[ip].real() + 1.0) * excp_fd(a * dens, dens) - bex), 0.0);
    }
  }
  for (int v = 0; v < nv; ++v) {                 // wfka between the transforms
    cd *w = &work[(size_t)v * n];
    fft.forward(w);
#pragma omp parallel for schedule(static)
    for (long ip = 0; ip < (long)n; ++ip) w[ip] *= wfka[(size_t)v * nga + indga[ip]];
    fft.inverse(w);
  }
  double eda = 0.0;
  for (int v = 0; v < nv; ++v) {                 // cal_eda
    const cd *w = &work[(size_t)v * n], *h = &huv[(size_t)v * n];
    const double ex = rho0 * excp_fd(pf[v], rho0) * w0[v];
    eda += grid_sum(P, [&](size_t i) { return (w[i].real() + ex) * (h[i].real() + 1.0) - ex; }) *
           in->rhov[v];
  }
  *result = (xmu1 + xmu2 + 0.5 * xmu3 - eda) * P.dv;
  return 0;
}

// anderson.cu:87-112
void leg(double *a, double *x, double *b, int n, int nn) {
  int i, j, k, k1;
  double s, p, q, r;
  double *ai, *ak;
  for (k = 0, ak = a; k < n - 1; ++k, ak += nn) {
    k1 = k + 1;
    p = ak[k];
    for (j = k1; j < n; ++j) ak[j] /= p;
    r = b[k] /= p;
    for (i = k1, ai = ak + nn; i < n; ++i, ai += nn) {
      q = ai[k];
      for (j = k1; j < n; ++j) ai[j] -= q * ak[j];
      b[i] -= q * r;
    }
  }
  x[n - 1] = b[n - 1] / ak[n - 1];
  for (k = n - 2, ak = a + nn * (n - 2); k >= 0; --k, ak -= nn) {
    k1 = k + 1;
    s = b[k];
    for (j = k1; j < n; ++j) s -= ak[j] * x[j];
    x[k] = s;
  }
}

}  // namespace

extern "C" int oracle_num_threads(void) { return omp_get_max_threads(); }

extern "C" int oracle_spline_eval(int np, const double *xp, const double *yp,
                                  int nq, const double *xq, double *yq) {
  std::vector<double> c0, c1, c2;
  spline_coe(np, xp, yp, c0, c1, c2);
  for (int i = 0; i < nq; ++i) yq[i] = splint(np, xp, yp, c0, c1, c2, xq[i]);
  return 0;
}

extern "C" int oracle_fft3d(int nx, int ny, int nz, double bx, double by,
                            double bz, double *a, int key) {
  Shifted3D f(nx, ny, nz, bx, by, bz);
  if (key == -1) f.forward(reinterpret_cast<cd *>(a));
  else f.inverse(reinterpret_cast<cd *>(a));
  return 0;
}

extern "C" int oracle_potentials(const OracleInput *in, double *u, double *e,
                                 double *fr, double *fk) {
  Problem P(in);
  potentials(P, u, e, fr, reinterpret_cast<cd *>(fk));
  return 0;
}

extern "C" int oracle_chi_grid(const OracleInput *in, double *x) {
  Problem P(in);
  std::vector<int> indga;
  std::vector<double> xu;
  int nga;
  if (chi_table(P, indga, xu, nga)) return -1;
  for (int a = 0; a < P.nv; ++a)
    for (int b = 0; b < P.nv; ++b)
      for (size_t ip = 0; ip < P.n; ++ip)
        x[((size_t)a * P.nv + b) * P.n + ip] =
            xu[((size_t)a * P.nv + b) * nga + indga[ip]];
  return 0;
}

extern "C" int oracle_solve(const OracleInput *in, OracleResult *out,
                            double *g_out, double *h_out, double *t_out,
                            double *euv, double *dulj, double *due,
                            double *trace) {
  Problem P(in);
  const int nv = P.nv;
  const size_t n = P.n;
  if (nv < 1 || nv > ORACLE_MAXV) return -2;
  memset(out, 0, sizeof(*out));
  double w0 = omp_get_wtime();

  // --- setup: potentials, chi, FFT (initialize.cu:4-13) ---
  std::vector<double> u((size_t)nv * n), e(n), fr(n);
  std::vector<cd> fk(n);
  potentials(P, u.data(), e.data(), fr.data(), fk.data());
  std::vector<int> indga;
  std::vector<double> xu, ga;
  int nga;
  if (chi_table(P, indga, xu, nga, &ga)) return -3;
  Shifted3D fft(P.nx, P.ny, P.nz, in->bx, in->by, in->bz);
  double w1 = omp_get_wtime();
  out->t_setup = w1 - w0;

  // --- iterate (iterate.cu:6-90) ---
  std::vector<cd> guv((size_t)nv * n), huv((size_t)nv * n);
  std::vector<double> t((size_t)nv * n), tr((size_t)nv * n);
  std::vector<double> tp((size_t)2 * nv * n, 0.0), rp((size_t)2 * nv * n, 0.0);
  std::vector<double> irho(nv);
  for (int iv = 0; iv < nv; ++iv) irho[iv] = 1.0 / in->rhov[iv];
  int count = in->count, binary = 0;  // anderson.cu:13-32

  int cu = in->chargeup;
  double cf, cuf = 0.0;
  if (in->t_init) {                   // restart (iterate.cu:30-33)
    std::copy(in->t_init, in->t_init + (size_t)nv * n, t.begin());
    cu = 0;
    cf = 1.0;
  } else if (cu == 0) {               // initialize_tuv.cu:17-21
    for (int iv = 0; iv < nv; ++iv)
      for (size_t ip = 0; ip < n; ++ip) t[iv * n + ip] = in->qv[iv] * fr[ip];
    cf = 1.0;
  } else {
    std::fill(t.begin(), t.end(), 0.0);
    cuf = 1.0 / cu;
    cf = 0.0;
  }

  int total = 0, status = 0;
  double rms = 0.0;
  for (int c = 0; c <= cu; ++c) {
    if (c > 0) {                      // add_tuv.cu:15-19
      cf += cuf;
      if (cf > 1.0) cf = 1.0;
      for (int iv = 0; iv < nv; ++iv)
        for (size_t ip = 0; ip < n; ++ip) t[iv * n + ip] += in->qv[iv] * cuf * fr[ip];
    }
    bool conver = false, diverge = false;
    for (int istep = 1; istep <= in->maxstep; ++istep) {
      // calculate.cu:4-58 + calculate_cuda.cu
      for (int iv = 0; iv < nv; ++iv) {
        double q = in->qv[iv] * cf;
        double *tv = &t[iv * n], *trv = &tr[iv * n], *uv = &u[iv * n];
        cd *gv = &guv[iv * n];
#pragma omp parallel for schedule(static)
        for (long ip = 0; ip < (long)n; ++ip) {
          double earg = -uv[ip] - e[ip] * q + tv[ip];
          double gg;
          if (in->closure == 0) gg = (earg >= 0.0) ? 1.0 + earg : std::exp(earg);
          else gg = std::exp(earg);
          trv[ip] = gg;                                   // kh / hnc
          gv[ip] = cd(gg - 1.0 - tv[ip] + q * fr[ip], 0.0);   // trm1mt
        }
        fft.forward(gv);
#pragma omp parallel for schedule(static)
        for (long ip = 0; ip < (long)n; ++ip) gv[ip] -= q * fk[ip];   // mqvfk
      }
      for (int a = 0; a < nv; ++a) {                      // oz
        cd *hv = &huv[a * n];
#pragma omp parallel for schedule(static)
        for (long ip = 0; ip < (long)n; ++ip) {
          double hr = 0.0, hi = 0.0;
          int ig = indga[ip];
          for (int b = 0; b < nv; ++b) {
            double x = xu[((size_t)a * nv + b) * nga + ig];
            hr += guv[b * n + ip].real() * x;
            hi += guv[b * n + ip].imag() * x;
          }
          hv[ip] = cd(hr, hi);
        }
        fft.inverse(hv);
      }
      for (int iv = 0; iv < nv; ++iv) {                   // tr
        cd *gv = &guv[iv * n], *hv = &huv[iv * n];
        double *trv = &tr[iv * n];
#pragma omp parallel for schedule(static)
        for (long ip = 0; ip < (long)n; ++ip) {
          gv[ip] = cd(trv[ip], gv[ip].imag());
          trv[ip] = hv[ip].real() + 1.0 - trv[ip];
        }
      }
      // cal_rms.cu:13-22
      double s2 = 0.0;
      for (int iv = 0; iv < nv; ++iv) {
        const double *trv = &tr[iv * n];
        s2 += grid_sum(P, [&](size_t ip) { return trv[ip] * trv[ip]; });
      }
      rms = std::sqrt(s2 / ((double)n * nv));
      ++total;
      if (trace) trace[total - 1] = rms;
      if (in->verbose) printf(" Step = %d Reside = %g\n", istep, rms);
      diverge = !std::isfinite(rms);
      if (diverge) break;
      if (rms <= in->conv) {
        conver = true;
      } else if (count > 0) {         // AN2::calculate, anderson.cu:43-49
        --count;
        for (int iv = 0; iv < nv; ++iv) {
          size_t biv = (size_t)(iv + binary * nv) * n;
          double *tv = &t[iv * n], *trv = &tr[iv * n];
          for (size_t ip = 0; ip < n; ++ip) {
            tp[biv + ip] = tv[ip];
            rp[biv + ip] = trv[ip];
            tv[ip] += trv[ip];
          }
        }
        binary = (binary == 0) ? 1 : 0;
      } else {                        // anderson.cu:50-62 + cal_theta :66-84
        double a[4] = {0, 0, 0, 0}, cc[2] = {0, 0}, x[2];
        for (int iv = 0; iv < nv; ++iv) {
          const double *R = &tr[iv * n];
          const double *r0 = &rp[(size_t)iv * n];
          const double *r1 = &rp[(size_t)(iv + nv) * n];
          double s[5];
          s[0] = grid_sum(P, [&](size_t i) { return R[i] * (R[i] - r0[i]); });
          s[1] = grid_sum(P, [&](size_t i) { return R[i] * (R[i] - r1[i]); });
          s[2] = grid_sum(P, [&](size_t i) { double d = R[i] - r0[i]; return d * d; });
          s[3] = grid_sum(P, [&](size_t i) { return (R[i] - r0[i]) * (R[i] - r1[i]); });
          s[4] = grid_sum(P, [&](size_t i) { double d = R[i] - r1[i]; return d * d; });
          cc[0] += s[0] * irho[iv];
          cc[1] += s[1] * irho[iv];
          a[0] += s[2] * irho[iv];
          a[1] += s[3] * irho[iv];
          a[3] += s[4] * irho[iv];
        }
        a[2] = a[1];
        leg(a, x, cc, 2, 2);
        double s1 = x[0] + in->mp * ((binary == 0) ? 0 : 1);
        double s2c = x[1] + in->mp * ((binary == 0) ? 1 : 0);
        const double mm = in->m;
        for (int iv = 0; iv < nv; ++iv) {       // newdt, anderson_cuda.cu:11-23
          double *tv = &t[iv * n];
          const double *trv = &tr[iv * n];
          double *tp0 = &tp[(size_t)iv * n], *tp1 = &tp[(size_t)(iv + nv) * n];
          double *rp0 = &rp[(size_t)iv * n], *rp1 = &rp[(size_t)(iv + nv) * n];
          double *tpb = binary ? tp1 : tp0, *rpb = binary ? rp1 : rp0;
#pragma omp parallel for schedule(static)
          for (long ip = 0; ip < (long)n; ++ip) {
            double tt = tv[ip], rr = trv[ip];
            double uu = tt + s1 * (tp0[ip] - tt) + s2c * (tp1[ip] - tt);
            double vv = tt + rr + s1 * (tp0[ip] + rp0[ip] - tt - rr) +
                        s2c * (tp1[ip] + rp1[ip] - tt - rr);
            tpb[ip] = tt;
            rpb[ip] = rr;
            tv[ip] = uu + mm * (vv - uu);
          }
        }
        binary = (binary == 0) ? 1 : 0;
      }
      if (conver) break;
    }
    if (diverge) {
      status = 1;
    } else if (!conver) {
      status = 2;
      break;
    }
  }
  out->iterations = total;
  out->rms = rms;
  out->status = status;
  double w2 = omp_get_wtime();
  out->t_iter = w2 - w1;

  // --- observables (output.cu:6-62) ---
  const double ibeta = kAvogadro * kBoltzmann * in->temper;
  out->ibeta = ibeta;
  for (int iv = 0; iv < nv; ++iv) {     // cal_exchem.cu:4-154
    const cd *hv = &huv[iv * n];
    const double *tv = &t[iv * n];
    double skh = grid_sum(P, [&](size_t i) {
      double h = hv[i].real(), tt = tv[i];
      return (h > 0.0) ? -(h * 0.5 + 1.0) * (h - tt) : h * 0.5 * tt - (h - tt);
    });
    double shnc = grid_sum(P, [&](size_t i) {
      double h = hv[i].real(), tt = tv[i];
      return h * 0.5 * tt - (h - tt);
    });
    double sgf = grid_sum(P, [&](size_t i) {
      double h = hv[i].real(), tt = tv[i];
      return -(h * 0.5 + 1.0) * (h - tt);
    });
    out->xmu_sc[iv] = (in->closure == 0 ? skh : shnc) * in->rhov[iv] * P.dv;
    out->xmu_sc_hnc[iv] = shnc * in->rhov[iv] * P.dv;
    out->xmu_gf[iv] = sgf * in->rhov[iv] * P.dv;
    out->sfe_sc += ibeta * out->xmu_sc[iv];
    out->sfe_sc_hnc += ibeta * out->xmu_sc_hnc[iv];
    out->sfe_gf += ibeta * out->xmu_gf[iv];
  }
  double cuv = 0.0;                     // cal_pmv.cu:5-22
  for (int iv = 0; iv < nv; ++iv) {
    const cd *hv = &huv[iv * n];
    const double *tv = &t[iv * n];
    double s = grid_sum(P, [&](size_t i) { return hv[i].real() - tv[i]; });
    cuv += s * in->rhov[iv];
  }
  cuv *= P.dv;
  out->cuv = cuv;
  out->pmv = in->xt * (1.0 - cuv) * ibeta;
  double pres = 0.0;                    // cal_pressure.cu:6-20
  for (int iv = 0; iv < nv; ++iv) pres += in->rhov[iv];
  pres *= 1.0e30 / kAvogadro;
  pres = 0.5 * (pres + 1.0 / (in->xt * ibeta));
  out->pressure = pres;
  out->correction = -pres * out->pmv * ibeta;   // output_xmu.cu:21

  // cal_euv.cu:7-76 and cal_grad.cu:8-145 (per (site, atom) grid sums of g)
  const int na = in->natom;
  const double cc = kHartree * kBohr * kAvogadro;
  std::vector<double> e_loc((size_t)2 * nv * na, 0.0), glj((size_t)na * 3, 0.0),
      ges((size_t)na * 3, 0.0);
  for (int iv = 0; iv < nv; ++iv) {
    const cd *gv = &guv[iv * n];
    for (int iu = 0; iu < na; ++iu) {
      double sig = (in->sig[iu] + in->sigv[iv]) * 0.5;
      double eps = std::sqrt(in->eps[iu] * in->epsv[iv]);
      double qq = in->q[iu] * in->qv[iv];
      double X = in->xyz[3 * iu], Y = in->xyz[3 * iu + 1], Z = in->xyz[3 * iu + 2];
      const long rows = (long)P.ny * P.nz;
      std::vector<double> part((size_t)rows * 8, 0.0);
#pragma omp parallel for schedule(static)
      for (long r = 0; r < rows; ++r) {
        int iy = (int)(r % P.ny), iz = (int)(r / P.ny);
        double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int ix = 0; ix < P.nx; ++ix) {
          size_t ip = (size_t)r * P.nx + ix;
          double dx = P.rx(ix) - X, dy = P.ry(iy) - Y, dz = P.rz(iz) - Z;
          double r2 = dx * dx + dy * dy + dz * dz;
          double r1 = std::sqrt(r2);
          if (r1 < sig * 0.5) continue;
          double g = gv[ip].real();
          double rs2i = sig * sig / r2;
          double rs6i = rs2i * rs2i * rs2i;
          acc[0] += eps * 4.0 * rs6i * (rs6i - 1.0) * g;
          acc[1] += qq / r1 * cc * g;
          double ulj = eps * 24.0 * rs6i / r2 * (2.0 * rs6i - 1.0) * g;
          acc[2] += ulj * dx; acc[3] += ulj * dy; acc[4] += ulj * dz;
          double uco = qq / (r2 * r1) * cc * g;
          acc[5] += uco * dx; acc[6] += uco * dy; acc[7] += uco * dz;
        }
        for (int k = 0; k < 8; ++k) part[(size_t)r * 8 + k] = acc[k];
      }
      double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (long r = 0; r < rows; ++r)
        for (int k = 0; k < 8; ++k) s[k] += part[(size_t)r * 8 + k];
      double rho = in->rhov[iv];
      e_loc[(size_t)na * iv + iu] = s[0] * rho;
      e_loc[(size_t)nv * na + (size_t)na * iv + iu] = s[1] * rho;
      for (int k = 0; k < 3; ++k) {
        glj[(size_t)iu * 3 + k] += s[2 + k] * rho;
        ges[(size_t)iu * 3 + k] += s[5 + k] * rho;
      }
    }
  }
  double slj = 0.0, ses = 0.0;
  for (size_t i = 0; i < (size_t)nv * na; ++i) slj += e_loc[i];
  for (size_t i = (size_t)nv * na; i < (size_t)2 * nv * na; ++i) ses += e_loc[i];
  out->se_lj = slj * P.dv;
  out->se_es = ses * P.dv;
  out->se = (slj + ses) * P.dv;
  if (euv) std::copy(e_loc.begin(), e_loc.end(), euv);
  if (dulj) std::copy(glj.begin(), glj.end(), dulj);
  if (due) std::copy(ges.begin(), ges.end(), due);
  if (g_out)
    for (size_t i = 0; i < (size_t)nv * n; ++i) g_out[i] = guv[i].real();
  if (h_out)
    for (size_t i = 0; i < (size_t)nv * n; ++i) h_out[i] = huv[i].real();
  if (t_out) std::copy(t.begin(), t.end(), t_out);
  if (in->cvv) {                        // output.cu:25
    double dft = 0.0;
    int rc = rmdft(P, fft, indga, ga, huv, &dft);
    if (rc) return rc;
    out->sfe_rmdft = ibeta * dft;
  }
  out->t_obs = omp_get_wtime() - w2;
  return 0;
}
