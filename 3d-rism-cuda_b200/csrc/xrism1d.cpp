// 1D extended RISM (XRISM) for the solvent: the site-site susceptibility
// X_ab(k) = w_ab(k) + rho_b h_ab(k) that the 3D solve reads from a .xvk file
// (solvent_read.cc:31-60).  The reference ships such tables but not the
// program that makes them; this is the library's own solver for them.
//
// Equations (pure solvent, any number of molecular species; sites i, j):
//   H = W C W + W C P H   in k space, per k:  H = (I - W C P)^-1 W C W
// with W the intramolecular matrix w_ij = sin(k l_ij)/(k l_ij) within a
// molecule (1 on the diagonal, 0 between molecules), P = diag(rho_i) the
// molecular density of each site's species, and the KH (or HNC) closure in
// r space.  The Coulomb tail is split as in the 3D code (cal_Coulomb.cu):
// u_L = q_i q_j ubeta (1 - e^-r)/r with the analytic transform
// 4 pi q_i q_j ubeta / (k^2 (k^2 + 1)); the iterated variable is the
// short-range t_s = h - c_s, c_s = c + beta u_L, and the closure sees
// -beta u_s + t_s with u_s = u - u_L.
//
// Grid: r_i = i dr, k_j = j dk, dk = pi / (N dr), i, j = 1 .. N-1, so the
// Fourier-Bessel pair is a type-I sine transform of length N-1:
//   F(k_j) = (4 pi dr / k_j) sum_i r_i f(r_i) sin(pi i j / N)
//   f(r_i) = (dk / (2 pi^2 r_i)) sum_j k_j F(k_j) sin(pi i j / N)
// computed with a radix-2 FFT of length 2N (N a power of two).  The table
// row j = N (k = pi/dr) has sin = 0 at every r_i: h = 0, X = w.
//
// DRISM (p->dielectric > 0; Perkyns and Pettitt, J. Chem. Phys. 97, 7656
// (1992)): the intramolecular matrix becomes W' = W + P chi, where chi
// couples the sites of molecules with a dipole moment mu,
//   chi_ij(k) = z_i(k) hc(k) z_j(k),  z_i = j0(k x_i) j0(k y_i) j1(k z_i),
//   hc(k) = (eps / Y - 3) / (4 pi rho_d) exp(-a^2 k^2 / 4),
//   Y = 4 pi beta sum_s rho_s mu_s^2 / 9,  rho_d = sum_s rho_s,
// with (x, y, z) each site's coordinates from its molecule's |q|-weighted
// centre and the dipole along z.  The equation above is solved for h - chi,
// and the closure and the tables see h.  The DIIS mixing defaults to 0.1
// there: at 0.3 it could settle on a second, unphysical solution (negative
// ion-ion structure at k -> 0).
//
// Iteration: DIIS (Pulay) on t_s with the residual R = t_s' - t_s, depth
// 10, mixing 0.3, falling back to damped Picard steps when the DIIS system
// is ill-conditioned.  Water-like solvents do not converge from t = 0 at
// full charge, so the charges are switched on along a continuation path
// lambda = 0 .. 1 (step 0.1, halved after a failed step, each intermediate
// state converged to 1e-6), and the last state to rms(R) <= conv (default
// 1e-12).
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "rism3d_b200.h"

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kAvogadro = 6.02214076e23;
constexpr double kBoltzmann = 1.380649e-23;
constexpr double kBohr = 0.5291771500001;
constexpr double kHartree = 4.359744722207185e-18;

std::string g_err1d;

// In-place radix-2 complex FFT (forward sign -1), n a power of two.
void fft(std::vector<std::complex<double>> &a, const std::vector<std::complex<double>> &tw) {
  const size_t n = a.size();
  for (size_t i = 1, j = 0; i < n; ++i) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    const size_t step = n / len;
    for (size_t i = 0; i < n; i += len)
      for (size_t k = 0; k < len / 2; ++k) {
        const std::complex<double> w = tw[k * step];
        const std::complex<double> u = a[i + k], v = a[i + k + len / 2] * w;
        a[i + k] = u + v;
        a[i + k + len / 2] = u - v;
      }
  }
}

// Type-I sine transform S_j = sum_{i=1}^{N-1} f_i sin(pi i j / N), j = 1..N-1
// (f and S indexed from 0 for i = 1), via the odd extension of length 2N.
struct Dst {
  int N;
  std::vector<std::complex<double>> tw, buf;
  explicit Dst(int n) : N(n), tw(n), buf(2 * (size_t)n) {
    for (int k = 0; k < n; ++k) tw[k] = std::polar(1.0, -kPi * k / n);
  }
  void run(const double *f, double *S) {
    const int n2 = 2 * N;
    buf[0] = 0.0;
    buf[N] = 0.0;
    for (int i = 1; i < N; ++i) {
      buf[i] = f[i - 1];
      buf[n2 - i] = -f[i - 1];
    }
    fft(buf, tw);
    // FFT of the odd sequence: Y_j = -2 i sum f_i sin(pi i j / N)
    for (int j = 1; j < N; ++j) S[j - 1] = -0.5 * buf[j].imag();
  }
};

// Small dense solve A X = B (n x n, m right-hand sides), partial pivoting.
bool solve_dense(int n, std::vector<double> &A, std::vector<double> &B, int m) {
  for (int c = 0; c < n; ++c) {
    int p = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(A[(size_t)r * n + c]) > std::fabs(A[(size_t)p * n + c])) p = r;
    if (std::fabs(A[(size_t)p * n + c]) < 1e-300) return false;
    if (p != c) {
      for (int k = 0; k < n; ++k) std::swap(A[(size_t)c * n + k], A[(size_t)p * n + k]);
      for (int k = 0; k < m; ++k) std::swap(B[(size_t)c * m + k], B[(size_t)p * m + k]);
    }
    const double d = A[(size_t)c * n + c];
    for (int r = c + 1; r < n; ++r) {
      const double f = A[(size_t)r * n + c] / d;
      if (f == 0.0) continue;
      for (int k = c; k < n; ++k) A[(size_t)r * n + k] -= f * A[(size_t)c * n + k];
      for (int k = 0; k < m; ++k) B[(size_t)r * m + k] -= f * B[(size_t)c * m + k];
    }
  }
  for (int r = n - 1; r >= 0; --r)
    for (int k = 0; k < m; ++k) {
      double s = B[(size_t)r * m + k];
      for (int c = r + 1; c < n; ++c) s -= A[(size_t)r * n + c] * B[(size_t)c * m + k];
      B[(size_t)r * m + k] = s / A[(size_t)r * n + r];
    }
  return true;
}

struct System {
  int ns = 0, ntype = 0, N = 0;
  double dr = 0, dk = 0, T = 0;
  int closure = 0;
  std::vector<int> spc, type;            // species index, type (|SYM| - 1)
  std::vector<double> sig, eps, q, x, y, z, rho;   // rho: molecules / A^3
  std::vector<int> rep;                  // first site of each type
  int npair = 0;
  std::vector<int> pi, pj;               // pair list i <= j
  std::vector<double> ulj, ues, uL_k, w; // [pair][r] x2, [pair][k] x2
  std::vector<double> us, uLl;           // the potential at the current lambda
  std::vector<double> chi;               // DRISM bridge [pair][k] (empty: XRISM)
};

int pair_index(const System &s, int i, int j) {
  if (i > j) std::swap(i, j);
  // pairs ordered (0,0) (0,1) .. (0,n-1) (1,1) ..
  return i * s.ns - i * (i - 1) / 2 + (j - i);
}

}  // namespace

extern "C" {

int rism1d_solve(const rism1d_params *p, int nsite, const rism1d_site *sites, double *xvv,
                 double *xt_out, int *iterations) {
  g_err1d.clear();
  if (!p || !sites || nsite < 1 || nsite > 64) { g_err1d = "bad arguments"; return RISM3D_BAD_INPUT; }
  const int N = p->ntab;
  if (N < 16 || (N & (N - 1)) != 0) { g_err1d = "ntab must be a power of two >= 16"; return RISM3D_UNSUPPORTED_SHAPE; }
  if (!(p->dr > 0) || !(p->temperature > 0)) { g_err1d = "dr and temperature must be positive"; return RISM3D_BAD_INPUT; }
  System s;
  s.ns = nsite; s.N = N; s.dr = p->dr; s.dk = kPi / (p->dr * N); s.T = p->temperature;
  s.closure = p->closure;
  int maxtype = 0;
  for (int i = 0; i < nsite; ++i) {
    const rism1d_site &t = sites[i];
    if (t.sym == 0 || t.spc < 1 || !(t.density > 0) || !(t.sigma >= 0) || !(t.epsilon >= 0)) {
      g_err1d = "site " + std::to_string(i) + ": bad species, type, density or LJ parameters";
      return RISM3D_BAD_INPUT;
    }
    s.spc.push_back(t.spc);
    s.type.push_back(std::abs(t.sym) - 1);
    maxtype = std::max(maxtype, std::abs(t.sym));
    s.sig.push_back(t.sigma); s.eps.push_back(t.epsilon); s.q.push_back(t.charge);
    s.x.push_back(t.x); s.y.push_back(t.y); s.z.push_back(t.z);
    s.rho.push_back(t.density * kAvogadro * 1.0e-27);
  }
  s.ntype = maxtype;
  s.rep.assign(s.ntype, -1);
  for (int i = 0; i < nsite; ++i)
    if (s.rep[s.type[i]] < 0) s.rep[s.type[i]] = i;
  for (int a = 0; a < s.ntype; ++a)
    if (s.rep[a] < 0) { g_err1d = "site types must be numbered 1..ntype"; return RISM3D_BAD_INPUT; }
  const int ns = nsite, M = N - 1;
  for (int i = 0; i < ns; ++i)
    for (int j = i; j < ns; ++j) { s.pi.push_back(i); s.pj.push_back(j); }
  s.npair = (int)s.pi.size();
  const double beta_lj = 1.0 / (kAvogadro * kBoltzmann * s.T);       // LJ in J/mol
  const double ubeta = kHartree * kBohr / (kBoltzmann * s.T);         // e^2/A -> kT
  std::vector<double> r(M), k(M);
  for (int i = 0; i < M; ++i) { r[i] = (i + 1) * s.dr; k[i] = (i + 1) * s.dk; }
  // short-range potential, analytic long-range transform, intramolecular w
  s.ulj.assign((size_t)s.npair * M, 0.0);
  s.ues.assign((size_t)s.npair * M, 0.0);
  s.uL_k.assign((size_t)s.npair * M, 0.0);
  s.w.assign((size_t)s.npair * M, 0.0);
  for (int pp = 0; pp < s.npair; ++pp) {
    const int i = s.pi[pp], j = s.pj[pp];
    const double sg = 0.5 * (s.sig[i] + s.sig[j]), ep = std::sqrt(s.eps[i] * s.eps[j]);
    const double qq = s.q[i] * s.q[j] * ubeta;
    const double dx = s.x[i] - s.x[j], dy = s.y[i] - s.y[j], dz = s.z[i] - s.z[j];
    const double l = std::sqrt(dx * dx + dy * dy + dz * dz);
    for (int m = 0; m < M; ++m) {
      const double sr2 = sg * sg / (r[m] * r[m]), sr6 = sr2 * sr2 * sr2;
      s.ulj[(size_t)pp * M + m] = 4.0 * ep * beta_lj * sr6 * (sr6 - 1.0);
      s.ues[(size_t)pp * M + m] = qq * std::exp(-r[m]) / r[m];
      s.uL_k[(size_t)pp * M + m] = qq * 4.0 * kPi / (k[m] * k[m] * (k[m] * k[m] + 1.0));
      double wv = 0.0;
      if (i == j) wv = 1.0;
      else if (s.spc[i] == s.spc[j]) wv = l > 0 ? std::sin(k[m] * l) / (k[m] * l) : 1.0;
      s.w[(size_t)pp * M + m] = wv;
    }
  }
  if (p->dielectric > 0) {
    // dipolar molecules: centre, dipole along z, and the bridge's strength
    const int nspc = *std::max_element(s.spc.begin(), s.spc.end());
    std::vector<double> cx(ns), cy(ns), cz(ns);
    std::vector<char> dip(ns, 0);
    double rhod = 0.0, rmu2 = 0.0;
    for (int sp = 1; sp <= nspc; ++sp) {
      double wx = 0, wy = 0, wz = 0, wt = 0, mx = 0, my = 0, mz = 0, rho_s = 0;
      for (int i = 0; i < ns; ++i) {
        if (s.spc[i] != sp) continue;
        const double wq = std::fabs(s.q[i]);
        wx += wq * s.x[i]; wy += wq * s.y[i]; wz += wq * s.z[i]; wt += wq;
        mx += s.q[i] * s.x[i]; my += s.q[i] * s.y[i]; mz += s.q[i] * s.z[i];
        rho_s = s.rho[i];
      }
      const double mu2 = mx * mx + my * my + mz * mz;
      if (!(mu2 > 1e-12)) continue;
      if (mx * mx + my * my > 1e-12 * mu2) {
        g_err1d = "DRISM: the dipole of species " + std::to_string(sp) + " is not along z";
        return RISM3D_BAD_INPUT;
      }
      const double sg = mz > 0 ? 1.0 : -1.0;
      for (int i = 0; i < ns; ++i) {
        if (s.spc[i] != sp) continue;
        cx[i] = s.x[i] - wx / wt; cy[i] = s.y[i] - wy / wt; cz[i] = sg * (s.z[i] - wz / wt);
        dip[i] = 1;
      }
      rhod += rho_s;
      rmu2 += rho_s * mu2;
    }
    if (rhod > 0) {
      const double yd = 4.0 * kPi * ubeta * rmu2 / 9.0;
      const double hc0 = (p->dielectric / yd - 3.0) / (4.0 * kPi * rhod);
      const double a = p->smear > 0 ? p->smear : 2.0;
      auto j0 = [](double x) { return std::fabs(x) < 1e-8 ? 1.0 : std::sin(x) / x; };
      auto j1 = [](double x) {
        return std::fabs(x) < 1e-4 ? x / 3.0 : std::sin(x) / (x * x) - std::cos(x) / x;
      };
      s.chi.assign((size_t)s.npair * M, 0.0);
      for (int pp = 0; pp < s.npair; ++pp) {
        const int i = s.pi[pp], j = s.pj[pp];
        if (!dip[i] || !dip[j]) continue;
        for (int m = 0; m < M; ++m) {
          const double kk = k[m];
          const double zi = j0(kk * cx[i]) * j0(kk * cy[i]) * j1(kk * cz[i]);
          const double zj = j0(kk * cx[j]) * j0(kk * cy[j]) * j1(kk * cz[j]);
          s.chi[(size_t)pp * M + m] = zi * zj * hc0 * std::exp(-a * a * kk * kk / 4.0);
        }
      }
    }
  }
  Dst dst(N);
  const size_t L = (size_t)s.npair * M;
  std::vector<double> ts(L, 0.0), cs(L), Ck(L), Tk(L), tn(L), Hk(L), tmp(M), tmp2(M);
  const double cf_r = 4.0 * kPi * s.dr, cf_k = s.dk / (2.0 * kPi * kPi);
  // one RISM cycle: t_s -> t_s'
  auto cycle = [&](const std::vector<double> &t_in, std::vector<double> &t_out, bool keep_h) {
    for (int pp = 0; pp < s.npair; ++pp) {
      const double *t = &t_in[(size_t)pp * M];
      const double *u = &s.us[(size_t)pp * M];
      double *c = &cs[(size_t)pp * M];
      for (int m = 0; m < M; ++m) {
        const double d = -u[m] + t[m];
        const double g = (s.closure == 0 && d > 0.0) ? 1.0 + d : std::exp(d);
        c[m] = g - 1.0 - t[m];
        tmp[m] = r[m] * c[m];
      }
      dst.run(tmp.data(), tmp2.data());
      double *C = &Ck[(size_t)pp * M];
      for (int m = 0; m < M; ++m) C[m] = cf_r * tmp2[m] / k[m];
    }
    // k space: H = (I - W C P)^-1 W C W, per k
    std::vector<double> Wm((size_t)ns * ns), Cm((size_t)ns * ns), A((size_t)ns * ns),
        B((size_t)ns * ns), WC((size_t)ns * ns);
    for (int m = 0; m < M; ++m) {
      for (int pp = 0; pp < s.npair; ++pp) {
        const int i = s.pi[pp], j = s.pj[pp];
        const double wv = s.w[(size_t)pp * M + m];
        const double xb = s.chi.empty() ? 0.0 : s.chi[(size_t)pp * M + m];
        const double cv = Ck[(size_t)pp * M + m] - s.uLl[(size_t)pp * M + m];
        Wm[(size_t)i * ns + j] = wv + s.rho[i] * xb;     // W' = W + P chi
        Wm[(size_t)j * ns + i] = wv + s.rho[j] * xb;
        Cm[(size_t)i * ns + j] = Cm[(size_t)j * ns + i] = cv;
      }
      for (int i = 0; i < ns; ++i)
        for (int j = 0; j < ns; ++j) {
          double a = 0.0;
          for (int l = 0; l < ns; ++l) a += Wm[(size_t)i * ns + l] * Cm[(size_t)l * ns + j];
          WC[(size_t)i * ns + j] = a;
        }
      for (int i = 0; i < ns; ++i)
        for (int j = 0; j < ns; ++j) {
          A[(size_t)i * ns + j] = (i == j ? 1.0 : 0.0) - WC[(size_t)i * ns + j] * s.rho[j];
          double b = 0.0;
          for (int l = 0; l < ns; ++l) b += WC[(size_t)i * ns + l] * Wm[(size_t)l * ns + j];
          B[(size_t)i * ns + j] = b;
        }
      if (!solve_dense(ns, A, B, ns)) return false;
      for (int pp = 0; pp < s.npair; ++pp) {
        const int i = s.pi[pp], j = s.pj[pp];
        const double h = 0.5 * (B[(size_t)i * ns + j] + B[(size_t)j * ns + i]) +
                         (s.chi.empty() ? 0.0 : s.chi[(size_t)pp * M + m]);
        if (keep_h) Hk[(size_t)pp * M + m] = h;
        Tk[(size_t)pp * M + m] = h - Ck[(size_t)pp * M + m];
      }
    }
    for (int pp = 0; pp < s.npair; ++pp) {
      const double *T = &Tk[(size_t)pp * M];
      for (int m = 0; m < M; ++m) tmp[m] = k[m] * T[m];
      dst.run(tmp.data(), tmp2.data());
      double *t = &t_out[(size_t)pp * M];
      for (int m = 0; m < M; ++m) t[m] = cf_k * tmp2[m] / r[m];
    }
    return true;
  };
  // DIIS at charge scale lambda from the current t_s
  const int depth = 10;
  const double mix = p->mixing > 0 ? p->mixing : (s.chi.empty() ? 0.3 : 0.1);
  const double conv = p->convergence > 0 ? p->convergence : 1e-12;
  const int maxit = p->maxstep > 0 ? p->maxstep : 10000;
  int it_total = 0;
  auto relax = [&](double lam, double tol, int limit, double &rms) -> int {
    s.us.resize(L);
    s.uLl.resize(L);
    for (size_t f = 0; f < L; ++f) { s.us[f] = s.ulj[f] + lam * s.ues[f]; s.uLl[f] = lam * s.uL_k[f]; }
    std::vector<std::vector<double>> hx, hr;
    rms = 0.0;
    for (int it = 0; it < limit; ++it) {
      ++it_total;
      if (!cycle(ts, tn, false)) return RISM3D_DIVERGED;
      std::vector<double> R(L);
      double ss = 0.0;
      for (size_t f = 0; f < L; ++f) { R[f] = tn[f] - ts[f]; ss += R[f] * R[f]; }
      rms = std::sqrt(ss / (double)L);
      if (!std::isfinite(rms) || rms > 1e3) return RISM3D_DIVERGED;
      if (p->verbose) printf(" 1D lambda %.4f step %d rms %.3e\n", lam, it + 1, rms);
      if (rms <= tol) return RISM3D_OK;
      hx.push_back(ts);
      hr.push_back(R);
      if ((int)hx.size() > depth) { hx.erase(hx.begin()); hr.erase(hr.begin()); }
      const int m = (int)hx.size();
      std::vector<double> A((size_t)(m + 1) * (m + 1), 0.0), b(m + 1, 0.0);
      for (int a = 0; a < m; ++a)
        for (int c = 0; c <= a; ++c) {
          double d = 0.0;
          for (size_t f = 0; f < L; ++f) d += hr[a][f] * hr[c][f];
          A[(size_t)a * (m + 1) + c] = A[(size_t)c * (m + 1) + a] = d;
        }
      double sc = 0.0;
      for (int a = 0; a < m; ++a) sc = std::max(sc, A[(size_t)a * (m + 1) + a]);
      for (int a = 0; a < m; ++a) {
        for (int c = 0; c < m; ++c) A[(size_t)a * (m + 1) + c] /= sc;
        A[(size_t)a * (m + 1) + m] = A[(size_t)m * (m + 1) + a] = -1.0;
      }
      b[m] = -1.0;
      bool ok = solve_dense(m + 1, A, b, 1);
      if (ok)
        for (int a = 0; a < m; ++a) ok = ok && std::isfinite(b[a]);
      if (ok) {
        for (size_t f = 0; f < L; ++f) {
          double v = 0.0;
          for (int a = 0; a < m; ++a) v += b[a] * (hx[a][f] + mix * hr[a][f]);
          ts[f] = v;
        }
      } else {                               // damped Picard step, fresh history
        for (size_t f = 0; f < L; ++f) ts[f] += mix * R[f];
        hx.clear();
        hr.clear();
      }
    }
    return RISM3D_NOT_CONVERGED;
  };
  // continuation in the charges
  double lam = 0.0, step = 0.1, rms = 0.0;
  std::vector<double> good = ts;
  int rc = relax(0.0, 1e-6, 2000, rms);
  if (rc != RISM3D_OK) { g_err1d = "1D iteration failed without charges"; return rc; }
  good = ts;
  while (lam < 1.0) {
    const double next = std::min(1.0, lam + step);
    rc = relax(next, next < 1.0 ? 1e-6 : conv, next < 1.0 ? 500 : maxit, rms);
    if (rc == RISM3D_OK) {
      lam = next;
      good = ts;
      step = std::min(0.2, step * 1.5);
    } else {
      if (next >= 1.0 && rc == RISM3D_NOT_CONVERGED && step < 1e-3) break;
      ts = good;
      step *= 0.5;
      if (step < 1e-4) break;
    }
    if (it_total > 20 * maxit) break;
  }
  if (iterations) *iterations = it_total;
  if (lam < 1.0 || rms > conv) { g_err1d = "1D iteration did not converge"; return RISM3D_NOT_CONVERGED; }
  // final cycle for h(k); X_ab(k) = sum over sites j of type b of
  // (w_ij + rho_j h_ij) with i the first site of type a
  cycle(ts, tn, true);
  // A physical solution has a positive-definite structure-factor matrix of
  // the species at the smallest k, S_mn = d_mn + sqrt(rho_m rho_n) h_mn
  // (first sites).  The equations for a salt solution also have solutions
  // with a negative concentration structure factor (plain XRISM always
  // lands there; DRISM can, depending on the iteration path): refused.
  {
    std::vector<int> first;
    for (int i = 0; i < ns; ++i) {
      bool seen = false;
      for (int f : first) seen = seen || s.spc[f] == s.spc[i];
      if (!seen) first.push_back(i);
    }
    const int ms = (int)first.size();
    std::vector<double> S((size_t)ms * ms);
    for (int a = 0; a < ms; ++a)
      for (int c = 0; c < ms; ++c) {
        const int pp = pair_index(s, first[a], first[c]);
        S[(size_t)a * ms + c] = (a == c ? 1.0 : 0.0) +
                                std::sqrt(s.rho[first[a]] * s.rho[first[c]]) * Hk[(size_t)pp * M];
      }
    for (int a = 0; a < ms; ++a) {                 // Cholesky: every pivot positive
      for (int c = 0; c < a; ++c) S[(size_t)a * ms + a] -= S[(size_t)a * ms + c] * S[(size_t)a * ms + c];
      const double d = S[(size_t)a * ms + a];
      if (!(d > 0.0)) {
        g_err1d = "the 1D solution is unphysical: the species structure factor at k -> 0 "
                  "is not positive definite (for a salt solution use DRISM, dielectric > 0)";
        return RISM3D_NOT_CONVERGED;
      }
      S[(size_t)a * ms + a] = std::sqrt(d);
      for (int b = a + 1; b < ms; ++b) {
        double v = S[(size_t)b * ms + a];
        for (int c = 0; c < a; ++c) v -= S[(size_t)b * ms + c] * S[(size_t)a * ms + c];
        S[(size_t)b * ms + a] = v / S[(size_t)a * ms + a];
      }
    }
  }
  const int nt = s.ntype;
  if (xvv) {
    for (int a = 0; a < nt; ++a)
      for (int b2 = 0; b2 < nt; ++b2)
        for (int m = 0; m < N; ++m) xvv[((size_t)a * nt + b2) * N + m] = 0.0;
    for (int a = 0; a < nt; ++a) {
      const int i = s.rep[a];
      for (int j = 0; j < ns; ++j) {
        const int b2 = s.type[j];
        const int pp = pair_index(s, i, j);
        double *X = &xvv[((size_t)a * nt + b2) * N];
        for (int m = 0; m < M; ++m)
          X[m] += s.w[(size_t)pp * M + m] + s.rho[j] * Hk[(size_t)pp * M + m];
        // k = pi / dr: every sin(k r_i) vanishes, h = 0
        const double kN = N * s.dk;
        double wv = 0.0;
        if (i == j) wv = 1.0;
        else if (s.spc[i] == s.spc[j]) {
          const double dx = s.x[i] - s.x[j], dy = s.y[i] - s.y[j], dz = s.z[i] - s.z[j];
          const double l = std::sqrt(dx * dx + dy * dy + dz * dz);
          wv = l > 0 ? std::sin(kN * l) / (kN * l) : 1.0;
        }
        X[M] += wv;
      }
    }
  }
  // isothermal compressibility from the k -> 0 structure (Kirkwood-Buff):
  // kT chi_T = 1 / sum_mn rho_m rho_n (A^-1)_mn, A_mn = rho_m d_mn +
  // rho_m rho_n h_mn(k=0), h_mn(0) = 4 pi int r^2 h(r) dr between the
  // first sites of species m and n
  if (xt_out) {
    std::vector<int> first;
    std::vector<double> rs;
    for (int i = 0; i < ns; ++i) {
      bool seen = false;
      for (int f : first) seen = seen || s.spc[f] == s.spc[i];
      if (!seen) { first.push_back(i); rs.push_back(s.rho[i]); }
    }
    const int ms = (int)first.size();
    // h(r) of the converged state: inverse transform of H
    std::vector<double> Am((size_t)ms * ms), Bm((size_t)ms * ms, 0.0);
    for (int a = 0; a < ms; ++a)
      for (int c = 0; c < ms; ++c) {
        const int pp = pair_index(s, first[a], first[c]);
        const double *H = &Hk[(size_t)pp * M];
        for (int m = 0; m < M; ++m) tmp[m] = k[m] * H[m];
        dst.run(tmp.data(), tmp2.data());
        double h0 = 0.0;
        for (int m = 0; m < M; ++m) h0 += r[m] * r[m] * (cf_k * tmp2[m] / r[m]);
        h0 *= 4.0 * kPi * s.dr;
        Am[(size_t)a * ms + c] = (a == c ? rs[a] : 0.0) + rs[a] * rs[c] * h0;
        Bm[(size_t)a * ms + c] = a == c ? 1.0 : 0.0;
      }
    if (!solve_dense(ms, Am, Bm, ms)) { g_err1d = "singular k = 0 structure"; return RISM3D_DIVERGED; }
    double sum = 0.0;
    for (int a = 0; a < ms; ++a)
      for (int c = 0; c < ms; ++c) sum += rs[a] * rs[c] * Bm[(size_t)a * ms + c];
    const double kTchi = 1.0 / sum;                           // A^3
    *xt_out = kTchi * 1.0e-30 / (kBoltzmann * s.T);           // 1/Pa
  }
  return RISM3D_OK;
}

int rism1d_write_xvk(const char *path, const rism1d_params *p, int nsite,
                     const rism1d_site *sites, const double *xvv, double xt) {
  g_err1d.clear();
  if (!path || !p || !sites || !xvv || nsite < 1) { g_err1d = "bad arguments"; return RISM3D_BAD_INPUT; }
  int nt = 0;
  for (int i = 0; i < nsite; ++i) nt = std::max(nt, std::abs(sites[i].sym));
  int nspc = 0;
  for (int i = 0; i < nsite; ++i) nspc = std::max(nspc, sites[i].spc);
  FILE *f = fopen(path, "w");
  if (!f) { g_err1d = std::string("cannot write ") + path; return RISM3D_BAD_INPUT; }
  const int N = p->ntab;
  fprintf(f, "##  reduced xvv(k) data with solvent parameters\n");
  fprintf(f, "## %9d %7d %7d %15.8f %15.8f\n", nsite, nt, N, p->dr, kPi / (p->dr * N));
  fprintf(f, "## %4d %16.8f %15.8E\n", nspc, p->temperature, xt);
  fprintf(f, "## ATOM SPC SYM sig[Angs]   eps[J/mol]  charge[e]    ---X---     ---Y---     ---Z---    density[M] \n");
  for (int i = 0; i < nsite; ++i) {
    const rism1d_site &t = sites[i];
    fprintf(f, "## %-4s %3d %3d %11.5f %11.5f %11.5f %11.5f %11.5f %11.5f %11.5f\n",
            t.name[0] ? t.name : "X", t.spc, t.sym, t.sigma, t.epsilon, t.charge, t.x, t.y, t.z,
            t.density);
  }
  fprintf(f, "##\n");
  for (int m = 0; m < N; ++m) {
    for (int a = 0; a < nt; ++a)         // row order read by solvent_read.cc:50-55
      for (int b = 0; b < nt; ++b)
        fprintf(f, " %.15E", xvv[((size_t)a * nt + b) * N + m]);
    fprintf(f, "\n");
  }
  fclose(f);
  return RISM3D_OK;
}

const char *rism1d_last_error(void) { return g_err1d.c_str(); }

}  // extern "C"
