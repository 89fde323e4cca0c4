// Reference file formats, host side (see rism3d_io.h for the citations).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <limits>
#include <sstream>

#include "rism3d_io.h"

namespace rism3d {
namespace io {

static const char *kVersion = "20220301";   // version.h:5
static const double kAvogadro = 6.02214076e23;

static bool natural_number(const std::string &s, int &out) {
  // read_input.cu:8-19: the whole token must parse as a non-negative int
  if (s.empty()) return false;
  char *end = nullptr;
  long v = strtol(s.c_str(), &end, 10);
  if (*end != '\0' || v < 0 || v > 100000000) return false;
  out = (int)v;
  return true;
}

bool read_control(const std::string &control, const std::string &structure,
                  ControlFile &c, std::string &err) {
  std::ifstream in(control.c_str());
  if (!in) { err = "cannot open control file " + control; return false; }
  std::string check, clos;
  if (!(in >> c.outlist >> c.ksave >> check)) { err = "truncated control file"; return false; }
  if (check != kVersion) { err = "This input file is for old version."; return false; }
  in >> clos;
  if (clos == "KH") c.closure = 0;
  else if (clos == "HNC") c.closure = 1;
  else { err = "Unexpected closure switch"; return false; }
  if (!(in >> c.fsolvent >> c.conv >> c.maxstep >> c.count >> c.m >> c.mp >>
        c.box[0] >> c.box[1] >> c.box[2] >> c.grid[0] >> c.grid[1] >> c.grid[2])) {
    err = "truncated control file";
    return false;
  }
  std::ifstream sin;
  std::istream *src = &in;
  if (!structure.empty()) {
    sin.open(structure.c_str());
    if (!sin) { err = "cannot open structure file " + structure; return false; }
    src = &sin;
  }
  std::string tmp;
  int num = 0;
  if (!(*src >> tmp) || !natural_number(tmp, num)) {
    err = "Number of solute atom is not a natural number.";
    return false;
  }
  c.sig.resize(num); c.eps.resize(num); c.q.resize(num); c.xyz.resize(3 * (size_t)num);
  for (int i = 0; i < num; ++i) {
    if (!(*src >> c.sig[i] >> c.eps[i] >> c.q[i] >> c.xyz[3 * i] >> c.xyz[3 * i + 1] >>
          c.xyz[3 * i + 2])) {
      err = "truncated solute atom list";
      return false;
    }
  }
  return true;
}

bool read_xvk(const std::string &path, SolventFile &s, std::string &err) {
  std::ifstream in(path.c_str());
  if (!in) { err = "Solvent file could not be opened!"; return false; }
  std::vector<std::string> lines;
  std::string line;
  while (std::getline(in, line)) lines.push_back(line);
  if (lines.size() < 4) { err = "truncated solvent file"; return false; }
  std::string d;
  int num = 0;
  {
    std::istringstream h1(lines[1]);
    if (!(h1 >> d >> num >> s.natv >> s.ntab >> s.dr)) { err = "bad solvent header"; return false; }
    std::istringstream h2(lines[2]);
    if (!(h2 >> d >> d >> s.temper >> s.xt)) { err = "bad solvent header"; return false; }
  }
  if (s.natv < 1 || s.natv > 8 || num < 1 || s.ntab < 4 || s.dr <= 0) {
    err = "unsupported solvent header";
    return false;
  }
  if ((int)lines.size() < num + 5) { err = "truncated solvent site table"; return false; }
  s.rho.assign(s.natv, 0.0); s.q.assign(s.natv, 0.0);
  s.sig.assign(s.natv, 0.0); s.eps.assign(s.natv, 0.0);
  for (int i = 0; i < num; ++i) {                 // solvent_read.cc:45-50
    std::istringstream a(lines[4 + i]);
    int sym;
    double sg, ep, q, den;
    if (!(a >> d >> d >> d >> sym >> sg >> ep >> q >> d >> d >> d >> den)) {
      err = "bad solvent site line";
      return false;
    }
    int i2 = std::abs(sym) - 1;                   // :71-77 merge by |SYM|
    if (i2 < 0 || i2 >= s.natv) { err = "solvent site SYM out of range"; return false; }
    s.sig[i2] = sg; s.eps[i2] = ep; s.q[i2] = q; s.rho[i2] += den;
  }
  for (int i = 0; i < s.natv; ++i) s.rho[i] *= kAvogadro * 1.0e-27;   // :78-80
  // chi rows start after the separator line that follows the site table
  // (the reader of solvent_read.cc:51-58 consumes the stream from there)
  std::string rest;
  for (size_t l = (size_t)num + 5; l < lines.size(); ++l) { rest += lines[l]; rest += ' '; }
  std::istringstream data(rest);
  const size_t need = (size_t)s.ntab * s.natv * s.natv;
  s.xvv.assign(need, 0.0);
  for (int k = 0; k < s.ntab; ++k)
    for (int a = 0; a < s.natv; ++a)
      for (int b = 0; b < s.natv; ++b) {
        double v;
        if (!(data >> v)) { err = "short chi table in solvent file"; return false; }
        s.xvv[((size_t)a * s.natv + b) * s.ntab + k] = v;
      }
  return true;
}

void centre(std::vector<double> &xyz, double shift[3]) {
  const size_t na = xyz.size() / 3;
  double lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = std::numeric_limits<double>::max();
    hi[d] = std::numeric_limits<double>::lowest();
  }
  for (size_t i = 0; i < na; ++i)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], xyz[3 * i + d]);
      hi[d] = std::max(hi[d], xyz[3 * i + d]);
    }
  for (int d = 0; d < 3; ++d) shift[d] = round(-(hi[d] - lo[d]) / 2 - lo[d]);
  for (size_t i = 0; i < na; ++i)
    for (int d = 0; d < 3; ++d) xyz[3 * i + d] += shift[d];
}

bool write_xmu(const std::string &path, const XmuValues &x) {
  std::ofstream o(path.c_str());
  if (!o) return false;
  o << " $RESULT" << std::endl;
  if (x.rmdft)
    o << "SFE_RMDFT= " << std::fixed << std::setprecision(5) << x.sfe_rmdft << " !(J/mol)"
      << std::endl << std::endl;
  double s = 0;
  for (int v = 0; v < x.natv; ++v) s += x.sfec_sc[v];
  o << "SFE_SC= " << std::fixed << std::setprecision(5) << s << " !(J/mol)" << std::endl;
  for (int v = 0; v < x.natv; ++v) o << "  SFEC_SC(" << v << ")= " << x.sfec_sc[v] << std::endl;
  o << std::endl;
  if (x.closure == 0) {
    s = 0;
    for (int v = 0; v < x.natv; ++v) s += x.sfec_sc_hnc[v];
    o << "SFE_SC_HNC= " << s << " !(J/mol)" << std::endl;
    for (int v = 0; v < x.natv; ++v) o << "  SFEC_SC_HNC(" << v << ")= " << x.sfec_sc_hnc[v] << std::endl;
    o << std::endl;
  }
  s = 0;
  for (int v = 0; v < x.natv; ++v) s += x.sfec_gf[v];
  o << "SFE_GF= " << s << " !(J/mol)" << std::endl;
  for (int v = 0; v < x.natv; ++v) o << "  SFEC_GF(" << v << ")= " << x.sfec_gf[v] << std::endl;
  o << std::endl;
  o << "SE= " << x.se << " !(J/mol)" << std::endl;
  o << "  SE_LJ= " << x.se_lj << std::endl;
  o << "  SE_ES= " << x.se_es << std::endl;
  o << std::endl;
  o << "PMV= " << x.pmv_l << " !(L/mol)" << std::endl;
  o << "Pressure= " << x.pressure << " !(J/m^3)" << std::endl;
  o << "Correction_Term= " << x.correction << " !(J/mol)" << std::endl;
  o << " $END" << std::endl;
  return (bool)o;
}

bool write_gra(const std::string &path, int natom, const double *dulj, const double *due) {
  std::ofstream o(path.c_str());
  if (!o) return false;
  for (int u = 0; u < natom; ++u) {
    o << std::scientific;
    for (int k = 0; k < 3; ++k) o << std::setw(16) << std::setprecision(8) << dulj[3 * u + k] << " ";
    for (int k = 0; k < 3; ++k) {
      o << std::setw(16) << std::setprecision(8) << due[3 * u + k];
      if (k < 2) o << " ";
    }
    o << std::endl;
  }
  return (bool)o;
}

bool write_guv(const std::string &path, int natv, const int grid[3], const double box[3],
               const double shift[3], const double *g, long long n) {
  std::ofstream o(path.c_str(), std::ios::out | std::ios::binary);
  if (!o) return false;
  o.write((const char *)&natv, sizeof(int));
  o.write((const char *)grid, sizeof(int) * 3);
  o.write((const char *)box, sizeof(double) * 3);
  o.write((const char *)shift, sizeof(double) * 3);
  o.write((const char *)g, sizeof(double) * (size_t)natv * n);
  return (bool)o;
}

bool write_grid_text(const std::string &path, const double box[3], const int grid[3],
                     int natom, const double *q, const double *sig, const double *eps,
                     const double *xyz, int natv, const double *vals, long long n) {
  std::ofstream o(path.c_str());
  if (!o) return false;
  o << box[0] << " " << box[1] << " " << box[2] << " " << std::endl
    << grid[0] << " " << grid[1] << " " << grid[2] << " " << std::endl
    << natom << std::endl;
  for (int u = 0; u < natom; ++u)
    o << q[u] << " " << sig[u] << " " << eps[u] << " " << xyz[3 * u] << " "
      << xyz[3 * u + 1] << " " << xyz[3 * u + 2] << std::endl;
  o << natv << std::endl;
  for (long long j = 0; j < n; ++j) {
    for (int v = 0; v < natv; ++v) o << vals[(size_t)v * n + j] << " ";
    o << std::endl;
  }
  return (bool)o;
}

bool write_euv(const std::string &path, int natom, int natv, const double *euv) {
  std::ofstream o(path.c_str());
  if (!o) return false;
  for (int u = 0; u < natom; ++u) {
    for (int v = 0; v < natv; ++v)
      o << std::scientific << std::setw(16) << std::setprecision(8) << euv[(size_t)natom * v + u] << " ";
    for (int v = 0; v < natv; ++v)
      o << std::scientific << std::setw(16) << std::setprecision(8)
        << euv[(size_t)natom * natv + (size_t)natom * v + u] << " ";
    o << std::endl;
  }
  return (bool)o;
}

bool write_qv(const std::string &path, const int grid[3], const double dr[3],
              const double *qv, long long n) {
  std::ofstream o(path.c_str());
  if (!o) return false;
  for (long long ig = 0; ig < n; ++ig) {
    double x = (ig % grid[0] - grid[0] / 2) * dr[0];
    double y = ((ig / grid[0]) % grid[1] - grid[1] / 2) * dr[1];
    double z = (ig / ((long long)grid[0] * grid[1]) - grid[2] / 2) * dr[2];
    o << "    " << std::fixed << std::setw(12) << std::setprecision(4) << x << std::setw(12)
      << std::setprecision(4) << y << std::setw(12) << std::setprecision(4) << z << "  "
      << std::scientific << std::setw(16) << std::setprecision(8) << qv[ig] << std::endl;
  }
  return (bool)o;
}

bool read_esp_cube(const std::string &path, const int grid[3], std::vector<double> &esp,
                   std::string &err) {
  std::ifstream in(path.c_str());
  if (!in) { err = "Error during read esp file: " + path; return false; }
  std::string line;
  std::getline(in, line);
  std::getline(in, line);
  int natom = 0, di = 0;
  double x0, y0, z0;
  if (!(in >> natom >> x0 >> y0 >> z0 >> di)) {
    err = "Error reading atom count and origin.";
    return false;
  }
  int cnt[3];
  double axis[3];
  for (int d = 0; d < 3; ++d)
    if (!(in >> cnt[d] >> axis[0] >> axis[1] >> axis[2])) {
      err = "Error reading the cube axes of " + path;
      return false;
    }
  if (cnt[0] != grid[0] || cnt[1] != grid[1] || cnt[2] != grid[2]) {
    err = "Error. cube file doesn't match input.";
    return false;
  }
  for (int i = 0; i < natom; ++i) {
    int z;
    double a, b, c, d;
    if (!(in >> z >> a >> b >> c >> d)) { err = "Error reading the cube atoms of " + path; return false; }
  }
  const size_t nx = grid[0], ny = grid[1], nz = grid[2];
  esp.assign(nx * ny * nz, 0.0);
  for (size_t ix = 0; ix < nx; ++ix)
    for (size_t iy = 0; iy < ny; ++iy)
      for (size_t iz = 0; iz < nz; ++iz)
        if (!(in >> esp[ix + nx * (iy + ny * iz)])) {
          err = "short ESP cube " + path;
          esp.clear();
          return false;
        }
  return true;
}

bool read_hard_sphere(const std::string &path, HardSphereFile &hs, std::string &err) {
  std::ifstream in(path.c_str());
  if (!in) { err = "Hardsphare file could not be opened!"; return false; }
  std::string line;
  int ntab2 = 0;
  if (!std::getline(in, line) || !(std::istringstream(line) >> ntab2) || ntab2 < 4) {
    err = "bad row count in hard-sphere file " + path;
    return false;
  }
  if (!std::getline(in, line) || !(std::istringstream(line) >> hs.pfhs >> hs.w0)) {
    err = "bad packing fraction line in hard-sphere file " + path;
    return false;
  }
  hs.ntab2 = ntab2;
  hs.k.resize(ntab2);
  hs.chs.resize(ntab2);
  hs.w.resize(ntab2);
  for (int i = 0; i < ntab2; ++i)
    if (!std::getline(in, line) || !(std::istringstream(line) >> hs.k[i] >> hs.chs[i] >> hs.w[i])) {
      err = "short hard-sphere file " + path;
      return false;
    }
  return true;
}

bool write_tuv(const std::string &path, const int grid[3], int natv, const double *t, long long n) {
  std::ofstream o(path.c_str());
  if (!o) return false;
  o << grid[0] << " " << grid[1] << " " << grid[2] << " " << natv << std::endl;
  for (size_t i = 0; i < (size_t)natv * n; ++i) o << t[i] << std::endl;
  return (bool)o;
}

bool read_tuv(const std::string &path, const int grid[3], int natv, std::vector<double> &t,
              std::string &warn) {
  std::ifstream in(path.c_str());
  if (!in) return false;
  int g0, g1, g2, nv;
  if (!(in >> g0 >> g1 >> g2 >> nv)) return false;
  if (g0 != grid[0] || g1 != grid[1] || g2 != grid[2] || nv != natv)
    warn = "restart grid or site count differs from the input (read_tuv.cu:14-20)";
  const size_t n = (size_t)grid[0] * grid[1] * grid[2] * natv;
  t.assign(n, 0.0);
  for (size_t i = 0; i < n; ++i)
    if (!(in >> t[i])) { t.clear(); return false; }
  return true;
}

}  // namespace io
}  // namespace rism3d
