// Host-side file formats of the reference (read_input.cu, solvent_read.cc,
// solute.cu, output_*.cu, read_tuv.cu / write_tuv.cu).  Readers return an
// error string instead of exiting.
#pragma once

#include <string>
#include <vector>

namespace rism3d {
namespace io {

struct ControlFile {
  std::string outlist;
  int ksave = 0;
  int closure = 0;           // 0 KH, 1 HNC
  std::string fsolvent;
  double conv = 1e-6;
  int maxstep = 10000;
  int count = 2;
  double m = 0.6, mp = 0.2;
  double box[3] = {0, 0, 0};
  int grid[3] = {0, 0, 0};
  std::vector<double> sig, eps, q, xyz;   // xyz[3*natom]
};

struct SolventFile {
  int natv = 0;
  int ntab = 0;
  double dr = 0;
  double temper = 0, xt = 0;
  std::vector<double> rho, q, sig, eps;   // merged site types, rho in 1/A^3
  std::vector<double> xvv;                // [natv][natv][ntab]
};

// read_input.cu:21-89.  `structure` may be empty (atoms follow in control).
bool read_control(const std::string &control, const std::string &structure,
                  ControlFile &out, std::string &err);
// solvent_read.cc:10-86
bool read_xvk(const std::string &path, SolventFile &out, std::string &err);
// solute.cu:13-43: integer shift centring the bounding box; applied to xyz
void centre(std::vector<double> &xyz, double shift[3]);

// output_xmu.cu:7-111
struct XmuValues {
  int natv = 0;
  int closure = 0;
  double sfec_sc[8], sfec_sc_hnc[8], sfec_gf[8];
  double se, se_lj, se_es, pmv_l, pressure, correction;
  bool rmdft = false;        // SFE_RMDFT line first (output_xmu.cu:25-28)
  double sfe_rmdft = 0;
};
bool write_xmu(const std::string &path, const XmuValues &x);
// output_grad.cu:7-30 (values already times dv)
bool write_gra(const std::string &path, int natom, const double *dulj, const double *due);
// output_guv.cu:7-25 (binary)
bool write_guv(const std::string &path, int natv, const int grid[3], const double box[3],
               const double shift[3], const double *g, long long n);
// output_huv.cu / output_cuv.cu (text; solute block as the reference prints it)
bool write_grid_text(const std::string &path, const double box[3], const int grid[3],
                     int natom, const double *q, const double *sig, const double *eps,
                     const double *xyz4, int natv, const double *vals, long long n);
// output_euv.cu:7-31 (values already times dv)
bool write_euv(const std::string &path, int natom, int natv, const double *euv);
// output_qv.cu:7-36
bool write_qv(const std::string &path, const int grid[3], const double dr[3],
              const double *qv_times_dv, long long n);
// cal_Coulomb.cu:41-88: ESP cube (two comment lines; natom, origin and one
// more number; three axis lines whose counts must equal `grid`; natom atom
// lines; values with z fastest).  esp receives [N] values, x fastest, Hartree/e.
bool read_esp_cube(const std::string &path, const int grid[3], std::vector<double> &esp,
                   std::string &err);
// RMDFT hard-sphere table, the -r file (solvent_read.cc:118-140): line 1
// ntab2; line 2 packing fraction and w(0) of site 0; then ntab2 rows
// k, chi_hs(k), w(k)
struct HardSphereFile {
  int ntab2 = 0;
  double pfhs = 0, w0 = 0;
  std::vector<double> k, chs, w;
};
bool read_hard_sphere(const std::string &path, HardSphereFile &out, std::string &err);
// write_tuv.cu:7-33 / read_tuv.cu:6-34
bool write_tuv(const std::string &path, const int grid[3], int natv, const double *t, long long n);
bool read_tuv(const std::string &path, const int grid[3], int natv, std::vector<double> &t,
              std::string &warn);

}  // namespace io
}  // namespace rism3d
