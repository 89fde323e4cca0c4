// rism1d-b200: solvent susceptibility tables (.xvk) from the 1D XRISM (or,
// with -D, DRISM) solve.
//
//   rism1d-b200 [-T kelvin] [-n ntab] [-r dr] [-c KH|HNC] [-e conv] [-D eps [-a smear]] [-v]
//               sites.txt out.xvk
//
// sites.txt: one line per site, "NAME SPC SYM sigma[A] eps[J/mol] q[e] x y z
// density[M]" (the column layout of an .xvk header; lines starting with #
// are skipped).  Defaults: 298.15 K, 4096 points, 0.05 A, KH, 1e-12.
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "rism3d_b200.h"

int main(int argc, char **argv) {
  rism1d_params p{};
  p.temperature = 298.15;
  p.ntab = 4096;
  p.dr = 0.05;
  p.closure = RISM3D_KH;
  p.convergence = 1e-12;
  int opt;
  while ((opt = getopt(argc, argv, "T:n:r:c:e:D:a:v")) != -1) {
    switch (opt) {
      case 'T': p.temperature = atof(optarg); break;
      case 'n': p.ntab = atoi(optarg); break;
      case 'r': p.dr = atof(optarg); break;
      case 'c': p.closure = strcmp(optarg, "HNC") == 0 ? RISM3D_HNC : RISM3D_KH; break;
      case 'e': p.convergence = atof(optarg); break;
      case 'D': p.dielectric = atof(optarg); break;
      case 'a': p.smear = atof(optarg); break;
      case 'v': p.verbose = 1; break;
      default:
        fprintf(stderr, "usage: %s [-T K] [-n ntab] [-r dr] [-c KH|HNC] [-e conv] [-D eps [-a smear]] [-v] sites out.xvk\n", argv[0]);
        return 1;
    }
  }
  if (argc - optind != 2) {
    fprintf(stderr, "usage: %s [-T K] [-n ntab] [-r dr] [-c KH|HNC] [-e conv] [-D eps [-a smear]] [-v] sites out.xvk\n", argv[0]);
    return 1;
  }
  std::ifstream in(argv[optind]);
  if (!in) { fprintf(stderr, "cannot open %s\n", argv[optind]); return 1; }
  std::vector<rism1d_site> sites;
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream ss(line);
    rism1d_site s{};
    std::string name;
    if (!(ss >> name >> s.spc >> s.sym >> s.sigma >> s.epsilon >> s.charge >> s.x >> s.y >> s.z >> s.density)) {
      fprintf(stderr, "bad site line: %s\n", line.c_str());
      return 1;
    }
    strncpy(s.name, name.c_str(), sizeof(s.name) - 1);
    sites.push_back(s);
  }
  int nt = 0;
  for (const rism1d_site &s : sites) nt = std::abs(s.sym) > nt ? std::abs(s.sym) : nt;
  std::vector<double> xvv((size_t)nt * nt * p.ntab);
  double xt = 0;
  int it = 0;
  int rc = rism1d_solve(&p, (int)sites.size(), sites.data(), xvv.data(), &xt, &it);
  if (rc != RISM3D_OK) { fprintf(stderr, "rism1d: %s\n", rism1d_last_error()); return 1; }
  rc = rism1d_write_xvk(argv[optind + 1], &p, (int)sites.size(), sites.data(), xvv.data(), xt);
  if (rc != RISM3D_OK) { fprintf(stderr, "rism1d: %s\n", rism1d_last_error()); return 1; }
  printf("%s: %d steps, chi_T = %.8E 1/Pa\n", argv[optind + 1], it, xt);
  return 0;
}
