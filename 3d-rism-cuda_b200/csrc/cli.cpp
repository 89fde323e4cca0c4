// rism3d-b200: drop-in for the reference executable (main.cu:6-64).
// Same flags: -c charge-up stages, -d device, -i control file, -s structure
// file, -r hard-sphere file (RMDFT correction; reads the .cvk beside the
// solvent file too), -e ESP cube (as in the
// reference it also disables centring), -f (no centring; takes an
// argument, getopt "f:"), -z zero solute charges (.xmu0).  Extra: -p 1 runs
// the FP32-bulk + FP64-polish iteration (default 0 = plain FP64).
#include <cstdio>
#include <cstdlib>
#include <string>
#include <unistd.h>

#include "rism3d_b200.h"

int main(int argc, char *argv[]) {
  int ch, cu = 0, dn = 0, prec = 0;
  std::string input, structure, hs, esp;
  bool centering = true, q0 = false;
  while ((ch = getopt(argc, argv, "c:d:i:s:r:e:f:zp:")) != -1) {
    switch (ch) {
      case 'c': cu = atoi(optarg); break;
      case 'd': dn = atoi(optarg); break;
      case 'i': input = optarg; break;
      case 's': structure = optarg; break;
      case 'r': hs = optarg; break;
      case 'e': esp = optarg; /* falls through, as main.cu:37-41 */
      case 'f': centering = false; break;
      case 'z': q0 = true; break;
      case 'p': prec = atoi(optarg); break;
    }
  }
  if (input.empty() || structure.empty()) {
    if (optind >= argc) { printf("No input file!\n"); return 1; }
    if (input.empty()) input = argv[optind];
  }
  printf("Set device %d\n", dn);
  rism3d_ctx *ctx = nullptr;
  int rc = rism3d_initialize(&ctx, input.c_str(), structure.c_str(), esp.c_str(), hs.c_str(),
                             centering ? 1 : 0, q0 ? 1 : 0, dn, prec);
  if (rc != RISM3D_OK) {
    fprintf(stderr, "Error: %s\n", rism3d_last_error(nullptr));
    return 1;
  }
  rc = rism3d_iterate(ctx, cu);
  if (rc != RISM3D_OK && rc != RISM3D_DIVERGED && rc != RISM3D_NOT_CONVERGED) {
    fprintf(stderr, "Error: %s\n", rism3d_last_error(ctx));
    rism3d_destroy(ctx);
    return 1;
  }
  rc = rism3d_output(ctx);
  if (rc != RISM3D_OK) fprintf(stderr, "Error: %s\n", rism3d_last_error(ctx));
  rism3d_destroy(ctx);
  return rc == RISM3D_OK ? 0 : 1;
}
