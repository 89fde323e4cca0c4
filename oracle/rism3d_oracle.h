/*
 * CPU FP64 restatement of the reference 3D-RISM solve path
 * (rismical-dev/3D-RISM-CUDA, src-cuda/).  TEST INFRASTRUCTURE ONLY: the
 * parity tests, __graft_entry__.smoke() and bench.py's cpu_baseline leg use
 * it as the checker / CPU baseline.  The product never links or calls it.
 *
 * Every routine follows the reference algorithm step for step (same half-
 * shifted k grid, same unique-|k| spline, same AN2 bookkeeping, same
 * integrands); only the FFT is this file's own mixed-radix code because the
 * reference calls cuFFT.
 */
#ifndef RISM3D_ORACLE_H
#define RISM3D_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_MAXV 16

typedef struct {
  /* cell (cell.cc:8-22) */
  int nx, ny, nz;
  double bx, by, bz;
  /* solvent (solvent_read.cc:10-86): merged site types */
  int natv;
  const double *rhov;   /* molecules / A^3 */
  const double *qv;     /* e */
  const double *sigv;   /* A */
  const double *epsv;   /* J/mol */
  double temper;        /* K */
  double xt;            /* isothermal compressibility, 1/Pa */
  int ntab;
  double dr;            /* ttab[i] = (i+1) pi / (dr ntab) */
  const double *xvv;    /* [natv][natv][ntab], row b fastest */
  /* solute (read_input.cu:72-76), coordinates already shifted */
  int natom;
  const double *sig, *eps, *q, *xyz;  /* xyz[3*natom] */
  /* control (read_input.cu:35-47) */
  int closure;          /* 0 KH, 1 HNC */
  double conv;
  int maxstep;
  int count;            /* AN2 Picard warm-up steps */
  double m, mp;         /* AN2 mixing and bias */
  int chargeup;         /* -c stages, 0 = none */
  const double *t_init; /* optional restart t_uv [natv][N] (read_tuv.cu) */
  int verbose;
  const double *esp;    /* optional ESP cube values [N], Hartree/e, x fastest
                           (cal_Coulomb.cu:41-96); replaces the point-charge e */
  /* optional RMDFT correction (cal_rmdft.cu:5-115, solvent_read.cc:88-140,
     solvent_spline2.cu:7-103); cvv NULL = off */
  const double *cvv;    /* [natv][natv][ntab] solvent c(k) on the chi knots (.cvk) */
  int ntab2;            /* rows of the hard-sphere table */
  const double *ttab2, *chs, *wfk;  /* [ntab2]: k, hard-sphere chi(k), weight w(k) */
  double pfhs, wfk0;    /* packing fraction and w(k = 0); site 0 only */
} OracleInput;

typedef struct {
  double xmu_sc[ORACLE_MAXV];     /* rho_v dv sum f  (times N_A kB T = J/mol) */
  double xmu_sc_hnc[ORACLE_MAXV];
  double xmu_gf[ORACLE_MAXV];
  double ibeta;                   /* N_A kB T, J/mol */
  double sfe_sc, sfe_sc_hnc, sfe_gf;   /* J/mol */
  double pmv;                     /* m^3/mol (x1000 = L/mol) */
  double pressure;                /* P/kBT, mol/m^3 */
  double cuv;                     /* sum rho dv int c */
  double se, se_lj, se_es;        /* J/mol */
  double correction;              /* J/mol */
  double rms;
  int iterations;                 /* total over charge-up stages */
  int status;                     /* 0 converged, 1 diverged, 2 maxstep */
  double t_setup, t_iter, t_obs;  /* wall seconds: potentials+chi, loop, output */
  double sfe_rmdft;               /* J/mol, when RMDFT tables are given */
} OracleResult;

/* Full solve + observables.  Optional outputs (may be NULL):
 *   g, h, t : [natv][N] real g (closure), Re h (OZ), t (absolute)
 *   euv     : [2][natv][natom] (LJ then ES), NOT multiplied by dv
 *   dulj, due: [natom][3], NOT multiplied by dv
 *   trace   : rms per step, up to maxstep*(chargeup+1) entries            */
int oracle_solve(const OracleInput *in, OracleResult *out,
                 double *g, double *h, double *t,
                 double *euv, double *dulj, double *due, double *trace);

/* Potential grids only (cal_LJ.cu, cal_Coulomb.cu): u [natv][N] (beta u_LJ),
 * e [N], fr [N], fk [2N] (re, im interleaved), all beta scaled.            */
int oracle_potentials(const OracleInput *in, double *u, double *e,
                      double *fr, double *fk);

/* Half-shifted 3D transform of fft3d.cu on a complex grid [N] (re, im).
 * key = -1 forward (dv dir FFT(dir dkf f)), +1 inverse.                    */
int oracle_fft3d(int nx, int ny, int nz, double bx, double by, double bz,
                 double *a, int key);

/* Unique-|k| interpolated chi (initialize_g.cu + solvent_spline.cu):
 * writes X [natv][natv][N] dense.                                          */
int oracle_chi_grid(const OracleInput *in, double *x);

/* Natural cubic spline of spline.cc / splint.cc on one table. */
int oracle_spline_eval(int np, const double *xp, const double *yp,
                       int nq, const double *xq, double *yq);

int oracle_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
