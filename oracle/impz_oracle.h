/*
 * impz_oracle.h -- CPU restatement of IMPACT-Z's per-step space-charge kick
 * and element push (Flagmap=1 map integrator, Flagbc=1 open boundaries,
 * one rank).  TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check and
 * the timed CPU baseline link this library as the checker.  The product
 * library never links it.
 *
 * PARITY UNPINNED: the reference is Fortran90 and no Fortran compiler is
 * available where this was written, and the reference ships no golden
 * outputs.  Every routine is restated line by line from the cited Fortran
 * (paths relative to the IMPACT-Z source tree) and pinned instead by
 * known-answer tests (analytic drift/quad matrices, brute-force convolution,
 * charge conservation, analytic moments).
 *
 * Data layout follows the reference: particle array Pts1(9,N) column-major,
 * i.e. pts[9*i + c] holds coordinate c (0-based) of particle i:
 *   x/Scxl, gamma*beta_x, y/Scxl, gamma*beta_y, phase[rad], gamma0-gamma,
 *   q/m, charge weight, id.                    (src/Appl/BeamBunch.f90:9-12)
 * 6x6 maps are column-major like the Fortran xm(6,6): xm[(j-1)+6*(k-1)] = xm(j,k).
 * Grids are column-major (nx,ny,nz): g[i + nx*(j + ny*k)].
 */
#ifndef IMPZ_ORACLE_H
#define IMPZ_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

#define ORC_DIAG_LEN 45   /* one row of fort.18/24/25/26/27/28/29/30, see orc_diagnostic1 */
#define ORC_RAW_LEN  44   /* 37 moment sums, 6 |max|, 1 max r^2 */

/* PhysConst (src/DataStruct/PhysConst.f90:25-35) */
void orc_physconst(double freq);
void orc_get_physconst(double out[5]); /* Pi, Clight, Scxl, Rad2deg, Scfreq */

/* OpenMP threads used by the particle loops (1 = sequential, bit-exact order) */
void orc_set_threads(int n);
/* per-step capture of orc_run's map-integrator space-charge steps: the
 * potential into phi[s*G..] and kick1's Ex,Ey,Ez into eg[3*s*G..] for
 * s < maxsteps (either may be NULL); resets the step counter */
void orc_set_field_probe(double *phi, double *eg, int maxsteps);
/* charge states of orc_run: nptlist[nchrg] (idchgold, updated by
 * chgupdate_BeamBunch after every conv1st) is copied to out[nchrg*r..]
 * at every record r < maxrows (fort.32); qmcclist NULL switches it off */
void orc_set_charge_states(const double *qmcclist, int nchrg, int *nptlist, int *out,
                           int maxrows);

/* ---- element maps ---------------------------------------------------- */
/* drift1_BeamBunch bitype 0 (BeamBunch.f90:276-298) */
void orc_drift_exact(double *pts, int n, double refptcl[6], double tau);
/* maplinear_Quadrupole + rk6i + intfunc1 (Quadrupole.f90:120-305) */
void orc_maplinear_quad(double t, double tau, double xm[36], double refpt[6],
                        double gradient, int mapstp, double chg, double mass);
/* maplinear_DriftTube (DriftTube.f90:113-288) */
void orc_maplinear_drift(double t, double tau, double xm[36], double refpt[6],
                         int mapstp, double chg, double mass);
/* maplinear_CCL with on-axis table (CCL.f90:122-365); zdat shifted to start at 0 */
void orc_maplinear_solrf(double t, double tau, double xm[36], double refpt[6], double zedge,
                         double escale, double freq, double phase_deg, int mapstp, double chg,
                         double mass, double length, double b0, int ncoef, const double *coef);
void orc_maplinear_tws(double t, double tau, double xm[36], double refpt[6], double zedge,
                       double escale, double freq, double phase_deg, int mapstp, double chg,
                       double mass, double length, double phase2_deg, int ncoef,
                       const double *coef);
void orc_maplinear_quad_fringe(double t, double tau, double xm[36], double refpt[6],
                               double zedge, int mapstp, double chg, double mass, int ndata,
                               const double *zdat, const double *gdat);
void orc_undulator(double tau, double kqlh, double refpt[6], double *pts, int n);
void orc_maplinear_constfoc(double t, double tau, double xm[36], double refpt[6],
                            const double k2[3], int mapstp);
void orc_maplinear_sol(double t, double tau, double xm[36], double refpt[6], double b0,
                       int mapstp, double chg, double mass);
void orc_maplinear_dtl(double t, double tau, double xm[36], double refpt[6],
                       double zedge, double escale, double freq, double phase_deg,
                       int mapstp, double chg, double mass,
                       int ndata, const double *zdat, const double *edat,
                       const double *epdat, const double *eppdat, double length,
                       double q1len, double q1grad, double q2len, double q2grad);
void orc_maplinear_ccl(double t, double tau, double xm[36], double refpt[6],
                       double zedge, double escale, double freq, double phase_deg,
                       int mapstp, double chg, double mass,
                       int ndata, const double *zdat, const double *edat,
                       const double *epdat, const double *eppdat);
/* the 6x6 loop of drift1_BeamBunch (BeamBunch.f90:310-320) */
void orc_apply_xm(double *pts, int n, const double xm[36]);
/* transfmapK_Quadrupole (Quadrupole.f90:509-607) */
void orc_transfmapK(double tau, double kquad, double refpt[6], double *pts, int n,
                    double qmass);
/* ideal RF branch of drift1_BeamBunch (BeamBunch.f90:324-440);
 * params = Param(2..6) of the gap: gradient[V/m], freq, phase[deg], fileid<0, radius */
void orc_ideal_rf(double *pts, int n, double refptcl[6], double mass, double tau,
                  double vgrad, double rffreq, double phase_deg, int nst, int nseg,
                  int ihlf);
/* Dipole maps (Dipole.f90:466-526, 528-591, 693-788) */
void orc_fpol(double h0, double h1, double tanphi, double tanphib, double k1,
              double psi, double *pts, double ang, int n, double gam0, double qm0);
void orc_bpol(double h0, double h1, double tanphi, double tanphib, double k1,
              double psi, double *pts, double ang, int n, double gam0, double qm0);
void orc_sector(double len, double beta0, double h0, double k1, double *pts, int n,
                double qm0);

/* ---- space charge ------------------------------------------------------ */
/* conv1st_BeamBunch, Flagbc=1 (BeamBunch.f90:1252-1352,1657-1663).
 * Compacts lost particles in place; returns the new particle count and
 * rescales *current by nptot/npt. */
int orc_conv1st(double *pts, int n, double *current, int *npt,
                const double refptcl[6], double xrad, double yrad,
                double ptrange[6]);
/* update_CompDom, Flagbc=1 (CompDom.f90:509-823) */
void orc_update_compdom(const double ptrange[6], const int mesh[3],
                        double range[6], double msize[3]);
/* deposit_BeamBunch (BeamBunch.f90:3678-3768).  counts (may be NULL) gets
 * the per-cell particle count of the (ix,jx,kx) cell of every deposited
 * particle; cells (may be NULL) gets the 0-based linear cell index or -1. */
void orc_deposit(const double *pts, int n, const int mesh[3], const double range[6],
                 const double msize[3], double *rho, int *counts, long long *cells);
/* greenf1tIntnew before the FFT (Field.f90:392-428): grn((nx+1),(ny+1),(nz+1)) */
void orc_igf(int nx, int ny, int nz, double hx, double hy, double hz, double *grn);
/* openBC3D (Field.f90:239-331): rho in, phi out (in place), FP64 FFTs */
int orc_poisson_open(int nx, int ny, int nz, double hx, double hy, double hz,
                     double *rho);
/* the same convolution by direct summation (known-answer test, small grids) */
void orc_poisson_direct(int nx, int ny, int nz, double hx, double hy, double hz,
                        const double *rho, double *phi);
/* cvbkforth1st_BeamBunch (BeamBunch.f90:1667-1701) */
void orc_cvbkforth1st(double *pts, int n, const double refptcl[6]);
/* kick1_BeamBunch E-field (BeamBunch.f90:1784-2005) then scatter1
 * (BeamBunch.f90:2041-2181).  eg (may be NULL) receives Ex,Ey,Ez grids. */
void orc_kick1(double *pts, int n, const double *phi, const int mesh[3],
               const double range[6], const double msize[3], double gam,
               double curr, double tau, double mass, double chrg, double *eg);
void orc_kick1w(double *pts, int n, const double *phi, const int mesh[3],
                const double range[6], const double msize[3], double gam,
                double curr, double tau, double mass, double chrg, double *eg,
                const double *wfield);
void orc_drift2(double *pts, int n, double refptcl[6], double tau);

/* read-in wakefield of type -41 elements (Data.f90:559-633,
 * AccSimulator.f90:959-978, 1273-1340, Field.f90:783-1001) */
int orc_wake_set(const double *z, const double *ew, const double *epw, const double *eppw,
                 int ntab, double scale, int transverse);
void orc_wake_off(void);
void orc_wake_elem(int bitype, const double *val);
void orc_wake_field_analytic(int nz, const double *densz, const double *xsum,
                             const double *ysum, const double range[6], double gam, double curr,
                             int npt, double mass, double chrg, double aa, double gg,
                             double leng, double *out);
void orc_wake_line(const double *pts, int n, int nz, const double range[6], double *densz,
                   double *xsum, double *ysum);
void orc_wake_field(int nz, const double *densz, const double *xsum, const double *ysum,
                    const double range[6], double gam, double curr, int npt, double mass,
                    double chrg, double *out);
/* CSR wake (csrwakeTrIGF_FieldQuant, Field.f90:1003-1303) and its glue
 * (AccSimulator.f90:1344-1390) */
void orc_csr_wake(int nx, double r0, double ptmin, double hx, double blength,
                  const double *rho, double gam, double *ez);
void orc_csr_field(int nz, const double *densz, const double range[6], double gam,
                   double curr, int npt, double mass, double chrg, double r0, double s0,
                   double blen, double *out);
void orc_laser_heater(double *pts, int n, int npt, double rsig, double wavelength, double ez,
                      double mass);
/* diagnostic1_Output (Output.f90:20-371): raw sums and one derived row */
void orc_moment_sums(const double *pts, int n, double raw[ORC_RAW_LEN]);
void orc_diag_row(double z, const double raw[ORC_RAW_LEN], int npt, int nlocal,
                  const double refptcl[6], double mass, double row[ORC_DIAG_LEN]);

/* ---- the step loop of run_AccSimulator (AccSimulator.f90:742-1504) ---- */
typedef struct {
  int type;        /* 0 drift, 1 quad, 4 dipole, 101..106 RF gap */
  int nseg, mapstp;
  double length;
  double val[24];  /* deck values v1..v24: Param(k) = val[k-2] for k >= 2 */
  /* on-axis RF table for linear RF maps (types 101..104), or, under the
   * Lorentz integrator, read3_Data's Fourier coefficients in zdat */
  int ndata;
  const double *zdat, *edat, *epdat, *eppdat;
} orc_elem;

/* the Lorentz integrator's kick in element e with zedge = Param(1); z and
 * tg = refptcl(5) at the kick; wraw = the per-plane wake {Ex, Ey, Ez}[nz]
 * of kick2wake or NULL; both return the new gamma0 */
double orc_kick2(double *pts, int n, const double *phi, const int mesh[3], const double range[6],
                 const double msize[3], double gam, double curr, double tau, double mass,
                 double chrg, const orc_elem *e, double zedge, double z, double tg, double qmi,
                 const double *wraw);
double orc_lorentz_nosc(double *pts, int n, double gam, double tau, double mass, double chrg,
                        const orc_elem *e, double zedge, double z, double tg, double qmi);

typedef struct {
  double current, mass, charge, freq;  /* A, eV, e, Hz */
  int npt;                             /* global particle count */
  int nlocal;
  double *pts;                         /* Pts1(9,nlocal) */
  double refptcl[6];
  double z;
  /* CSR bend bookkeeping of run_AccSimulator (AccSimulator.f90:638-740) */
  double zbleng, sentr, bendlencsr, r0;
  int flagbendcsr;
  /* Flagmap: 1 (0 too) the linear map integrator, 2 the Lorentz integrator
   * (drifts, quadrupoles, constant focusing, solenoids, RF cavities
   * 101..104 over Fourier coefficients) */
  int flagmap;
} orc_beam;

/* runs elements [0,nelem); writes one ORC_DIAG_LEN row per diagnostic
 * (the initial one first) into rows (capacity maxrows); returns the number of
 * rows written or a negative error code. */
int orc_run(const orc_elem *elems, int nelem, orc_beam *beam, const int mesh[3],
            double *rows, int maxrows);

#ifdef __cplusplus
}
#endif
#endif
