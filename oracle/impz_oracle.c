/*
 * impz_oracle.c -- CPU restatement of IMPACT-Z's per-step space-charge kick
 * and element push.  TEST INFRASTRUCTURE ONLY (the checker and the timed CPU
 * baseline); the product never links it.  PARITY UNPINNED: no Fortran
 * compiler is available to run the reference, and the reference ships no
 * golden outputs; see impz_oracle.h.
 *
 * Every routine cites the Fortran it restates (paths relative to the
 * IMPACT-Z tree).  Expressions keep the reference's evaluation order
 * (Fortran evaluates a*b*c as (a*b)*c, x**2 as x*x, x**3 as (x*x)*x) and
 * its default-real (FP32) literals where they change the value:
 *   asin(1.0) in conv1st, 1.0/(Meshnum-3.0) in update_CompDom,
 *   1.0e-7 in scatter1, (1.0/3.0) in diagnostic1.
 * Build with -ffp-contract=off: the x86-64 reference build issues no FMA.
 */
#include "impz_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ */
static struct {
  double Pi, Clight, Scxl, Rad2deg, Scfreq;
} PC;

static int g_threads = 1;

void orc_set_threads(int n) { g_threads = n < 1 ? 1 : n; }

/* Optional per-step field capture of orc_run (test infrastructure): the
 * potential (G values) and kick1's Ex, Ey, Ez (3G) of space-charge steps
 * 0..maxsteps-1 are copied to phi + s*G and eg + 3*s*G. */
static struct {
  double *phi, *eg;
  int maxsteps, step;
} g_probe;

void orc_set_field_probe(double *phi, double *eg, int maxsteps) {
  g_probe.phi = phi;
  g_probe.eg = eg;
  g_probe.maxsteps = (phi || eg) ? maxsteps : 0;
  g_probe.step = 0;
}

/* Optional charge-state bookkeeping of orc_run (test infrastructure):
 * chgupdate_BeamBunch (BeamBunch.f90:688-728) after every conv1st updates
 * nptlist (idchgold: the count of particles whose Pts1(7) is within
 * relative eps of qmcclist(j)), and every record copies it to out + nchrg*r,
 * as diagnostic1 writes it to fort.32 (Output.f90:352). */
static struct {
  const double *qmc;
  int nchrg, maxrows;
  int *cur, *out;
} g_chg;

void orc_set_charge_states(const double *qmcclist, int nchrg, int *nptlist, int *out,
                           int maxrows) {
  g_chg.qmc = qmcclist;
  g_chg.nchrg = (qmcclist && nptlist) ? nchrg : 0;
  g_chg.cur = nptlist;
  g_chg.out = out;
  g_chg.maxrows = out ? maxrows : 0;
}

/* chgupdate_BeamBunch (BeamBunch.f90:697-722); eps = 1.0e-4, a default-real
 * literal */
static void orc_chgupdate(const double *pts, int n) {
  if (!g_chg.nchrg) return;
  const double eps = (double)1.0e-4f;
  for (int j = 0; j < g_chg.nchrg; j++) g_chg.cur[j] = 0;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < g_chg.nchrg; j++) {
      const double dd = fabs((pts[9 * (size_t)i + 6] - g_chg.qmc[j]) / g_chg.qmc[j]);
      if (dd < eps) g_chg.cur[j]++;
    }
}

/* PhysConst.f90:25-35 */
void orc_physconst(double freq) {
  PC.Clight = 299792458.0;
  PC.Pi = 2 * asin(1.0);
  PC.Scxl = PC.Clight / (2 * PC.Pi * freq);
  PC.Rad2deg = 180.0 / PC.Pi;
  PC.Scfreq = freq;
}

void orc_get_physconst(double out[5]) {
  out[0] = PC.Pi;
  out[1] = PC.Clight;
  out[2] = PC.Scxl;
  out[3] = PC.Rad2deg;
  out[4] = PC.Scfreq;
}

#define P(i, c) pts[9 * (size_t)(i) + (c)]

/* ------------------------------------------------------------------ */
/* drift1_BeamBunch, bitype 0: exact drift (BeamBunch.f90:276-298) */
/* drift2_BeamBunch (BeamBunch.f90:467-509): the Lorentz integrator's drift
 * by 0.5*tau; returns nothing, advances refptcl(5) */
void orc_drift2(double *pts, int n, double refptcl[6], double tau) {
  const double xl = PC.Scxl;
  const double gamma0 = -refptcl[5];
  const double beta0 = sqrt(1.0 - 1.0 / gamma0 / gamma0);
  for (int i = 0; i < n; i++) {
    const double pz = sqrt((gamma0 - P(i, 5)) * (gamma0 - P(i, 5)) - 1.0 - P(i, 1) * P(i, 1) -
                           P(i, 3) * P(i, 3));
    P(i, 0) = P(i, 0) + 0.5 * tau * P(i, 1) / (xl * pz);
    P(i, 2) = P(i, 2) + 0.5 * tau * P(i, 3) / (xl * pz);
    P(i, 4) = P(i, 4) + 0.5 * tau * ((gamma0 - P(i, 5)) / (xl * pz) - 1.0 / (beta0 * xl));
  }
  refptcl[4] = refptcl[4] + 0.5 * tau / (xl * beta0);
}

void orc_drift_exact(double *pts, int n, double refptcl[6], double tau) {
  const double Scxl = PC.Scxl;
  double gam0 = -refptcl[5];
  double gambet0 = sqrt(gam0 * gam0 - 1.0);
  double beta0 = gambet0 / gam0;
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads)
  for (int i = 0; i < n; i++) {
    double tmppx = P(i, 1), tmppy = P(i, 3), tmppt = P(i, 5);
    double d = tmppt - gam0;
    double tmph = sqrt(((d * d - 1) - tmppx * tmppx) - tmppy * tmppy);
    P(i, 0) = P(i, 0) + ((tmppx * tau) / tmph) / Scxl;
    P(i, 2) = P(i, 2) + ((tmppy * tau) / tmph) / Scxl;
    P(i, 4) = P(i, 4) - ((1. / beta0 + (tmppt - gam0) / tmph) * tau) / Scxl;
  }
  refptcl[4] = refptcl[4] + tau / (Scxl * beta0);
}

/* ------------------------------------------------------------------ */
/* rk6i_* (Quadrupole.f90:202-252, identical in DriftTube/CCL): 8-stage RK6 */
typedef void (*orc_rhs)(double t, const double *y, double *f, const void *ctx);

static void rk6in(double h, int ns, double *t, double *y, int NV, orc_rhs fn,
                  const void *ctx) {
  double yt[22], a[22], b[22], c[22], d[22], e[22], f[22], g[22], o[22], p[22];
  double tint = *t, tt;
  int v;
  for (int i = 1; i <= ns; i++) {
    fn(*t, y, f, ctx);
    for (v = 0; v < NV; v++) a[v] = h * f[v];
    for (v = 0; v < NV; v++) yt[v] = y[v] + a[v] / 9.0;
    tt = *t + h / 9.0;
    fn(tt, yt, f, ctx);
    for (v = 0; v < NV; v++) b[v] = h * f[v];
    for (v = 0; v < NV; v++) yt[v] = y[v] + (a[v] + 3.0 * b[v]) / 24.0;
    tt = *t + h / 6.0;
    fn(tt, yt, f, ctx);
    for (v = 0; v < NV; v++) c[v] = h * f[v];
    for (v = 0; v < NV; v++) yt[v] = y[v] + ((a[v] - 3.0 * b[v]) + 4.0 * c[v]) / 6.0;
    tt = *t + h / 3.0;
    fn(tt, yt, f, ctx);
    for (v = 0; v < NV; v++) d[v] = h * f[v];
    for (v = 0; v < NV; v++)
      yt[v] = y[v] + (((278.0 * a[v] - 945.0 * b[v]) + 840.0 * c[v]) + 99.0 * d[v]) / 544.0;
    tt = *t + .5 * h;
    fn(tt, yt, f, ctx);
    for (v = 0; v < NV; v++) e[v] = h * f[v];
    for (v = 0; v < NV; v++)
      yt[v] = y[v] + (((((-106.0 * a[v]) + 273.0 * b[v]) - 104.0 * c[v]) - 107.0 * d[v]) +
                      48.0 * e[v]) / 6.0;
    tt = *t + 2.0 * h / 3.0;
    fn(tt, yt, f, ctx);
    for (v = 0; v < NV; v++) g[v] = h * f[v];
    for (v = 0; v < NV; v++)
      yt[v] = y[v] + (((((110974.0 * a[v] - 236799.0 * b[v]) + 68376.0 * c[v]) +
                        103803.0 * d[v]) - 10240.0 * e[v]) + 1926.0 * g[v]) / 45648.0;
    tt = *t + 5.0 * h / 6.0;
    fn(tt, yt, f, ctx);
    for (v = 0; v < NV; v++) o[v] = h * f[v];
    for (v = 0; v < NV; v++)
      yt[v] = y[v] + ((((((-101195.0 * a[v]) + 222534.0 * b[v]) - 71988.0 * c[v]) -
                         26109.0 * d[v]) - 2.e4 * e[v]) - 72.0 * g[v] + 22824.0 * o[v]) /
                         25994.0;
    tt = *t + h;
    fn(tt, yt, f, ctx);
    for (v = 0; v < NV; v++) p[v] = h * f[v];
    for (v = 0; v < NV; v++)
      y[v] = y[v] + ((((((41.0 * a[v] + 216.0 * c[v]) + 27.0 * d[v]) + 272.0 * e[v]) +
                       27.0 * g[v]) + 216.0 * o[v]) + 41.0 * p[v]) / 840.0;
    *t = tint + i * h;
  }
}

static void rk6i(double h, int ns, double *t, double *y, orc_rhs fn, const void *ctx) {
  rk6in(h, ns, t, y, 18, fn, ctx);
}

/* the 18 linear-ODE derivatives shared by intfunc1_* given s11,s33,s55 */
static void lin_rhs(const double *y, double *f, double s11, double s33, double s55) {
  const double Scxl = PC.Scxl;
  f[6] = y[7] / Scxl;
  f[7] = -s11 * y[6];
  f[8] = y[9] / Scxl;
  f[9] = -s11 * y[8];
  f[10] = y[11] / Scxl;
  f[11] = -s33 * y[10];
  f[12] = y[13] / Scxl;
  f[13] = -s33 * y[12];
  f[14] = y[15] / Scxl;
  f[15] = -s55 * y[14];
  f[16] = y[17] / Scxl;
  f[17] = -s55 * y[16];
}

typedef struct {
  double bgrad, qmcc;
  /* fringe-field profile (Param(3) > 1e-5): the gradient table of
   * read1_Data, looked up at t - zedge by getfldfrg_Quadrupole */
  int ndata;
  const double *zdat, *gdat;
  double zedge;
} quad_ctx;

/* getfldfrg_Quadrupole (Quadrupole.f90:404-430): bisection + linear
 * interpolation of the gradient table */
static double quad_fringe(double zz, const quad_ctx *q) {
  const double *zd = q->zdat - 1, *gd = q->gdat - 1;
  int klo = 1, khi = q->ndata;
  while (khi - klo > 1) {
    const int k = (khi + klo) / 2;
    if (zd[k] > zz) khi = k; else klo = k;
  }
  const double hstep = zd[khi] - zd[klo];
  const double slope = (gd[khi] - gd[klo]) / hstep;
  return gd[klo] + slope * (zz - zd[klo]);
}

/* intfunc1_Quadrupole (Quadrupole.f90:254-305) */
static void quad_rhs(double t, const double *y, double *f, const void *vctx) {
  const quad_ctx *q = (const quad_ctx *)vctx;
  double gamma0, beta0, gbet, brho, s11, s33, s55;
  const double bgrad = q->ndata > 1 ? quad_fringe(t - q->zedge, q) : q->bgrad;
  f[0] = 0.0; f[1] = 0.0; f[2] = 0.0; f[3] = 0.0;
  gamma0 = -y[5];
  beta0 = sqrt(gamma0 * gamma0 - 1.) / gamma0;
  gbet = sqrt((gamma0 - 1.0) * (gamma0 + 1.0));
  f[4] = 1.0 / (beta0 * PC.Scxl);
  f[5] = 0.0;
  brho = gbet / PC.Clight / q->qmcc;
  s11 = bgrad / brho * PC.Scxl;
  s33 = -(bgrad / brho * PC.Scxl);
  s55 = 0.0;
  lin_rhs(y, f, s11, s33, s55);
}

/* intfunc1_DriftTube (DriftTube.f90:245-288) */
static void drift_rhs(double t, const double *y, double *f, const void *vctx) {
  (void)t; (void)vctx;
  double gamma0 = -y[5];
  double beta0 = sqrt(gamma0 * gamma0 - 1.) / gamma0;
  f[0] = 0.0; f[1] = 0.0; f[2] = 0.0; f[3] = 0.0;
  f[4] = 1.0 / (beta0 * PC.Scxl);
  f[5] = 0.0;
  lin_rhs(y, f, 0.0, 0.0, 0.0);
}

static void y_init(double *y, const double refpt[6]) {
  memset(y, 0, 18 * sizeof(double));
  y[4] = refpt[4];
  y[5] = refpt[5];
  y[6] = 1.0; y[9] = 1.0; y[10] = 1.0; y[13] = 1.0; y[14] = 1.0; y[17] = 1.0;
}

#define XM(j, k) xm[((j)-1) + 6 * ((k)-1)]

/* the xm assembly shared by maplinear_* (Quadrupole.f90:183-198) */
static void xm_assemble(double xm[36], const double *y, double squi, double squf,
                        double sqi3, double sqf3, double dlti, double dltf,
                        double thli, double thlf) {
  const double *Y = y - 1; /* 1-based like the Fortran */
  XM(1, 1) = Y[7] * squi / squf + Y[9] * squi / squf * dlti;
  XM(2, 1) = (Y[8] - Y[7] * dltf) * squi * squf + (Y[10] - Y[9] * dltf) * squi * squf * dlti;
  XM(1, 2) = Y[9] / (squi * squf);
  XM(2, 2) = (Y[10] - Y[9] * dltf) * squf / squi;
  XM(3, 3) = Y[11] * squi / squf + Y[13] * squi / squf * dlti;
  XM(4, 3) = (Y[12] - Y[11] * dltf) * squi * squf + (Y[14] - Y[13] * dltf) * squi * squf * dlti;
  XM(3, 4) = Y[13] / (squi * squf);
  XM(4, 4) = (Y[14] - Y[13] * dltf) * squf / squi;
  XM(5, 5) = Y[15] * sqi3 / sqf3 + Y[17] * sqi3 / sqf3 * thli;
  XM(6, 5) = (Y[16] - Y[15] * thlf) * sqi3 * sqf3 + (Y[18] - Y[17] * thlf) * sqi3 * sqf3 * thli;
  XM(5, 6) = Y[17] / (sqi3 * sqf3);
  XM(6, 6) = (Y[18] - Y[17] * thlf) * sqf3 / sqi3;
}

/* maplinear_Quadrupole (Quadrupole.f90:120-200) */
static void maplinear_quad(double t, double tau, double xm[36], double refpt[6],
                           const quad_ctx *qc, int mapstp) {
  double y[18], h, t0, gi, betai, ui, squi, sqi3, gf, betaf, uf, squf, sqf3, s;
  const quad_ctx q = *qc;
  memset(xm, 0, 36 * sizeof(double));
  y_init(y, refpt);
  h = tau / mapstp;
  t0 = t;
  gi = -refpt[5];
  betai = sqrt(gi * gi - 1.) / gi;
  ui = gi * betai;
  squi = sqrt(ui);
  s = sqrt(ui);
  sqi3 = s * s * s;
  rk6i(h, mapstp, &t0, y, quad_rhs, &q);
  refpt[4] = y[4];
  refpt[5] = y[5];
  gf = -refpt[5];
  betaf = sqrt(gf * gf - 1.) / gf;
  uf = gf * betaf;
  squf = sqrt(uf);
  s = sqrt(uf);
  sqf3 = s * s * s;
  xm_assemble(xm, y, squi, squf, sqi3, sqf3, 0.0, 0.0, 0.0, 0.0);
}

/* maplinear_DriftTube (DriftTube.f90:113-191) */
void orc_maplinear_drift(double t, double tau, double xm[36], double refpt[6],
                         int mapstp, double chg, double mass) {
  (void)chg; (void)mass;
  double y[18], h, t0, gi, betai, ui, squi, sqi3, gf, betaf, uf, squf, sqf3, s;
  memset(xm, 0, 36 * sizeof(double));
  y_init(y, refpt);
  h = tau / mapstp;
  t0 = t;
  gi = -refpt[5];
  betai = sqrt(gi * gi - 1.) / gi;
  ui = gi * betai;
  squi = sqrt(ui);
  s = sqrt(ui);
  sqi3 = s * s * s;
  rk6i(h, mapstp, &t0, y, drift_rhs, NULL);
  refpt[4] = y[4];
  refpt[5] = y[5];
  gf = -refpt[5];
  betaf = sqrt(gf * gf - 1.) / gf;
  uf = gf * betaf;
  squf = sqrt(uf);
  s = sqrt(uf);
  sqf3 = s * s * s;
  xm_assemble(xm, y, squi, squf, sqi3, sqf3, 0.0, 0.0, 0.0, 0.0);
}

void orc_maplinear_quad(double t, double tau, double xm[36], double refpt[6],
                        double gradient, int mapstp, double chg, double mass) {
  const quad_ctx q = {gradient, chg / mass, 0, NULL, NULL, 0.0};
  maplinear_quad(t, tau, xm, refpt, &q, mapstp);
}

/* the fringe-field quadrupole: gradient profile (z from 0, G) at zedge */
void orc_maplinear_quad_fringe(double t, double tau, double xm[36], double refpt[6],
                               double zedge, int mapstp, double chg, double mass, int ndata,
                               const double *zdat, const double *gdat) {
  const quad_ctx q = {0.0, chg / mass, ndata, zdat, gdat, zedge};
  maplinear_quad(t, tau, xm, refpt, &q, mapstp);
}

/* ---- CCL linear gap ---------------------------------------------------- */
typedef struct {
  double zedge, escale, ww, theta0, qmcc;
  int ndata;
  const double *zdat, *edat, *epdat, *eppdat;
  /* DTL (type 101): the element length and its drift-tube quadrupoles,
   * Param(7..10) (DTL.f90:26-29) */
  int dtl;
  double dlen, q1len, q1grad, q2len, q2grad;
} ccl_ctx;

/* getaxfldE_CCL (CCL.f90:331-365): bisection + linear interpolation */
static void ccl_field(double z, const ccl_ctx *c, double *ez1, double *ezp1, double *ezpp1) {
  double zz = z - c->zedge, hstep, slope;
  int klo = 1, khi = c->ndata, k;
  const double *zd = c->zdat - 1, *ed = c->edat - 1, *epd = c->epdat - 1, *eppd = c->eppdat - 1;
  while (khi - klo > 1) {
    k = (khi + klo) / 2;
    if (zd[k] > zz) khi = k; else klo = k;
  }
  hstep = zd[khi] - zd[klo];
  slope = (ed[khi] - ed[klo]) / hstep;
  *ez1 = ed[klo] + slope * (zz - zd[klo]);
  slope = (epd[khi] - epd[klo]) / hstep;
  *ezp1 = epd[klo] + slope * (zz - zd[klo]);
  slope = (eppd[khi] - eppd[klo]) / hstep;
  *ezpp1 = eppd[klo] + slope * (zz - zd[klo]);
  *ez1 = *ez1 * c->escale;
  *ezp1 = *ezp1 * c->escale;
  *ezpp1 = *ezpp1 * c->escale;
}

/* intfunc1_CCL (CCL.f90:269-328) */
static void ccl_rhs(double t, const double *y, double *f, const void *vctx) {
  const ccl_ctx *c = (const ccl_ctx *)vctx;
  const double Scxl = PC.Scxl;
  double ez1, ezp1, ezpp1, gamma0, beta0, sinphi, cosphi, rfdsgn, s11tmp, s11, s33, s55, q;
  ccl_field(t, c, &ez1, &ezp1, &ezpp1);
  f[0] = 0.0; f[1] = 0.0; f[2] = 0.0; f[3] = 0.0;
  gamma0 = -y[5];
  beta0 = sqrt(gamma0 * gamma0 - 1.) / gamma0;
  sinphi = sin(c->ww * y[4] + c->theta0);
  cosphi = cos(c->ww * y[4] + c->theta0);
  rfdsgn = ez1 * cosphi;
  f[4] = 1.0 / (beta0 * Scxl);
  f[5] = -(c->qmcc * rfdsgn);
  q = c->qmcc * rfdsgn / (beta0 * beta0) / (gamma0 * gamma0);
  s11tmp = 0.5 * (1.0 + 0.5 * (gamma0 * gamma0)) * (q * q) +
           c->qmcc * 0.5 / ((beta0 * beta0) * beta0) / ((gamma0 * gamma0) * gamma0) * ez1 *
               sinphi * c->ww / Scxl;
  if (c->dtl) {
    /* intfunc1_DTL (DTL.f90:286-347): the drift-tube quadrupole gradient of
     * getBgradfld_DTL (DTL.f90:395-418) focuses x and defocuses y */
    const double zz = t - c->zedge;
    const double bgrad = zz < c->q1len ? c->q1grad : (zz < c->dlen - c->q2len ? 0.0 : c->q2grad);
    const double gbet = sqrt((gamma0 - 1.0) * (gamma0 + 1.0));
    const double brho = gbet / PC.Clight / c->qmcc;
    s11 = (s11tmp + bgrad / brho) * Scxl;
    s33 = (s11tmp - bgrad / brho) * Scxl;
  } else {
    s11 = s11tmp * Scxl;
    s33 = s11tmp * Scxl;
  }
  s55 = -(1.5 * c->qmcc / (beta0 * beta0) / gamma0 * ezp1 * cosphi) +
        ((beta0 * beta0) + 0.5) / ((beta0 * beta0) * beta0) / gamma0 * c->qmcc * ez1 * sinphi *
            c->ww / Scxl +
        1.5 * (1.0 - 0.5 * (gamma0 * gamma0)) * (q * q);
  s55 = Scxl * s55;
  lin_rhs(y, f, s11, s33, s55);
}

/* maplinear_CCL (CCL.f90:122-215); maplinear_CCDTL and maplinear_SC
 * (CCDTL.f90:122-215, SC.f90:122-215) are the same map; maplinear_DTL
 * (DTL.f90:136-232) adds the drift-tube quadrupoles (dtlq = length,
 * Param(7..10), NULL for the others) */
static void maplinear_rf(double t, double tau, double xm[36], double refpt[6], double zedge,
                         double escale, double freq, double phase_deg, int mapstp, double chg,
                         double mass, int ndata, const double *zdat, const double *edat,
                         const double *epdat, const double *eppdat, const double *dtlq) {
  const double Scxl = PC.Scxl;
  ccl_ctx c;
  c.dtl = dtlq != NULL;
  c.dlen = dtlq ? dtlq[0] : 0.0;
  c.q1len = dtlq ? dtlq[1] : 0.0;
  c.q1grad = dtlq ? dtlq[2] : 0.0;
  c.q2len = dtlq ? dtlq[3] : 0.0;
  c.q2grad = dtlq ? dtlq[4] : 0.0;
  double y[18], h, t0, gi, betai, ui, squi, sqi3, gf, betaf, uf, squf, sqf3, s;
  double ein, e1in, e2in, ef, e1f, e2f, sinthi, costhi, uprimi, qpwi, dlti, thli;
  double sinthf, costhf, uprimf, qpwf, dltf, thlf, tfin;
  c.zedge = zedge;
  c.escale = escale;
  c.ww = freq / PC.Scfreq;
  /* theta0 = Param(4)*asin(1.0)/90 with a default-real asin(1.0) */
  c.theta0 = phase_deg * (double)asinf(1.0f) / 90;
  c.qmcc = chg / mass;
  c.ndata = ndata;
  c.zdat = zdat; c.edat = edat; c.epdat = epdat; c.eppdat = eppdat;
  memset(xm, 0, 36 * sizeof(double));
  y_init(y, refpt);
  h = tau / mapstp;
  t0 = t;
  gi = -refpt[5];
  betai = sqrt(gi * gi - 1.) / gi;
  ui = gi * betai;
  squi = sqrt(ui);
  s = sqrt(ui);
  sqi3 = s * s * s;
  ccl_field(t, &c, &ein, &e1in, &e2in);
  sinthi = sin(c.ww * refpt[4] + c.theta0);
  costhi = cos(c.ww * refpt[4] + c.theta0);
  uprimi = c.qmcc * ein / betai * costhi;
  qpwi = 0.5 * c.qmcc * Scxl / (ui * c.ww);
  dlti = Scxl * (0.5 * uprimi / ui - qpwi * e1in * sinthi);
  thli = 1.5 * Scxl * (uprimi / ui);
  rk6i(h, mapstp, &t0, y, ccl_rhs, &c);
  refpt[4] = y[4];
  refpt[5] = y[5];
  gf = -refpt[5];
  betaf = sqrt(gf * gf - 1.) / gf;
  uf = gf * betaf;
  squf = sqrt(uf);
  s = sqrt(uf);
  sqf3 = s * s * s;
  tfin = t + tau;
  ccl_field(tfin, &c, &ef, &e1f, &e2f);
  sinthf = sin(c.ww * refpt[4] + c.theta0);
  costhf = cos(c.ww * refpt[4] + c.theta0);
  uprimf = c.qmcc * ef / betaf * costhf;
  qpwf = 0.5 * c.qmcc * Scxl / (uf * c.ww);
  dltf = Scxl * (0.5 * uprimf / uf - qpwf * e1f * sinthf);
  thlf = 1.5 * Scxl * (uprimf / uf);
  xm_assemble(xm, y, squi, squf, sqi3, sqf3, dlti, dltf, thli, thlf);
}

void orc_maplinear_ccl(double t, double tau, double xm[36], double refpt[6],
                       double zedge, double escale, double freq, double phase_deg,
                       int mapstp, double chg, double mass,
                       int ndata, const double *zdat, const double *edat,
                       const double *epdat, const double *eppdat) {
  maplinear_rf(t, tau, xm, refpt, zedge, escale, freq, phase_deg, mapstp, chg, mass, ndata, zdat,
               edat, epdat, eppdat, NULL);
}

void orc_maplinear_dtl(double t, double tau, double xm[36], double refpt[6],
                       double zedge, double escale, double freq, double phase_deg,
                       int mapstp, double chg, double mass,
                       int ndata, const double *zdat, const double *edat,
                       const double *epdat, const double *eppdat, double length,
                       double q1len, double q1grad, double q2len, double q2grad) {
  const double q[5] = {length, q1len, q1grad, q2len, q2grad};
  maplinear_rf(t, tau, xm, refpt, zedge, escale, freq, phase_deg, mapstp, chg, mass, ndata, zdat,
               edat, epdat, eppdat, q);
}

/* ---- SolRF (type 105) linear map ------------------------------------ */
typedef struct {
  double zedge, escale, len, ww, theta0, qmcc, b0;
  int ncoef;
  const double *F; /* read3_Data's coefficients, 1-based through F[k-1] */
} solrf_ctx;

/* getaxfldE_SolRF (SolRF.f90:355-466) */
static void solrf_field(double z, const solrf_ctx *c, double *ez1, double *ezp1) {
  const double *F = c->F - 1;
  const double epstol = (double)1.0e-10f;
  *ez1 = 0.0;
  *ezp1 = 0.0;
  if (((z >= c->zedge) && (z <= (c->zedge + c->len))) || (fabs(z - c->zedge) <= epstol) ||
      (fabs(z - c->zedge - c->len) <= epstol)) {
    const double zlc = z - c->zedge;
    const int numpar1 = (int)(F[1] + 0.1);
    const double zstart1 = F[2], zend1 = F[3], zlength1 = F[4];
    if (((zlc >= zstart1) && (zlc <= zend1)) || (fabs(zlc - zstart1) <= epstol) ||
        (fabs(zlc - zend1) <= epstol)) {
      const double zmid = zlength1 / 2;
      const double zz = z - c->zedge - zstart1 - zmid;
      const double zlen = zlength1;
      const int ntmp = 4;
      double e = F[ntmp + 1] / 2, ep = 0.0;
      for (int i = 2; i <= (numpar1 - 1) / 2 + 1; i++) {
        e = e + F[2 * i - 2 + ntmp] * cos((i - 1) * 2 * PC.Pi * zz / zlen) +
            F[2 * i - 1 + ntmp] * sin((i - 1) * 2 * PC.Pi * zz / zlen);
        ep = ep + (i - 1) * 2 * PC.Pi / zlen *
                      (-F[2 * i - 2 + ntmp] * sin((i - 1) * 2 * PC.Pi * zz / zlen) +
                       F[2 * i - 1 + ntmp] * cos((i - 1) * 2 * PC.Pi * zz / zlen));
      }
      *ez1 = e * c->escale;
      *ezp1 = ep * c->escale;
    }
  }
}

/* intfunc1_SolRF (SolRF.f90:287-353) */
static void solrf_rhs(double t, const double *y, double *f, const void *vctx) {
  const solrf_ctx *c = (const solrf_ctx *)vctx;
  const double Scxl = PC.Scxl;
  double ez1, ezp1;
  solrf_field(t, c, &ez1, &ezp1);
  f[0] = 0.0; f[1] = 0.0; f[2] = 0.0; f[3] = 0.0;
  const double gamma0 = -y[5];
  const double beta0 = sqrt(gamma0 * gamma0 - 1.) / gamma0;
  const double gbet = sqrt((gamma0 - 1.0) * (gamma0 + 1.0));
  const double sinphi = sin(c->ww * y[4] + c->theta0);
  const double cosphi = cos(c->ww * y[4] + c->theta0);
  const double rfdsgn = ez1 * cosphi;
  f[4] = 1.0 / (beta0 * Scxl);
  f[5] = -(c->qmcc * rfdsgn);
  const double brho = gbet / PC.Clight / c->qmcc;
  const double q = c->qmcc * rfdsgn / (beta0 * beta0) / (gamma0 * gamma0);
  const double s11tmp = 0.5 * (1.0 + 0.5 * (gamma0 * gamma0)) * (q * q) +
                        c->qmcc * 0.5 / ((beta0 * beta0) * beta0) / ((gamma0 * gamma0) * gamma0) *
                            ez1 * sinphi * c->ww / Scxl;
  const double sol = 0.5 * c->b0 / brho;
  const double s11 = (s11tmp + sol * sol / 2) * Scxl;
  const double s33 = (s11tmp + sol * sol / 2) * Scxl;
  double s55 = -(1.5 * c->qmcc / (beta0 * beta0) / gamma0 * ezp1 * cosphi) +
               ((beta0 * beta0) + 0.5) / ((beta0 * beta0) * beta0) / gamma0 * c->qmcc * ez1 *
                   sinphi * c->ww / Scxl +
               1.5 * (1.0 - 0.5 * (gamma0 * gamma0)) * (q * q);
  s55 = Scxl * s55;
  lin_rhs(y, f, s11, s33, s55);
  const double c2alpha = -c->b0 / brho / 2;
  f[18] = -c2alpha * y[20];
  f[19] = -c2alpha * y[21];
  f[20] = c2alpha * y[18];
  f[21] = c2alpha * y[19];
}

/* maplinear_SolRF (SolRF.f90:126-233): coef = read3_Data's coefficients
 * (ncoef values), b0 = the solenoid field Param(12) */
void orc_maplinear_solrf(double t, double tau, double xm[36], double refpt[6], double zedge,
                         double escale, double freq, double phase_deg, int mapstp, double chg,
                         double mass, double length, double b0, int ncoef, const double *coef) {
  const double Scxl = PC.Scxl;
  solrf_ctx c;
  double y[22];
  c.zedge = zedge; c.escale = escale; c.len = length;
  c.ww = freq / PC.Scfreq;
  c.theta0 = phase_deg * (double)asinf(1.0f) / 90;
  c.qmcc = chg / mass;
  c.b0 = b0;
  c.ncoef = ncoef;
  c.F = coef;
  memset(xm, 0, 36 * sizeof(double));
  y_init(y, refpt);
  y[18] = 1.0; y[19] = 0.0; y[20] = 0.0; y[21] = 1.0;
  const double h = tau / mapstp;
  double t0 = t;
  const double gi = -refpt[5];
  const double betai = sqrt(gi * gi - 1.) / gi;
  const double ui = gi * betai;
  const double squi = sqrt(ui);
  double s = sqrt(ui);
  const double sqi3 = s * s * s;
  double ein, e1in;
  solrf_field(t, &c, &ein, &e1in);
  const double sinthi = sin(c.ww * refpt[4] + c.theta0);
  const double costhi = cos(c.ww * refpt[4] + c.theta0);
  const double uprimi = c.qmcc * ein / betai * costhi;
  const double qpwi = 0.5 * c.qmcc * Scxl / (ui * c.ww);
  const double dlti = Scxl * (0.5 * uprimi / ui - qpwi * e1in * sinthi);
  const double thli = 1.5 * Scxl * (uprimi / ui);
  rk6in(h, mapstp, &t0, y, 22, solrf_rhs, &c);
  refpt[4] = y[4];
  refpt[5] = y[5];
  const double gf = -refpt[5];
  const double betaf = sqrt(gf * gf - 1.) / gf;
  const double uf = gf * betaf;
  const double squf = sqrt(uf);
  s = sqrt(uf);
  const double sqf3 = s * s * s;
  double ef, e1f;
  solrf_field(t + tau, &c, &ef, &e1f);
  const double sinthf = sin(c.ww * refpt[4] + c.theta0);
  const double costhf = cos(c.ww * refpt[4] + c.theta0);
  const double uprimf = c.qmcc * ef / betaf * costhf;
  const double qpwf = 0.5 * c.qmcc * Scxl / (uf * c.ww);
  const double dltf = Scxl * (0.5 * uprimf / uf - qpwf * e1f * sinthf);
  const double thlf = 1.5 * Scxl * (uprimf / uf);
  xm_assemble(xm, y, squi, squf, sqi3, sqf3, dlti, dltf, thli, thlf);
  const double *Y = y - 1;
#define XM(j, k) xm[((j)-1) + 6 * ((k)-1)]
  XM(1, 1) = Y[19] * (Y[7] * squi / squf + Y[9] * squi / squf * dlti);
  XM(2, 1) = Y[19] * ((Y[8] - Y[7] * dltf) * squi * squf + (Y[10] - Y[9] * dltf) * squi * squf *
                                                                 dlti);
  XM(1, 2) = Y[19] * Y[9] / (squi * squf);
  XM(2, 2) = Y[19] * (Y[10] - Y[9] * dltf) * squf / squi;
  XM(1, 3) = Y[20] * (Y[7] * squi / squf + Y[9] * squi / squf * dlti);
  XM(2, 3) = Y[20] * ((Y[8] - Y[7] * dltf) * squi * squf + (Y[10] - Y[9] * dltf) * squi * squf *
                                                                 dlti);
  XM(1, 4) = Y[20] * Y[9] / (squi * squf);
  XM(2, 4) = Y[20] * (Y[10] - Y[9] * dltf) * squf / squi;
  XM(3, 1) = Y[21] * (Y[11] * squi / squf + Y[13] * squi / squf * dlti);
  XM(4, 1) = Y[21] * ((Y[12] - Y[11] * dltf) * squi * squf +
                      (Y[14] - Y[13] * dltf) * squi * squf * dlti);
  XM(3, 2) = Y[21] * Y[13] / (squi * squf);
  XM(4, 2) = Y[21] * (Y[14] - Y[13] * dltf) * squf / squi;
  XM(3, 3) = Y[22] * (Y[11] * squi / squf + Y[13] * squi / squf * dlti);
  XM(4, 3) = Y[22] * ((Y[12] - Y[11] * dltf) * squi * squf +
                      (Y[14] - Y[13] * dltf) * squi * squf * dlti);
  XM(3, 4) = Y[22] * Y[13] / (squi * squf);
  XM(4, 4) = Y[22] * (Y[14] - Y[13] * dltf) * squf / squi;
#undef XM
}

/* ---- ConstFoc (type 2) linear map ------------------------------------- */
/* intfunc1_ConstFoc (ConstFoc.f90), k2 = kx0^2, ky0^2, kz0^2 */
static void constfoc_rhs(double t, const double *y, double *f, const void *vctx) {
  (void)t;
  const double *k2 = (const double *)vctx;
  const double Scxl = PC.Scxl;
  f[0] = 0.0; f[1] = 0.0; f[2] = 0.0; f[3] = 0.0;
  const double gamma0 = -y[5];
  const double beta0 = sqrt(gamma0 * gamma0 - 1.) / gamma0;
  f[4] = 1.0 / (beta0 * Scxl);
  f[5] = 0.0;
  lin_rhs(y, f, k2[0] * Scxl, k2[1] * Scxl, k2[2] * Scxl);
}

/* maplinear_ConstFoc (ConstFoc.f90) */
void orc_maplinear_constfoc(double t, double tau, double xm[36], double refpt[6],
                            const double k2[3], int mapstp) {
  double y[18];
  memset(xm, 0, 36 * sizeof(double));
  y_init(y, refpt);
  const double h = tau / mapstp;
  double t0 = t;
  const double gi = -refpt[5];
  const double betai = sqrt(gi * gi - 1.) / gi;
  const double ui = gi * betai;
  const double squi = sqrt(ui);
  double s = sqrt(ui);
  const double sqi3 = s * s * s;
  rk6i(h, mapstp, &t0, y, constfoc_rhs, k2);
  refpt[4] = y[4];
  refpt[5] = y[5];
  const double gf = -refpt[5];
  const double betaf = sqrt(gf * gf - 1.) / gf;
  const double uf = gf * betaf;
  const double squf = sqrt(uf);
  s = sqrt(uf);
  const double sqf3 = s * s * s;
  xm_assemble(xm, y, squi, squf, sqi3, sqf3, 0.0, 0.0, 0.0, 0.0);
}

/* ---- Sol (type 3) linear map ------------------------------------------ */
typedef struct { double b0, qmcc; } sol_ctx;

/* intfunc1_Sol (Sol.f90:264-316) */
static void sol_rhs(double t, const double *y, double *f, const void *vctx) {
  (void)t;
  const sol_ctx *c = (const sol_ctx *)vctx;
  const double Scxl = PC.Scxl;
  f[0] = 0.0; f[1] = 0.0; f[2] = 0.0; f[3] = 0.0;
  const double gamma0 = -y[5];
  const double beta0 = sqrt(gamma0 * gamma0 - 1.) / gamma0;
  const double gbet = sqrt((gamma0 - 1.0) * (gamma0 + 1.0));
  f[4] = 1.0 / (beta0 * Scxl);
  f[5] = 0.0;
  const double brho = gbet / PC.Clight / c->qmcc;
  const double sol = 0.5 * c->b0 / brho;
  const double s11 = (sol * sol) * Scxl;
  const double s33 = (sol * sol) * Scxl;
  lin_rhs(y, f, s11, s33, 0.0);
  const double c2alpha = -c->b0 / brho / 2;
  f[18] = -c2alpha * y[20];
  f[19] = -c2alpha * y[21];
  f[20] = c2alpha * y[18];
  f[21] = c2alpha * y[19];
}

/* maplinear_Sol (Sol.f90:120-210) */
void orc_maplinear_sol(double t, double tau, double xm[36], double refpt[6], double b0,
                       int mapstp, double chg, double mass) {
  sol_ctx c = {b0, chg / mass};
  double y[22];
  memset(xm, 0, 36 * sizeof(double));
  y_init(y, refpt);
  y[18] = 1.0; y[19] = 0.0; y[20] = 0.0; y[21] = 1.0;
  const double h = tau / mapstp;
  double t0 = t;
  const double gi = -refpt[5];
  const double betai = sqrt(gi * gi - 1.) / gi;
  const double ui = gi * betai;
  const double squi = sqrt(ui);
  double s = sqrt(ui);
  const double sqi3 = s * s * s;
  const double dlti = 0.0, thli = 0.0;
  rk6in(h, mapstp, &t0, y, 22, sol_rhs, &c);
  refpt[4] = y[4];
  refpt[5] = y[5];
  const double gf = -refpt[5];
  const double betaf = sqrt(gf * gf - 1.) / gf;
  const double uf = gf * betaf;
  const double squf = sqrt(uf);
  s = sqrt(uf);
  const double sqf3 = s * s * s;
  const double dltf = 0.0, thlf = 0.0;
  xm_assemble(xm, y, squi, squf, sqi3, sqf3, dlti, dltf, thli, thlf);
  const double *Y = y - 1;
#define XM(j, k) xm[((j)-1) + 6 * ((k)-1)]
  XM(1, 1) = Y[19] * (Y[7] * squi / squf + Y[9] * squi / squf * dlti);
  XM(2, 1) = Y[19] * ((Y[8] - Y[7] * dltf) * squi * squf + (Y[10] - Y[9] * dltf) * squi * squf *
                                                                 dlti);
  XM(1, 2) = Y[19] * Y[9] / (squi * squf);
  XM(2, 2) = Y[19] * (Y[10] - Y[9] * dltf) * squf / squi;
  XM(1, 3) = Y[20] * (Y[7] * squi / squf + Y[9] * squi / squf * dlti);
  XM(2, 3) = Y[20] * ((Y[8] - Y[7] * dltf) * squi * squf + (Y[10] - Y[9] * dltf) * squi * squf *
                                                                 dlti);
  XM(1, 4) = Y[20] * Y[9] / (squi * squf);
  XM(2, 4) = Y[20] * (Y[10] - Y[9] * dltf) * squf / squi;
  XM(3, 1) = Y[21] * (Y[11] * squi / squf + Y[13] * squi / squf * dlti);
  XM(4, 1) = Y[21] * ((Y[12] - Y[11] * dltf) * squi * squf +
                      (Y[14] - Y[13] * dltf) * squi * squf * dlti);
  XM(3, 2) = Y[21] * Y[13] / (squi * squf);
  XM(4, 2) = Y[21] * (Y[14] - Y[13] * dltf) * squf / squi;
  XM(3, 3) = Y[22] * (Y[11] * squi / squf + Y[13] * squi / squf * dlti);
  XM(4, 3) = Y[22] * ((Y[12] - Y[11] * dltf) * squi * squf +
                      (Y[14] - Y[13] * dltf) * squi * squf * dlti);
  XM(3, 4) = Y[22] * Y[13] / (squi * squf);
  XM(4, 4) = Y[22] * (Y[14] - Y[13] * dltf) * squf / squi;
#undef XM
}

/* ---- TWS (type 106) linear map --------------------------------------- */
typedef struct {
  double zedge, escale, len, ww, theta0, theta2, qmcc;
  const double *F;
} tws_ctx;

/* getaxfldE_TWS (TWS.f90:350-466); its pi is a default-real 2*asin(1.0) */
static void tws_field(double z, const tws_ctx *c, double *ez1, double *ezp1, double *ez12,
                      double *ezp12) {
  const double *F = c->F - 1;
  const double pi = (double)(2 * asinf(1.0f));
  const double epstol = (double)1.0e-10f;
  *ez1 = 0.0; *ezp1 = 0.0; *ez12 = 0.0; *ezp12 = 0.0;
  if (!(((z >= c->zedge) && (z <= (c->zedge + c->len))) || (fabs(z - c->zedge) <= epstol) ||
        (fabs(z - c->zedge - c->len) <= epstol)))
    return;
  const double zlc = z - c->zedge;
  const int numpar1 = (int)(F[1] + 0.1);
  for (int w = 0; w < 2; w++) {
    const int k0 = w == 0 ? 0 : numpar1 + 4;
    const int numpar = (int)(F[k0 + 1] + 0.1);
    const double zstart = F[k0 + 2], zend = F[k0 + 3], zlength = F[k0 + 4];
    if (!(((zlc >= zstart) && (zlc <= zend)) || (fabs(zlc - zstart) <= epstol) ||
          (fabs(zlc - zend) <= epstol)))
      continue;
    const double zmid = zlength / 2;
    const double zz = z - c->zedge - zstart - zmid;
    const double zlen = zlength;
    const int ntmp = k0 + 4;
    double e = F[ntmp + 1] / 2, ep = 0.0;
    for (int i = 2; i <= (numpar - 1) / 2 + 1; i++) {
      e = e + F[2 * i - 2 + ntmp] * cos((i - 1) * 2 * pi * zz / zlen) +
          F[2 * i - 1 + ntmp] * sin((i - 1) * 2 * pi * zz / zlen);
      ep = ep + (i - 1) * 2 * pi / zlen *
                    (-F[2 * i - 2 + ntmp] * sin((i - 1) * 2 * pi * zz / zlen) +
                     F[2 * i - 1 + ntmp] * cos((i - 1) * 2 * pi * zz / zlen));
    }
    if (w == 0) { *ez1 = e * c->escale; *ezp1 = ep * c->escale; }
    else { *ez12 = e * c->escale; *ezp12 = ep * c->escale; }
  }
}

/* intfunc1_TWS (TWS.f90:231-340) */
static void tws_rhs(double t, const double *y, double *f, const void *vctx) {
  const tws_ctx *c = (const tws_ctx *)vctx;
  const double Scxl = PC.Scxl;
  double ez1, ezp1, ez12, ezp12;
  tws_field(t, c, &ez1, &ezp1, &ez12, &ezp12);
  f[0] = 0.0; f[1] = 0.0; f[2] = 0.0; f[3] = 0.0;
  const double gamma0 = -y[5];
  const double beta0 = sqrt(gamma0 * gamma0 - 1.) / gamma0;
  const double sinphi = sin(c->ww * y[4] + c->theta0);
  const double cosphi = cos(c->ww * y[4] + c->theta0);
  const double sinphi2 = sin(c->ww * y[4] + c->theta0 + c->theta2);
  const double cosphi2 = cos(c->ww * y[4] + c->theta0 + c->theta2);
  const double rfdsgn = ez1 * cosphi + ez12 * cosphi2;
  f[4] = 1.0 / (beta0 * Scxl);
  f[5] = -(c->qmcc * rfdsgn);
  const double q = c->qmcc * rfdsgn / (beta0 * beta0) / (gamma0 * gamma0);
  const double s11tmp = 0.5 * (1.0 + 0.5 * (gamma0 * gamma0)) * (q * q) +
                        c->qmcc * 0.5 / ((beta0 * beta0) * beta0) / ((gamma0 * gamma0) * gamma0) *
                            (ez1 * sinphi + ez12 * sinphi2) * c->ww / Scxl;
  double s55 =
      -(1.5 * c->qmcc / (beta0 * beta0) / gamma0 * (ezp1 * cosphi + ezp12 * cosphi2)) +
      ((beta0 * beta0) + 0.5) / ((beta0 * beta0) * beta0) / gamma0 * c->qmcc *
          (ez1 * sinphi + ez12 * sinphi2) * c->ww / Scxl +
      1.5 * (1.0 - 0.5 * (gamma0 * gamma0)) * (q * q);
  s55 = Scxl * s55;
  lin_rhs(y, f, s11tmp * Scxl, s11tmp * Scxl, s55);
}

/* maplinear_TWS (TWS.f90:129-229): coef = read3_Data's two series,
 * phase2_deg = Param(12) */
void orc_maplinear_tws(double t, double tau, double xm[36], double refpt[6], double zedge,
                       double escale, double freq, double phase_deg, int mapstp, double chg,
                       double mass, double length, double phase2_deg, int ncoef,
                       const double *coef) {
  const double Scxl = PC.Scxl;
  tws_ctx c;
  double y[18];
  (void)ncoef;
  c.zedge = zedge; c.escale = escale; c.len = length;
  c.ww = freq / PC.Scfreq;
  c.theta0 = phase_deg * (double)asinf(1.0f) / 90;
  c.theta2 = phase2_deg * (double)asinf(1.0f) / 90;
  c.qmcc = chg / mass;
  c.F = coef;
  memset(xm, 0, 36 * sizeof(double));
  y_init(y, refpt);
  const double h = tau / mapstp;
  double t0 = t;
  const double gi = -refpt[5];
  const double betai = sqrt(gi * gi - 1.) / gi;
  const double ui = gi * betai;
  const double squi = sqrt(ui);
  double s = sqrt(ui);
  const double sqi3 = s * s * s;
  double ein, e1in, ein2, e1in2;
  tws_field(t, &c, &ein, &e1in, &ein2, &e1in2);
  const double sinthi = sin(c.ww * refpt[4] + c.theta0);
  const double costhi = cos(c.ww * refpt[4] + c.theta0);
  const double sinthi2 = sin(c.ww * refpt[4] + c.theta0 + c.theta2);
  const double costhi2 = cos(c.ww * refpt[4] + c.theta0 + c.theta2);
  const double uprimi = c.qmcc * (ein * costhi + ein2 * costhi2) / betai;
  const double qpwi = 0.5 * c.qmcc * Scxl / (ui * c.ww);
  const double dlti = Scxl * (0.5 * uprimi / ui - qpwi * (e1in * sinthi + e1in2 * sinthi2));
  const double thli = 1.5 * Scxl * (uprimi / ui);
  rk6i(h, mapstp, &t0, y, tws_rhs, &c);
  refpt[4] = y[4];
  refpt[5] = y[5];
  const double gf = -refpt[5];
  const double betaf = sqrt(gf * gf - 1.) / gf;
  const double uf = gf * betaf;
  const double squf = sqrt(uf);
  s = sqrt(uf);
  const double sqf3 = s * s * s;
  double ef, e1f, ef2, e1f2;
  tws_field(t + tau, &c, &ef, &e1f, &ef2, &e1f2);
  const double sinthf = sin(c.ww * refpt[4] + c.theta0);
  const double costhf = cos(c.ww * refpt[4] + c.theta0);
  const double sinthf2 = sin(c.ww * refpt[4] + c.theta0 + c.theta2);
  const double costhf2 = cos(c.ww * refpt[4] + c.theta0 + c.theta2);
  const double uprimf = c.qmcc * (ef * costhf + ef2 * costhf2) / betaf;
  const double qpwf = 0.5 * c.qmcc * Scxl / (uf * c.ww);
  const double dltf = Scxl * (0.5 * uprimf / uf - qpwf * (e1f * sinthf + e1f2 * sinthf2));
  const double thlf = 1.5 * Scxl * (uprimf / uf);
  xm_assemble(xm, y, squi, squf, sqi3, sqf3, dlti, dltf, thli, thlf);
}

/* 6x6 loop of drift1_BeamBunch (BeamBunch.f90:310-320) */
void orc_apply_xm(double *pts, int n, const double xm[36]) {
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads)
  for (int i = 0; i < n; i++) {
    double temp[6];
    for (int j = 0; j < 6; j++) {
      double s = 0.0;
      for (int k = 0; k < 6; k++) s = s + P(i, k) * xm[j + 6 * k];
      temp[j] = s;
    }
    for (int j = 0; j < 6; j++) P(i, j) = temp[j];
  }
}

/* transfmapK_Quadrupole (Quadrupole.f90:509-607) */
/* transfUndulator_Quadrupole (Quadrupole.f90:611-665), kqlh = Param(2) */
void orc_undulator(double tau, double kqlh, double refpt[6], double *pts, int n) {
  const double Scxl = PC.Scxl;
  const double beta0 = sqrt(1.0 - 1.0 / (refpt[5] * refpt[5]));
  const double argh = tau * sqrt(kqlh);
  const double argh2 = argh * argh, argh4 = argh2 * argh2, argh6 = argh4 * argh2;
  const double sincargh = 1 - argh2 / 6 + argh4 / 120 - argh6 / 5040;
  const double r34h = tau * sincargh;
  const double xm11 = 1.0, xm12 = tau, xm21 = 0.0, xm22 = 1.0;
  const double xm33 = cos(tau * sqrt(kqlh));
  const double xm34 = r34h;
  const double xm43 = -sin(tau * sqrt(kqlh)) * sqrt(kqlh);
  const double xm44 = cos(tau * sqrt(kqlh));
  for (int i = 0; i < n; i++) {
    const double gam = -refpt[5] - P(i, 5);
    const double gambetz = sqrt(gam * gam - 1.0 - P(i, 1) * P(i, 1) - P(i, 3) * P(i, 3));
    const double betaz = gambetz / gam;
    const double t1 = xm11 * P(i, 0) + xm12 * P(i, 1) / gambetz / Scxl;
    const double t2 = gambetz * Scxl * xm21 * P(i, 0) + xm22 * P(i, 1);
    const double t3 = xm33 * P(i, 2) + xm34 * P(i, 3) / gambetz / Scxl;
    const double t4 = gambetz * Scxl * xm43 * P(i, 2) + xm44 * P(i, 3);
    const double t5 = P(i, 4) + (1.0 / betaz - 1.0 / beta0) * tau / Scxl;
    P(i, 0) = t1; P(i, 1) = t2; P(i, 2) = t3; P(i, 3) = t4; P(i, 4) = t5;
  }
  refpt[4] = refpt[4] + tau / beta0 / Scxl;
}

void orc_transfmapK(double tau, double kquad, double refpt[6], double *pts, int n,
                    double qmass) {
  const double Scxl = PC.Scxl;
  double gambet0 = sqrt(refpt[5] * refpt[5] - 1.0);
  double beta0 = sqrt(1.0 - 1.0 / (refpt[5] * refpt[5]));
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads)
  for (int i = 0; i < n; i++) {
    double gam, gambetz, betaz, kstr, rtkstr, rtkstrzz, cs, ss, t;
    double xm11, xm12, xm21, xm22, xm33, xm34, xm43, xm44, tmp[6];
    gam = -refpt[5] - P(i, 5);
    gambetz = sqrt(((gam * gam - 1.0) - P(i, 1) * P(i, 1)) - P(i, 3) * P(i, 3));
    betaz = gambetz / gam;
    gambetz = sqrt(gam * gam - 1.0);
    kstr = P(i, 6) / qmass * gambet0 / gambetz * kquad;
    rtkstr = sqrt(fabs(kstr));
    rtkstrzz = rtkstr * tau;
    if (kstr > 0.0) {
      cs = cos(rtkstrzz);
      ss = sin(rtkstrzz);
      xm11 = cs; xm12 = ss / rtkstr; xm21 = -(rtkstr * ss); xm22 = cs;
      t = exp(rtkstrzz);
      cs = (t * t + 1.0) / (t + t);
      ss = (t * t - 1.0) / (t + t);
      xm33 = cs; xm34 = ss / rtkstr; xm43 = ss * rtkstr; xm44 = cs;
    } else if (kstr < 0.0) {
      t = exp(rtkstrzz);
      cs = (t * t + 1.0) / (t + t);
      ss = (t * t - 1.0) / (t + t);
      xm11 = cs; xm12 = ss / rtkstr; xm21 = rtkstr * ss; xm22 = cs;
      cs = cos(rtkstrzz);
      ss = sin(rtkstrzz);
      xm33 = cs; xm34 = ss / rtkstr; xm43 = -(ss * rtkstr); xm44 = cs;
    } else {
      xm11 = 1.0; xm12 = tau; xm21 = 0.0; xm22 = 1.0;
      xm33 = 1.0; xm34 = tau; xm43 = 0.0; xm44 = 1.0;
    }
    tmp[0] = xm11 * P(i, 0) + xm12 * P(i, 1) / gambetz / Scxl;
    tmp[1] = gambetz * Scxl * xm21 * P(i, 0) + xm22 * P(i, 1);
    tmp[2] = xm33 * P(i, 2) + xm34 * P(i, 3) / gambetz / Scxl;
    tmp[3] = gambetz * Scxl * xm43 * P(i, 2) + xm44 * P(i, 3);
    tmp[4] = P(i, 4) + (1.0 / betaz - 1.0 / beta0) * tau / Scxl;
    tmp[5] = P(i, 5);
    for (int j = 0; j < 6; j++) P(i, j) = tmp[j];
  }
  refpt[4] = refpt[4] + tau / beta0 / Scxl;
}

/* ideal RF gap branch of drift1_BeamBunch (BeamBunch.f90:324-440) */
void orc_ideal_rf(double *pts, int n, double refptcl[6], double mass, double tau,
                  double vgrad, double rffreq, double phase_deg, int nst, int nseg,
                  int ihlf) {
  const double Scxl = PC.Scxl;
  double vtmp = vgrad / mass;
  double harm = rffreq / PC.Scfreq;
  double phi0lc = phase_deg * asin(1.0) / 90;
  double gam0, gambet, beta0, gambet0;
  if (nst == 1 && ihlf % 2 == 0) {
    gam0 = -refptcl[5];
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads)
    for (int i = 0; i < n; i++) {
      double gam = gam0 - P(i, 5);
      double gambetz = sqrt(((gam * gam - 1.0) - P(i, 1) * P(i, 1)) - P(i, 3) * P(i, 3));
      double phi = P(i, 4) * harm + phi0lc;
      double cosphi = cos(phi);
      double vg = vtmp * cosphi * Scxl;
      P(i, 1) = P(i, 1) - 0.5 * vg * gambetz / gam * P(i, 0);
      P(i, 3) = P(i, 3) - 0.5 * vg * gambetz / gam * P(i, 2);
    }
  }
  gam0 = -refptcl[5];
  gambet = sqrt(gam0 * gam0 - 1.0);
  beta0 = gambet / gam0;
  refptcl[4] = refptcl[4] + 0.5 * tau / (Scxl * beta0);
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads)
  for (int i = 0; i < n; i++) {
    double gami_1 = gam0 - P(i, 5);
    double gambeti_1 = sqrt(gami_1 * gami_1 - 1.0);
    double gambetzi_1 = sqrt(((gami_1 * gami_1 - 1.0) - P(i, 1) * P(i, 1)) - P(i, 3) * P(i, 3));
    double phi = P(i, 4) * harm + phi0lc;
    double dgami = tau * vtmp * cos(phi);
    double gami_2 = gami_1 + dgami;
    double gambeti_2 = sqrt(gami_2 * gami_2 - 1.0);
    double fact;
    if (fabs(vtmp) < 1.0e-10)
      fact = tau / Scxl;
    else
      fact = gambeti_1 / dgami * log(gambeti_2 / gambeti_1) * tau / Scxl;
    P(i, 0) = P(i, 0) + fact * P(i, 1) / gambetzi_1;
    P(i, 2) = P(i, 2) + fact * P(i, 3) / gambetzi_1;
    P(i, 4) = P(i, 4) + (tau / Scxl) / (gambet * gambet * gambet) * P(i, 5);
  }
  refptcl[5] = refptcl[5] - tau * vtmp * cos(phi0lc);
  gam0 = -refptcl[5];
  gambet0 = sqrt(gam0 * gam0 - 1.0);
  beta0 = gambet0 / gam0;
  refptcl[4] = refptcl[4] + 0.5 * tau / (Scxl * beta0);
  if (nst == nseg && ihlf % 2 == 1) {
    gam0 = -refptcl[5];
    double c0 = cos(phi0lc);
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads)
    for (int i = 0; i < n; i++) {
      double gam = gam0 - P(i, 5);
      double gambetz = sqrt(((gam * gam - 1.0) - P(i, 1) * P(i, 1)) - P(i, 3) * P(i, 3));
      double phi = P(i, 4) * harm + phi0lc;
      double cosphi = cos(phi);
      double vg = vtmp * cosphi * Scxl;
      P(i, 1) = P(i, 1) + 0.5 * vg * gambetz / gam * P(i, 0);
      P(i, 3) = P(i, 3) + 0.5 * vg * gambetz / gam * P(i, 2);
      phi = P(i, 4) * harm + phi0lc;
      P(i, 5) = P(i, 5) + (double)(2 * nseg) * tau * vtmp * (c0 - cos(phi));
    }
  }
}

/* Fpol_Dipole (Dipole.f90:466-526) */
void orc_fpol(double h0, double h1, double tanphi, double tanphib, double k1,
              double psi, double *pts, double ang, int n, double gam0, double qm0) {
  const double Scxl = PC.Scxl;
  double tanphi2 = tanphi * tanphi;
  double secphi2 = 1.0 + tanphi2;
  double secphi = 1.0 / cos(ang);
  double secphi3 = secphi2 * secphi;
  double secphib2 = 1. + tanphib * tanphib;
  double beta0 = sqrt(1.0 - 1.0 / (gam0 * gam0));
  double gambet = beta0 * gam0;
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads)
  for (int i = 0; i < n; i++) {
    double a[6], gamn, gambetz;
    P(i, 0) = P(i, 0) * Scxl;
    gamn = gam0 - P(i, 5);
    gambetz = sqrt(((gamn * gamn - 1.0) - P(i, 1) * P(i, 1)) - P(i, 3) * P(i, 3));
    P(i, 1) = P(i, 1) / gambetz;
    P(i, 2) = P(i, 2) * Scxl;
    P(i, 3) = P(i, 3) / gambetz;
    P(i, 4) = -(P(i, 4) * beta0 * Scxl);
    P(i, 5) = -(P(i, 5) / beta0 / gambet) - (P(i, 6) - qm0) / qm0;
    double x = P(i, 0), xp = P(i, 1), y = P(i, 2), yp = P(i, 3), d = P(i, 5);
    a[0] = x - 0.5 * h0 * tanphi2 * (x * x) + 0.5 * h0 * secphi2 * (y * y);
    a[1] = h0 * tanphi * x + xp + h0 * tanphi2 * x * xp +
           (0.5 * h0 * h1 * secphi3 + k1 * tanphi) * (x * x) -
           (0.5 * h0 * h1 * secphi3 + k1 * tanphi - (h0 * h0) * tanphi * tanphi2 -
            0.5 * (h0 * h0) * tanphi) * (y * y) -
           h0 * tanphi2 * y * yp - h0 * tanphi * x * d;
    a[2] = y + h0 * tanphi2 * x * y;
    a[3] = -(h0 * tanphib * y) + yp - h0 * tanphi2 * x * yp - h0 * secphi2 * xp * y -
           (h0 * h1 * secphi3 + 2 * k1 * tanphi) * x * y +
           (h0 * tanphi - h0 * psi * secphib2) * y * d;
    a[4] = P(i, 4);
    a[5] = P(i, 5);
    gambetz = sqrt(gamn * gamn - 1.0) / sqrt((a[1] * a[1] + a[3] * a[3]) + 1);
    P(i, 0) = a[0] / Scxl;
    P(i, 1) = a[1] * gambetz;
    P(i, 2) = a[2] / Scxl;
    P(i, 3) = a[3] * gambetz;
    P(i, 4) = -a[4] / Scxl / beta0;
    P(i, 5) = -(beta0 * gambet * (a[5] + (P(i, 6) - qm0) / qm0));
  }
}

/* Bpol_Dipole (Dipole.f90:528-591) */
void orc_bpol(double h0, double h1, double tanphi, double tanphib, double k1,
              double psi, double *pts, double ang, int n, double gam0, double qm0) {
  const double Scxl = PC.Scxl;
  double tanphi2 = tanphi * tanphi;
  double secphi2 = 1.0 + tanphi2;
  double secphi = 1.0 / cos(ang);
  double secphi3 = secphi2 * secphi;
  double secphib2 = 1. + tanphib * tanphib;
  double beta0 = sqrt(1.0 - 1.0 / (gam0 * gam0));
  double gambet = beta0 * gam0;
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads)
  for (int i = 0; i < n; i++) {
    double a[6], gamn, gambetz;
    P(i, 0) = P(i, 0) * Scxl;
    gamn = gam0 - P(i, 5);
    gambetz = sqrt(((gamn * gamn - 1.0) - P(i, 1) * P(i, 1)) - P(i, 3) * P(i, 3));
    P(i, 1) = P(i, 1) / gambetz;
    P(i, 2) = P(i, 2) * Scxl;
    P(i, 3) = P(i, 3) / gambetz;
    P(i, 4) = -(P(i, 4) * beta0 * Scxl);
    P(i, 5) = -(P(i, 5) / beta0 / gambet) - (P(i, 6) - qm0) / qm0;
    double x = P(i, 0), xp = P(i, 1), y = P(i, 2), yp = P(i, 3), d = P(i, 5);
    a[0] = x + 0.5 * h0 * tanphi2 * (x * x) - 0.5 * h0 * secphi2 * (y * y);
    a[1] = h0 * tanphi * x + xp - h0 * tanphi2 * x * xp +
           (0.5 * h0 * h1 * secphi3 + k1 * tanphi - (h0 * h0) * tanphi2 * tanphi / 2) * (x * x) -
           (0.5 * h0 * h1 * secphi3 + k1 * tanphi + (h0 * h0) * tanphi * tanphi2 / 2) * (y * y) +
           h0 * tanphi2 * y * yp - h0 * tanphi * x * d;
    a[2] = y - h0 * tanphi2 * x * y;
    a[3] = -(h0 * tanphib * y) + yp + h0 * tanphi2 * x * yp + h0 * secphi2 * xp * y -
           (h0 * h1 * secphi3 + 2 * k1 * tanphi - (h0 * h0) * secphi2 * tanphi) * x * y +
           (h0 * tanphi - h0 * psi * secphib2) * y * d;
    a[4] = P(i, 4);
    a[5] = P(i, 5);
    gambetz = sqrt(gamn * gamn - 1.0) / sqrt((a[1] * a[1] + a[3] * a[3]) + 1);
    P(i, 0) = a[0] / Scxl;
    P(i, 1) = a[1] * gambetz;
    P(i, 2) = a[2] / Scxl;
    P(i, 3) = a[3] * gambetz;
    P(i, 4) = -a[4] / Scxl / beta0;
    P(i, 5) = -(beta0 * gambet * (a[5] + (P(i, 6) - qm0) / qm0));
  }
}

/* Sector_Dipole: 2nd-order Brown map (Dipole.f90:693-788) */
void orc_sector(double len, double beta0, double h0, double k1, double *pts, int n,
                double qm0) {
  (void)k1;
  const double Scxl = PC.Scxl;
  double rho = 1.0 / h0, theta = len * h0;
  double st = sin(theta), ct = cos(theta), sh = sin(theta / 2.0);
  double R11 = ct, R12 = rho * st, R16 = rho * (1.0 - ct), R21 = -st / rho, R22 = ct, R26 = st;
  double R51 = -R26, R52 = -R16, R56 = rho * (st - (beta0 * beta0) * theta);
  double T111 = -(st * st) / (2.0 * rho), T112 = st * ct, T116 = st * st;
  double T122 = rho * ct * (sh * sh);
  double T126 = -(rho * st * (-1.0 + ct));
  double T166 = -(rho * (st * st)) / 2.0;
  double T144 = rho * (-1.0 + ct) / 2.0;
  double T216 = st / rho, T222 = -st / 2.0, T266 = -st, T244 = -st / 2.0;
  double T314 = st, T324 = 2.0 * rho * (sh * sh), T346 = rho * (theta - st);
  double T522 = -(0.5 * rho * st), T544 = T522, T526 = rho * (ct - 1.0);
  double gambet = beta0 / sqrt(1.0 - beta0 * beta0);
  double gam2 = 1.0 / (1.0 - beta0 * beta0);
  double gam0 = sqrt(gam2);
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads)
  for (int i = 0; i < n; i++) {
    double gami = -P(i, 5) + gam0;
    double gambeti = sqrt(gami * gami - 1.0);
    double gambetx = P(i, 1), gambety = P(i, 3);
    double gambetz = sqrt((gambeti * gambeti - gambetx * gambetx) - gambety * gambety);
    double x0 = P(i, 0) * Scxl, xp0 = P(i, 1) / gambetz, y0 = P(i, 2) * Scxl;
    double yp0 = P(i, 3) / gambetz, z0 = -(P(i, 4) * beta0 * Scxl);
    double eta = -(P(i, 5) / beta0 / gambet) - (P(i, 6) - qm0) / qm0;
    double a0 = R11 * x0 + R12 * xp0 + R16 * eta + T111 * (x0 * x0) + T112 * x0 * xp0 +
                T116 * x0 * eta + T122 * (xp0 * xp0) + T126 * xp0 * eta + T166 * (eta * eta) +
                T144 * (yp0 * yp0);
    double a1 = R21 * x0 + R22 * xp0 + R26 * eta + T216 * x0 * eta + T222 * (xp0 * xp0) +
                T266 * (eta * eta) + T244 * (yp0 * yp0);
    double a2 = y0 + len * yp0 + T314 * x0 * yp0 + T324 * xp0 * yp0 + T346 * yp0 * eta;
    double a3 = yp0;
    double a4 = R51 * x0 + R52 * xp0 + z0 + R56 * eta + T522 * (xp0 * xp0) +
                T544 * (yp0 * yp0) + T526 * xp0 * eta;
    double a5 = eta;
    double xp = a1, yp = a3;
    gambetz = gambeti / sqrt((xp * xp + yp * yp) + 1.0);
    P(i, 0) = a0 / Scxl;
    P(i, 1) = a1 * gambetz;
    P(i, 2) = a2 / Scxl;
    P(i, 3) = a3 * gambetz;
    P(i, 4) = -a4 / Scxl / beta0;
    P(i, 5) = -(beta0 * gambet * (a5 + (P(i, 6) - qm0) / qm0));
  }
}

/* ------------------------------------------------------------------ */
/* conv1st_BeamBunch, Flagbc=1 (BeamBunch.f90:1252-1352, 1657-1663) */
int orc_conv1st(double *pts, int n, double *current, int *npt,
                const double refptcl[6], double xrad, double yrad,
                double ptrange[6]) {
  /* pilc = 2.0*asin(1.0) in default (single) precision */
  const double pilc = (double)(2.0f * asinf(1.0f));
  const double xl = PC.Scxl;
  double gam = -refptcl[5];
  double rad = (xrad + yrad) / 2;
  int ilost = 0;
  for (int k = 0; k < 3; k++) {
    ptrange[2 * k] = (double)1.0e20f;
    ptrange[2 * k + 1] = -(double)1.0e20f;
  }
  for (int i0 = 0; i0 < n; i0++) {
    int i = i0 - ilost;
    int ntmp5 = (int)(P(i0, 4) / pilc);
    double tmp5 = P(i0, 4) - ntmp5 * pilc;
    P(i0, 4) = tmp5 - (ntmp5 % 2) * pilc;
    double rcpgammai = 1.0 / (-P(i0, 5) + gam);
    double tmpbet = 1.0 - rcpgammai * rcpgammai * ((1 + P(i0, 1) * P(i0, 1)) + P(i0, 3) * P(i0, 3));
    double betai = sqrt(fabs(tmpbet));
    double tmpx = P(i0, 0) * xl;
    P(i, 0) = (P(i0, 0) - P(i0, 1) * P(i0, 4) * rcpgammai) * xl;
    double tmp0 = fmin(tmpx, P(i, 0));
    if (ptrange[0] > tmp0) ptrange[0] = tmp0;
    tmp0 = fmax(tmpx, P(i, 0));
    if (ptrange[1] < tmp0) ptrange[1] = tmp0;
    P(i, 1) = P(i0, 1);
    double tmpy = P(i0, 2) * xl;
    P(i, 2) = (P(i0, 2) - P(i0, 3) * P(i0, 4) * rcpgammai) * xl;
    tmp0 = fmin(tmpy, P(i, 2));
    if (ptrange[2] > tmp0) ptrange[2] = tmp0;
    tmp0 = fmax(tmpy, P(i, 2));
    if (ptrange[3] < tmp0) ptrange[3] = tmp0;
    P(i, 3) = P(i0, 3);
    P(i, 4) = -(gam * betai * P(i0, 4) * xl);
    if (ptrange[4] > P(i, 4)) ptrange[4] = P(i, 4);
    if (ptrange[5] < P(i, 4)) ptrange[5] = P(i, 4);
    P(i, 5) = P(i0, 5);
    double radtest = sqrt(P(i, 0) * P(i, 0) + P(i, 2) * P(i, 2));
    if (radtest >= rad || tmpbet <= 0.0) ilost++;
    P(i, 6) = P(i0, 6);
    P(i, 7) = P(i0, 7);
    P(i, 8) = P(i0, 8);
  }
  int nplc = n - ilost;
  int nptot = nplc; /* MPI_ALLREDUCE over one rank */
  *current = *current * nptot / *npt;
  *npt = nptot;
  return nplc;
}

/* update_CompDom, Flagbc=1 (CompDom.f90:509-557, 614-622, 803-819) */
void orc_update_compdom(const double ptrange[6], const int mesh[3],
                        double range[6], double msize[3]) {
  for (int k = 0; k < 3; k++) {
    double t1 = ptrange[2 * k], t2 = ptrange[2 * k + 1];
    /* eps = 1.0/(Meshnum-3.0) evaluated in default (single) precision */
    double eps = (double)(1.0f / ((float)mesh[k] - 3.0f));
    double mn = t1 - eps * (t2 - t1);
    double mx = t2 + eps * (t2 - t1);
    range[2 * k] = mn;
    range[2 * k + 1] = mx;
    msize[k] = (mx - mn) / (mesh[k] - 1);
  }
}

/* deposit_BeamBunch (BeamBunch.f90:3678-3768) */
void orc_deposit(const double *pts, int n, const int mesh[3], const double range[6],
                 const double msize[3], double *rho, int *counts, long long *cells) {
  const int nx = mesh[0], ny = mesh[1], nz = mesh[2];
  const double hx = msize[0], hy = msize[1], hz = msize[2];
  const double hxi = 1.0 / hx, hyi = 1.0 / hy, hzi = 1.0 / hz;
  const double xmin = range[0], ymin = range[2], zmin = range[4];
  const size_t G = (size_t)nx * ny * nz;
  memset(rho, 0, G * sizeof(double));
  if (counts) memset(counts, 0, G * sizeof(int));
#define R(i, j, k) rho[((i)-1) + (size_t)nx * (((j)-1) + (size_t)ny * ((k)-1))]
  for (int i = 0; i < n; i++) {
    int ix = (int)((P(i, 0) - xmin) * hxi + 1);
    double ab = ((xmin - P(i, 0)) + ix * hx) * hxi;
    int jx = (int)((P(i, 2) - ymin) * hyi + 1);
    double cd = ((ymin - P(i, 2)) + jx * hy) * hyi;
    int kx = (int)((P(i, 4) - zmin) * hzi + 1);
    double ef = ((zmin - P(i, 4)) + kx * hz) * hzi;
    int ix1 = ix + 1, jx1 = jx + 1, kx1 = kx + 1;
    if (ix < 1 || ix1 > nx || jx < 1 || jx1 > ny || kx < 1 || kx1 > nz) {
      if (cells) cells[i] = -1;
      continue;
    }
    double w = P(i, 7);
    R(ix, jx, kx) = R(ix, jx, kx) + ab * cd * ef * w;
    R(ix, jx1, kx) = R(ix, jx1, kx) + ab * (1.0 - cd) * ef * w;
    R(ix, jx1, kx1) = R(ix, jx1, kx1) + ab * (1.0 - cd) * (1.0 - ef) * w;
    R(ix, jx, kx1) = R(ix, jx, kx1) + ab * cd * (1.0 - ef) * w;
    R(ix1, jx, kx1) = R(ix1, jx, kx1) + (1.0 - ab) * cd * (1.0 - ef) * w;
    R(ix1, jx1, kx1) = R(ix1, jx1, kx1) + (1.0 - ab) * (1.0 - cd) * (1.0 - ef) * w;
    R(ix1, jx1, kx) = R(ix1, jx1, kx) + (1.0 - ab) * (1.0 - cd) * ef * w;
    R(ix1, jx, kx) = R(ix1, jx, kx) + (1.0 - ab) * cd * ef * w;
    long long c = (ix - 1) + (long long)nx * ((jx - 1) + (long long)ny * (kx - 1));
    if (counts) counts[c]++;
    if (cells) cells[i] = c;
  }
#undef R
}

/* ------------------------------------------------------------------ */
/* greenf1tIntnew before its FFTs (Field.f90:392-428) */
void orc_igf(int nx, int ny, int nz, double hx, double hy, double hz, double *grn) {
  const int ax = nx + 2, ay = ny + 2, az = nz + 2;
  double *tmp = (double *)malloc((size_t)ax * ay * az * sizeof(double));
#define T(i, j, k) tmp[((i)-1) + (size_t)ax * (((j)-1) + (size_t)ay * ((k)-1))]
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads)
  for (int k0 = 1; k0 <= az; k0++)
    for (int j0 = 1; j0 <= ay; j0++)
      for (int i0 = 1; i0 <= ax; i0++) {
        double v1 = (i0 - 1) * hx - hx / 2;
        double v2 = (j0 - 1) * hy - hy / 2;
        double v3 = (k0 - 1) * hz - hz / 2;
        double rr = sqrt(v1 * v1 + v2 * v2 + v3 * v3);
        double aa = -(v3 * v3 * atan(v1 * v2 / (v3 * rr)) / 2);
        double bb = -(v2 * v2 * atan(v1 * v3 / (v2 * rr)) / 2);
        double cc = -(v1 * v1 * atan(v2 * v3 / (v1 * rr)) / 2);
        double dd = v2 * v3 * log(v1 + rr);
        double ee = v1 * v3 * log(v2 + rr);
        double ff = v1 * v2 * log(v3 + rr);
        double gg2 = aa + bb + cc + dd + ee + ff;
        T(i0, j0, k0) = gg2 / (hx * hy * hz);
      }
  const int gx = nx + 1, gy = ny + 1;
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads)
  for (int k0 = 1; k0 <= nz + 1; k0++)
    for (int j0 = 1; j0 <= ny + 1; j0++)
      for (int i0 = 1; i0 <= nx + 1; i0++)
        grn[(i0 - 1) + (size_t)gx * ((j0 - 1) + (size_t)gy * (k0 - 1))] =
            T(i0 + 1, j0 + 1, k0 + 1) - T(i0, j0 + 1, k0 + 1) - T(i0 + 1, j0, k0 + 1) +
            T(i0, j0, k0 + 1) - T(i0 + 1, j0 + 1, k0) + T(i0, j0 + 1, k0) +
            T(i0 + 1, j0, k0) - T(i0, j0, k0);
#undef T
  free(tmp);
}

/* radix-2 complex FFT, in place, on n points spaced by stride; sign -1 or +1,
 * unnormalised.  Any correct FFT reproduces the reference's FFTPACK
 * convolution (FFT.f90:26-250) to rounding. */
static void fft1(double complex *a, int n, size_t stride, int sign, const double complex *tw) {
  /* tw[k] = exp(-2 pi i k / n), k < n/2 */
  for (int i = 1, j = 0; i < n; i++) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      double complex t = a[i * stride];
      a[i * stride] = a[j * stride];
      a[j * stride] = t;
    }
  }
  for (int len = 2; len <= n; len <<= 1) {
    int step = n / len;
    for (int i = 0; i < n; i += len)
      for (int k = 0; k < len / 2; k++) {
        double complex w = tw[k * step];
        if (sign > 0) w = conj(w);
        double complex u = a[(i + k) * stride];
        double complex v = a[(i + k + len / 2) * stride] * w;
        a[(i + k) * stride] = u + v;
        a[(i + k + len / 2) * stride] = u - v;
      }
  }
}

static double complex *twiddles(int n) {
  double complex *tw = (double complex *)malloc((size_t)(n / 2 + 1) * sizeof(double complex));
  for (int k = 0; k < n / 2; k++) {
    double a = -2.0 * PC.Pi * k / n;
    tw[k] = cos(a) + I * sin(a);
  }
  return tw;
}

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* 3D FFT of a (n1,n2,n3) complex array (column-major).  Forward passes run
 * x, y, z and skip the lines that are still zero (input nonzero only for
 * j < ey, k < ez); inverse passes run z, y, x and skip the lines the cropped
 * output does not need.  ey = n2, ez = n3 transforms everything. */
static void fft3(double complex *a, int n1, int n2, int n3, int ey, int ez, int sign,
                 int inverse) {
  double complex *t1 = twiddles(n1), *t2 = twiddles(n2), *t3 = twiddles(n3);
  for (int pass = 0; pass < 3; pass++) {
    int axis = inverse ? 2 - pass : pass;
    if (axis == 0) {
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads) collapse(2)
      for (int k = 0; k < ez; k++)
        for (int j = 0; j < ey; j++) fft1(a + (size_t)n1 * (j + (size_t)n2 * k), n1, 1, sign, t1);
    } else if (axis == 1) {
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads) collapse(2)
      for (int k = 0; k < ez; k++)
        for (int i = 0; i < n1; i++) fft1(a + i + (size_t)n1 * n2 * k, n2, n1, sign, t2);
    } else {
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads) collapse(2)
      for (int j = 0; j < n2; j++)
        for (int i = 0; i < n1; i++) fft1(a + i + (size_t)n1 * j, n3, (size_t)n1 * n2, sign, t3);
    }
  }
  free(t1); free(t2); free(t3);
}

/* openBC3D + greenf1tIntnew's mirroring (Field.f90:239-331, 430-515):
 * phi = IFFT(FFT(rho_zero_padded) * FFT(G_even_extended)) / (n1 n2 n3), cropped. */
int orc_poisson_open(int nx, int ny, int nz, double hx, double hy, double hz,
                     double *rho) {
  const int n1 = 2 * nx, n2 = 2 * ny, n3 = 2 * nz;
  if (!is_pow2(n1) || !is_pow2(n2) || !is_pow2(n3)) return -1;
  const size_t N = (size_t)n1 * n2 * n3;
  double complex *r = (double complex *)calloc(N, sizeof(double complex));
  double complex *g = (double complex *)malloc(N * sizeof(double complex));
  double *grn = (double *)malloc((size_t)(nx + 1) * (ny + 1) * (nz + 1) * sizeof(double));
  if (!r || !g || !grn) { free(r); free(g); free(grn); return -2; }
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        r[i + (size_t)n1 * (j + (size_t)n2 * k)] = rho[i + (size_t)nx * (j + (size_t)ny * k)];
  orc_igf(nx, ny, nz, hx, hy, hz, grn);
  for (int k = 0; k < n3; k++) {
    int kk = k <= nz ? k : n3 - k;
    for (int j = 0; j < n2; j++) {
      int jj = j <= ny ? j : n2 - j;
      for (int i = 0; i < n1; i++) {
        int ii = i <= nx ? i : n1 - i;
        g[i + (size_t)n1 * (j + (size_t)n2 * k)] =
            grn[ii + (size_t)(nx + 1) * (jj + (size_t)(ny + 1) * kk)];
      }
    }
  }
  fft3(r, n1, n2, n3, ny, nz, -1, 0);
  fft3(g, n1, n2, n3, n2, n3, -1, 0);
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads)
  for (size_t q = 0; q < N; q++) r[q] = r[q] * g[q];
  fft3(r, n1, n2, n3, ny, nz, +1, 1);
  const double scale = 1.0 / ((double)n1 * n2 * n3);
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        rho[i + (size_t)nx * (j + (size_t)ny * k)] =
            creal(r[i + (size_t)n1 * (j + (size_t)n2 * k)]) * scale;
  free(r); free(g); free(grn);
  return 0;
}

void orc_poisson_direct(int nx, int ny, int nz, double hx, double hy, double hz,
                        const double *rho, double *phi) {
  double *grn = (double *)malloc((size_t)(nx + 1) * (ny + 1) * (nz + 1) * sizeof(double));
  orc_igf(nx, ny, nz, hx, hy, hz, grn);
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        double s = 0.0;
        for (int c = 0; c < nz; c++)
          for (int b = 0; b < ny; b++)
            for (int a = 0; a < nx; a++)
              s += rho[a + (size_t)nx * (b + (size_t)ny * c)] *
                   grn[abs(i - a) + (size_t)(nx + 1) * (abs(j - b) + (size_t)(ny + 1) * abs(k - c))];
        phi[i + (size_t)nx * (j + (size_t)ny * k)] = s;
      }
  free(grn);
}

/* ------------------------------------------------------------------ */
/* cvbkforth1st_BeamBunch (BeamBunch.f90:1667-1701) */
void orc_cvbkforth1st(double *pts, int n, const double refptcl[6]) {
  const double xl = PC.Scxl, xk = 1 / xl;
  double gamma0 = -refptcl[5];
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads)
  for (int i = 0; i < n; i++) {
    double rcpgammai = 1.0 / (-P(i, 5) + gamma0);
    double betai = sqrt(1.0 - rcpgammai * rcpgammai * ((1 + P(i, 1) * P(i, 1)) + P(i, 3) * P(i, 3)));
    P(i, 4) = P(i, 4) * xk / (-(gamma0 * betai));
    P(i, 0) = P(i, 0) * xk + P(i, 1) * P(i, 4) * rcpgammai;
    P(i, 2) = P(i, 2) * xk + P(i, 3) * P(i, 4) * rcpgammai;
  }
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads)
  for (int i = 0; i < n; i++) {
    double rcpgammai = 1.0 / (-P(i, 5) + gamma0);
    double betai = sqrt(1.0 - rcpgammai * rcpgammai * ((1 + P(i, 1) * P(i, 1)) + P(i, 3) * P(i, 3)));
    P(i, 0) = P(i, 0) * xl;
    P(i, 2) = P(i, 2) * xl;
    P(i, 4) = -(gamma0 * betai * P(i, 4) * xl);
  }
}

/* kick1_BeamBunch field differences (BeamBunch.f90:1784-2005) + scatter1
 * (BeamBunch.f90:2041-2181), one rank, Flagbc=1 */
void orc_kick1(double *pts, int n, const double *phi, const int mesh[3],
               const double range[6], const double msize[3], double gam,
               double curr, double tau, double mass, double chrg, double *eg) {
  orc_kick1w(pts, n, phi, mesh, range, msize, gam, curr, tau, mass, chrg, eg, NULL);
}

/* kick1wake_BeamBunch (BeamBunch.f90:4694-5046): kick1 with a per-plane
 * field added to the node fields before the gather (BeamBunch.f90:5015-5033);
 * wfield = {dEx[nz], dEy[nz], dEz[nz]} in grid-field units (orc_wake_field),
 * NULL for none. */
/* The Lorentz integrator's kick (kick2/scatter2_BeamBunch, BeamBunch.f90:
 * 2187-3071, the analytic-field branch) in element e with zedge = Param(1):
 * 0 drift, 1 quadrupole, 2 constant focusing, 3 solenoid, 101..104 the RF
 * cavities over read3_Data's Fourier coefficients (e->zdat, e->ndata); z =
 * the kick's position, tg = refptcl(5) there, qmi = the bunch's Pts1(7)
 * (each particle's own row 7 enters the update, as rays(7,n) does) */
typedef struct {
  const orc_elem *e;
  double zedge, z, tg, qmi;
  /* kick2wake (BeamBunch.f90:5048-5410): the per-plane wake {Ex, Ey,
   * Ez}[nz] as the wake routines return it, or NULL */
  const double *wraw;
  /* the RF cavities' terms at z that getfldpts_DTL / getfldpts_CCL
   * compute once per call (DTL.f90:858-958, CCL.f90:722-809) */
  double bgrad, ez1, ezp1, f1, f1p, ww, theta0, xl, clite;
  /* SolRF / TWS (SolRF.f90:482-628, TWS.f90): inside the element, the
   * first series' terms (on1), and the second series' (on2): TWS's second
   * wave at theta0 + theta2, or SolRF's solenoid (bscale times the sums) */
  int inside, on1, on2;
  double xlrep, tsc, w1[4], w2[4], sol[4], theta2;
  /* EMfld 110 with discrete x-y-z data (Param(13) = 1, Param(14) = 2):
   * getfld6xyz_EMfld's field plane at z (complex Ex, Ey, Ez, Bx, By, Bz per
   * node, x fastest), the grid and the RF constants */
  double *plane;
  int enx, eny;
  double exmin, ehx, ehxi, eymin, ehy, ehyi, escale, eww, etheta0;
} lorentz_kick;

static void kick_common(double *pts, int n, const double *phi, const int mesh[3],
                        const double range[6], const double msize[3], double gam, double curr,
                        double tau, double mass, double chrg, double *eg, const double *wfield,
                        const lorentz_kick *lz);

void orc_kick1w(double *pts, int n, const double *phi, const int mesh[3],
                const double range[6], const double msize[3], double gam,
                double curr, double tau, double mass, double chrg, double *eg,
                const double *wfield) {
  kick_common(pts, n, phi, mesh, range, msize, gam, curr, tau, mass, chrg, eg, wfield, NULL);
}

/* read3_Data's coefficient Fcoef(i), i from 1, with the count made odd by
 * a trailing zero (Data.f90:348-409) */
static double fcoef(const orc_elem *e, int i) { return i <= e->ndata ? e->zdat[i - 1] : 0.0; }

/* the on-axis part of getfld_DTL / CCDTL / CCL / SC (DTL.f90:769-855,
 * CCDTL.f90, CCL.f90:525-606, SC.f90): the drift-tube quadrupoles'
 * gradient (DTL only), Ez and its derivatives from the Fourier series at
 * z - zmid, and the radial-expansion factors; pi and c are the reference's
 * default-real literals there */
static void lz_rf_axis(lorentz_kick *lz) {
  const orc_elem *e = lz->e;
  const double clite = (double)299792458.0f;
  const double pi = (double)(2 * asinf(1.0f));
  const double escale = e->val[0];
  const double len = e->length;
  const double zmid = lz->zedge + len / 2;
  lz->ww = e->val[1] / PC.Scfreq;
  lz->xl = PC.Scxl / lz->ww;
  lz->theta0 = e->val[2] * (double)asinf(1.0f) / 90;
  lz->clite = clite;
  lz->bgrad = 0.0;
  if (e->type == 101) {
    const double zz = lz->z - lz->zedge;
    const double len1 = e->val[5], bgrad1 = e->val[6];
    const double len2 = len - e->val[7], bgrad2 = e->val[8];
    if (zz < len1)
      lz->bgrad = bgrad1;
    else if (zz < len2)
      lz->bgrad = 0.0;
    else
      lz->bgrad = bgrad2;
  }
  const double zz = lz->z - zmid;
  const int nd = e->ndata % 2 == 0 ? e->ndata + 1 : e->ndata;
  double ez1 = fcoef(e, 1) / 2, ezp1 = 0.0, ezpp1 = 0.0, ezppp = 0.0;
  for (int i = 2; i <= (nd - 1) / 2 + 1; i++) {
    const double a = fcoef(e, 2 * i - 2), b = fcoef(e, 2 * i - 1);
    const double arg = (i - 1) * 2 * pi * zz / len;
    const double k = (i - 1) * 2 * pi / len;
    ez1 = ez1 + a * cos(arg) + b * sin(arg);
    ezp1 = ezp1 + k * (-(a * sin(arg)) + b * cos(arg));
    ezpp1 = ezpp1 + k * k * (-(a * cos(arg)) - b * sin(arg));
    ezppp = ezppp + k * k * k * (a * sin(arg) - b * cos(arg));
  }
  ez1 = ez1 * escale;
  ezp1 = ezp1 * escale;
  ezpp1 = ezpp1 * escale;
  ezppp = ezppp * escale;
  lz->ez1 = ez1;
  lz->ezp1 = ezp1;
  lz->f1 = -((ezpp1 + ez1 / lz->xl / lz->xl) / 4);
  lz->f1p = -((ezppp + ezp1 / lz->xl / lz->xl) / 4);
}

/* one Fourier series of getfld_SolRF / getfld_TWS: npar terms from
 * Fcoef(ntmp+1) at zz over the period zlen; Ez and three derivatives */
static void lz_series(const orc_elem *e, int ntmp, int npar, double zz, double zlen, double pi,
                      double out[4]) {
  double ez1 = fcoef(e, ntmp + 1) / 2, ezp1 = 0.0, ezpp1 = 0.0, ezppp = 0.0;
  for (int i = 2; i <= (npar - 1) / 2 + 1; i++) {
    const double a = fcoef(e, 2 * i - 2 + ntmp), b = fcoef(e, 2 * i - 1 + ntmp);
    ez1 = ez1 + a * cos((i - 1) * 2 * pi * zz / zlen) + b * sin((i - 1) * 2 * pi * zz / zlen);
    ezp1 = ezp1 + (i - 1) * 2 * pi / zlen *
                      (-(a * sin((i - 1) * 2 * pi * zz / zlen)) +
                       b * cos((i - 1) * 2 * pi * zz / zlen));
    const double k = (i - 1) * 2 * pi / zlen;
    ezpp1 = ezpp1 + k * k *
                        (-(a * cos((i - 1) * 2 * pi * zz / zlen)) -
                         b * sin((i - 1) * 2 * pi * zz / zlen));
    ezppp = ezppp + k * k * k *
                        (a * sin((i - 1) * 2 * pi * zz / zlen) -
                         b * cos((i - 1) * 2 * pi * zz / zlen));
  }
  out[0] = ez1;
  out[1] = ezp1;
  out[2] = ezpp1;
  out[3] = ezppp;
}

/* the on-axis part of getfld_SolRF / getfld_TWS at z */
static void lz_rfw_axis(lorentz_kick *lz) {
  const orc_elem *e = lz->e;
  const double clite = (double)299792458.0f;
  const double pi = (double)(2 * asinf(1.0f));
  const double zedge = lz->zedge, z = lz->z, escale = e->val[0], len = e->length;
  lz->inside = z > zedge && z < zedge + len;
  if (!lz->inside) return;
  lz->ww = e->val[1] * 2 * pi;
  lz->xlrep = lz->ww / clite;
  lz->theta0 = e->val[2] * (double)asinf(1.0f) / 90;
  lz->tsc = 2 * pi * PC.Scfreq;
  lz->clite = clite;
  const double zlc = z - zedge;
  const int numpar1 = (int)(fcoef(e, 1) + 0.1);
  const double zstart1 = fcoef(e, 2), zend1 = fcoef(e, 3), zlength1 = fcoef(e, 4);
  double t[4];
  lz->on1 = zlc >= zstart1 && zlc <= zend1;
  if (lz->on1) {
    const double zmid = zlength1 / 2;
    lz_series(e, 4, numpar1, z - zedge - zstart1 - zmid, zlength1, pi, t);
    const double ez1 = t[0] * escale, ezp1 = t[1] * escale;
    const double ezpp1 = t[2] * escale, ezppp = t[3] * escale;
    lz->w1[0] = ez1;
    lz->w1[1] = ezp1;
    lz->w1[2] = -((ezpp1 + ez1 * lz->xlrep * lz->xlrep) / 4);
    lz->w1[3] = -((ezppp + ezp1 * lz->xlrep * lz->xlrep) / 4);
  }
  const int numpar2 = (int)(fcoef(e, 5 + numpar1) + 0.1);
  const double zstart2 = fcoef(e, 6 + numpar1), zend2 = fcoef(e, 7 + numpar1);
  const double zlength2 = fcoef(e, 8 + numpar1);
  lz->theta2 = e->val[10] * pi / 180;
  lz->on2 = zlc >= zstart2 && zlc <= zend2;
  if (lz->on2) {
    const double zmid = zlength2 / 2;
    lz_series(e, numpar1 + 8, numpar2, z - zedge - zstart2 - zmid, zlength2, pi, t);
    if (e->type == 106) {
      const double ez1 = t[0] * escale, ezp1 = t[1] * escale;
      const double ezpp1 = t[2] * escale, ezppp = t[3] * escale;
      lz->w2[0] = ez1;
      lz->w2[1] = ezp1;
      lz->w2[2] = -((ezpp1 + ez1 * lz->xlrep * lz->xlrep) / 4);
      lz->w2[3] = -((ezppp + ezp1 * lz->xlrep * lz->xlrep) / 4);
    } else {
      for (int i = 0; i < 4; i++) lz->sol[i] = t[i];
    }
  }
}

/* read4_Data's grid of element 110 (Data.f90:415-554): e->zdat holds the
 * three header records (xmin, xmax, NxIntvRfg; ymin, ymax, NyIntvRfg; zmin,
 * zmax, NzIntvRfg) as nine doubles, e->edat the complex Ex, Ey, Ez, Bx, By,
 * Bz of each grid node (re, im pairs, twelve doubles per node) in file
 * order (x fastest, then y, then z), e->ndata the node count.
 * getfld6xyz_EMfld (EMfld.f90:854-916): the plane at z, linear between the
 * first two and the last two planes, quadratic (three planes) elsewhere. */
#define EMG(c, i, j, k) e->edat[12 * ((size_t)((i)-1) + (size_t)(nxp) * \
                                      ((size_t)((j)-1) + (size_t)(nyp) * ((size_t)((k)-1)))) + (c)]
static void lz_emfld_plane(lorentz_kick *lz) {
  const orc_elem *e = lz->e;
  const double *hd = e->zdat;
  const int nxi = (int)(hd[2] + 0.1), nyi = (int)(hd[5] + 0.1), nzi = (int)(hd[8] + 0.1);
  const int nxp = nxi + 1, nyp = nyi + 1;
  lz->enx = nxi;
  lz->eny = nyi;
  lz->exmin = hd[0];
  lz->ehx = (hd[1] - hd[0]) / nxi;
  lz->ehxi = 1.0 / lz->ehx;
  lz->eymin = hd[3];
  lz->ehy = (hd[4] - hd[3]) / nyi;
  lz->ehyi = 1.0 / lz->ehy;
  lz->escale = e->val[0];
  lz->eww = e->val[1] / PC.Scfreq;
  lz->etheta0 = e->val[2] * (double)asinf(1.0f) / 90;
  lz->plane = (double *)malloc((size_t)12 * nxp * nyp * sizeof(double));
  const double hz = (hd[7] - hd[6]) / nzi;
  const double zz = lz->z - lz->zedge;
  int iz = (int)(zz / hz + 1);
  if (iz == nzi + 1) iz = iz - 1;
  for (int j = 1; j <= nyp; j++)
    for (int i = 1; i <= nxp; i++)
      for (int c = 0; c < 12; c++) {
        double v;
        if (iz == 1 || iz == nzi) {
          const int iz1 = iz + 1;
          const double ef = (iz * hz - zz) / hz;
          v = EMG(c, i, j, iz) * ef + EMG(c, i, j, iz1) * (1.0 - ef);
        } else {
          const double ab = (zz - (iz - 1) * hz) / hz;
          const int iz1 = iz + 1;
          int iz2;
          double wix, wix1, wix2;
          if (ab <= 0.5) {
            iz2 = iz - 1;
            wix = 0.75 - ab * ab;
            wix1 = (0.5 + ab) * (0.5 + ab) / 2;
            wix2 = (0.5 - ab) * (0.5 - ab) / 2;
          } else {
            iz2 = iz + 2;
            wix = (1.5 - ab) * (1.5 - ab) / 2;
            wix1 = 0.75 - (1 - ab) * (1 - ab);
            wix2 = (ab - 0.5) * (ab - 0.5) / 2;
          }
          v = EMG(c, i, j, iz) * wix + EMG(c, i, j, iz1) * wix1 + EMG(c, i, j, iz2) * wix2;
        }
        lz->plane[12 * ((size_t)(i - 1) + (size_t)nxp * (j - 1)) + c] = v;
      }
}
#undef EMG

/* one complex field component c (0..5) of the plane at node (i, j), 1-based */
static void emp(const lorentz_kick *lz, int c, int i, int j, double *re, double *im) {
  const double *q = lz->plane + 12 * ((size_t)(i - 1) + (size_t)(lz->enx + 1) * (j - 1));
  *re = q[2 * c];
  *im = q[2 * c + 1];
}

/* scatter2's quadratic weights along one axis of the x-y grid
 * (BeamBunch.f90:2804-2860): node i, its neighbour i1 = i+1 and a third
 * node i2, with the one-sided forms at the first and the last interval */
static void emfld_w(int i, double ab, int nint, int *i2, double w[3]) {
  if (i == 1 && ab <= 0.5) {
    *i2 = i;
    w[0] = 0.75 - ab * ab;
    w[1] = (0.5 + ab) * (0.5 + ab) / 2;
    w[2] = 0.0;
  } else if (i == nint && ab > 0.5) {
    *i2 = i;
    w[0] = (1.5 - ab) * (1.5 - ab) / 2;
    w[1] = 0.75 - (1 - ab) * (1 - ab);
    w[2] = 0.0;
  } else if (ab <= 0.5) {
    *i2 = i - 1;
    w[0] = 0.75 - ab * ab;
    w[1] = (0.5 + ab) * (0.5 + ab) / 2;
    w[2] = (0.5 - ab) * (0.5 - ab) / 2;
  } else {
    *i2 = i + 2;
    w[0] = (1.5 - ab) * (1.5 - ab) / 2;
    w[1] = 0.75 - (1 - ab) * (1 - ab);
    w[2] = (ab - 0.5) * (ab - 0.5) / 2;
  }
}

/* the field of element 110 at (x, y) [m] and time tt (scatter2 with
 * FlagDisc = 1, FlagCart = 2, BeamBunch.f90:2794-2880): nine-point
 * quadratic interpolation of the complex plane, times escale e^{i(ww tt +
 * theta0)}, real part */
static void lz_emfld(const lorentz_kick *lz, const double pos[4], double f[6]) {
  const double xx = pos[0], yy = pos[1];
  const int ix = (int)((xx - lz->exmin) * lz->ehxi + 1), ix1 = ix + 1;
  const int iy = (int)((yy - lz->eymin) * lz->ehyi + 1), iy1 = iy + 1;
  const double ab = (xx - lz->exmin - (ix - 1) * lz->ehx) * lz->ehxi;
  const double cd = (yy - lz->eymin - (iy - 1) * lz->ehy) * lz->ehyi;
  int ix2, iy2;
  double wx[3], wy[3];
  emfld_w(ix, ab, lz->enx, &ix2, wx);
  emfld_w(iy, cd, lz->eny, &iy2, wy);
  const double ph = lz->eww * pos[3] + lz->etheta0;
  const double tr = lz->escale * cos(ph), ti = lz->escale * sin(ph);
  const int ii[3] = {ix, ix1, ix2}, jj[3] = {iy, iy1, iy2};
  for (int c = 0; c < 6; c++) {
    double sr = 0.0, si = 0.0;
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) {
        double vr, vi;
        emp(lz, c, ii[a], jj[b], &vr, &vi);
        if (a == 0 && b == 0) {
          sr = vr * wx[a] * wy[b];
          si = vi * wx[a] * wy[b];
        } else {
          sr = sr + vr * wx[a] * wy[b];
          si = si + vi * wx[a] * wy[b];
        }
      }
    f[c] = sr * tr - si * ti;
  }
}

/* scatter2's ez0 of element 110 (BeamBunch.f90:2612-2632): bilinear in
 * the plane at x = y = 0 times escale e^{i(ww tg + theta0)}, real part */
static double lz_emfld_ez0(const lorentz_kick *lz) {
  const double xx = 0.0, yy = 0.0;
  const int ix = (int)((xx - lz->exmin) / lz->ehx + 1), ix1 = ix + 1;
  const double efx = (lz->exmin - xx + ix * lz->ehx) / lz->ehx;
  const int iy = (int)((yy - lz->eymin) / lz->ehy + 1), iy1 = iy + 1;
  const double efy = (lz->eymin - yy + iy * lz->ehy) / lz->ehy;
  const double ph = lz->eww * lz->tg + lz->etheta0;
  const double tr = lz->escale * cos(ph), ti = lz->escale * sin(ph);
  double r[4], im[4];
  emp(lz, 2, ix, iy, &r[0], &im[0]);
  emp(lz, 2, ix, iy1, &r[1], &im[1]);
  emp(lz, 2, ix1, iy, &r[2], &im[2]);
  emp(lz, 2, ix1, iy1, &r[3], &im[3]);
  const double wa[4] = {efx, efx, 1.0 - efx, 1.0 - efx}, wb[4] = {efy, 1.0 - efy, efy, 1.0 - efy};
  double sr = 0.0, si = 0.0;
  for (int k = 0; k < 4; k++) {
    sr = k ? sr + r[k] * wa[k] * wb[k] : r[k] * wa[k] * wb[k];
    si = k ? si + im[k] * wa[k] * wb[k] : im[k] * wa[k] * wb[k];
  }
  return sr * tr - si * ti;
}

static lorentz_kick lz_make(const orc_elem *e, double zedge, double z, double tg, double qmi) {
  lorentz_kick lz;
  memset(&lz, 0, sizeof(lz));
  lz.e = e;
  lz.zedge = zedge;
  lz.z = z;
  lz.tg = tg;
  lz.qmi = qmi;
  lz.wraw = NULL;
  if (e->type >= 101 && e->type <= 104) lz_rf_axis(&lz);
  if (e->type == 105 || e->type == 106) lz_rfw_axis(&lz);
  if (e->type == 110) lz_emfld_plane(&lz);
  return lz;
}

/* getfldfrgAna2_Quadrupole (Quadrupole.f90:456-506): the Enge profile of
 * the gradient at zz from the quadrupole's entrance and its first two
 * derivatives */
static void quad_ana2(const lorentz_kick *lz, double zz, double *bgrad, double *bgradp,
                      double *bgradpp) {
  const double c1 = -0.00004, c2 = 4.518219;
  const double bb = lz->e->val[0];
  const double dd = 2 * lz->e->val[2];
  const double z10 = (lz->e->length - lz->e->val[1]) / 2;
  const double z20 = lz->e->length - z10;
  const double z3 = z10 + 1.5 * dd;
  const double z4 = z20 - 1.5 * dd;
  double tmpz, s1, s2, s3, s4, tmp1, q;
  if (zz < z3) {
    tmpz = -(zz - z10) / dd;
    s1 = c1 + c2 * tmpz;
    *bgrad = bb / (1.0 + exp(s1));
    s2 = -c2 / dd;
  } else if (zz > z4) {
    tmpz = (zz - z20) / dd;
    s1 = c1 + c2 * tmpz;
    *bgrad = bb / (1.0 + exp(s1));
    s2 = c2 / dd;
  } else {
    *bgrad = bb;
    *bgradp = 0.0;
    *bgradpp = 0.0;
    return;
  }
  tmp1 = exp(s1) * s2;
  q = 1.0 + exp(s1);
  *bgradp = -bb * tmp1 / (q * q);
  s3 = 0.0;
  s4 = exp(s1) * (s3 + s2 * s2);
  *bgradpp = bb * (-s4 / (q * q) + 2 * tmp1 * tmp1 / (q * q * q));
}

/* getfld_BeamLineElem (BeamLineElem.f90:827-867) at pos = (x [m], y [m],
 * z [m], t) for the elements above: getfld_DriftTube (DriftTube.f90:
 * 290-305), getfld_Quadrupole (Quadrupole.f90:369-402), getfld_ConstFoc
 * (ConstFoc.f90:297-322, with its placeholder qmcc = gambetz = 1),
 * getfld_Sol (Sol.f90:391-435) and the RF cavities (scatter2 takes the
 * DTL's and CCL's through getfldpts_*, the same values); f = (Ex, Ey, Ez,
 * Bx, By, Bz) */
static void lz_getfld(const lorentz_kick *lz, const double pos[4], double f[6]) {
  for (int i = 0; i < 6; i++) f[i] = 0.0;
  const double zz = pos[2] - lz->zedge;
  if (lz->e->type == 110) {
    lz_emfld(lz, pos, f);
  } else if (lz->e->type == 1) {
    double bgrad = lz->e->val[0], bgradp = 0.0, bgradpp = 0.0;
    if (lz->e->val[1] > 1.0e-5) quad_ana2(lz, zz, &bgrad, &bgradp, &bgradpp);
    if (lz->e->val[1] > 0.0) {
      f[3] = bgrad * pos[1] -
             bgradpp * (pos[1] * pos[1] * pos[1] + 3 * (pos[0] * pos[0]) * pos[1]) / 12;
      f[4] = bgrad * pos[0] -
             bgradpp * (pos[0] * pos[0] * pos[0] + 3 * pos[0] * (pos[1] * pos[1])) / 12;
      f[5] = bgradp * pos[0] * pos[1];
    } else {
      f[3] = bgrad * pos[1];
      f[4] = bgrad * pos[0];
    }
  } else if (lz->e->type == 2) {
    const double qmcc = 1.0, gambetz = 1.0, pz = gambetz;
    f[2] = lz->e->val[2] * pos[3] * pz * pz * pz * PC.Scxl / qmcc;
    f[3] = -(lz->e->val[0] * pos[1] * pz / qmcc / PC.Clight);
    f[4] = lz->e->val[1] * pos[0] * pz / qmcc / PC.Clight;
  } else if (lz->e->type == 3) {
    const double x0 = lz->e->val[2], x02 = 2 * x0, b0 = lz->e->val[0];
    if (zz >= 0.0 && zz < x02) {
      const double bb = b0 / x02, bgrad = bb;
      f[3] = -(bgrad / 2 * pos[0]);
      f[4] = -(bgrad / 2 * pos[1]);
      f[5] = bb * zz;
    } else if (zz >= x02 && zz <= lz->e->length - x02) {
      f[5] = b0;
    } else if (zz > lz->e->length - x02 && zz <= lz->e->length) {
      const double bb = -b0 / x02, bgrad = bb, zshift = lz->e->length - x02;
      f[3] = -(bgrad / 2 * pos[0]);
      f[4] = -(bgrad / 2 * pos[1]);
      f[5] = b0 + bb * (zz - zshift);
    }
  } else if (lz->e->type >= 101 && lz->e->type <= 104) {
    /* the per-particle part of getfld_DTL / getfldpts_DTL (DTL.f90:
     * 836-855, 932-956) and of CCDTL, CCL, SC, with the on-axis terms of
     * lz_rf_axis; the DTL adds its drift-tube quadrupoles' B = G (y, x, 0) */
    const double tt = pos[3];
    const double tmpcos = cos(lz->ww * tt + lz->theta0);
    const double tmpsin = sin(lz->ww * tt + lz->theta0);
    const double r2 = pos[0] * pos[0] + pos[1] * pos[1];
    const double xlc = lz->xl * lz->clite;
    const double tmpex = -(pos[0] * (lz->ezp1 / 2 + lz->f1p * r2 / 4) * tmpcos);
    const double tmpey = -(pos[1] * (lz->ezp1 / 2 + lz->f1p * r2 / 4) * tmpcos);
    const double tmpez = (lz->ez1 + lz->f1 * r2) * tmpcos;
    const double tmpbx = pos[1] / xlc * (lz->ez1 / 2 + lz->f1 * r2 / 4) * tmpsin;
    const double tmpby = -(pos[0] / xlc * (lz->ez1 / 2 + lz->f1 * r2 / 4) * tmpsin);
    if (lz->e->type == 101) {
      f[3] = lz->bgrad * pos[1];
      f[4] = lz->bgrad * pos[0];
    }
    f[0] = f[0] + tmpex;
    f[1] = f[1] + tmpey;
    f[2] = f[2] + tmpez;
    f[3] = f[3] + tmpbx;
    f[4] = f[4] + tmpby;
  } else if (lz->e->type == 5) {
    /* getfld_Multipole (Multipole.f90:403-452), MAD notation, with
     * getfldfrg_Multipole's interpolation (455-480) for Param(4) > 0 */
    const int idpole = (int)(lz->e->val[0] + 0.1);
    double bgrad;
    if (lz->e->val[2] > 0.0) {
      int klo = 1, khi = lz->e->ndata;
      const double *zd = lz->e->zdat - 1, *ed = lz->e->edat - 1;
      while (khi - klo > 1) {
        const int k = (khi + klo) / 2;
        if (zd[k] > zz)
          khi = k;
        else
          klo = k;
      }
      const double hstep = zd[khi] - zd[klo];
      const double slope = (ed[khi] - ed[klo]) / hstep;
      bgrad = ed[klo] + slope * (zz - zd[klo]);
    } else {
      bgrad = lz->e->val[1];
    }
    const double x = pos[0], y = pos[1];
    if (idpole == 2) {
      f[3] = bgrad * y * x;
      f[4] = bgrad * (x * x - y * y) / 2;
    } else if (idpole == 3) {
      f[3] = bgrad * (3 * (x * x) * y - y * y * y) / 6;
      f[4] = bgrad * (x * x * x - 3 * x * (y * y)) / 6;
    } else {
      f[3] = bgrad * (x * x * x * y - x * (y * y * y)) / 6;
      f[4] = bgrad * ((x * x) * (x * x) - 6 * (x * x) * (y * y) + (y * y) * (y * y)) / 24;
    }
  } else if ((lz->e->type == 105 || lz->e->type == 106) && lz->inside) {
    /* the per-particle lines of getfld_SolRF (SolRF.f90:482-628) and
     * getfld_TWS (TWS.f90) with the on-axis terms of lz_rfw_axis */
    const double tt = pos[3] / lz->tsc;
    const double r2 = pos[0] * pos[0] + pos[1] * pos[1];
    for (int w = 0; w < 2; w++) {
      const double *c = w == 0 ? lz->w1 : lz->w2;
      if (w == 0 ? !lz->on1 : !(lz->on2 && lz->e->type == 106)) continue;
      const double ph = w == 0 ? lz->ww * tt + lz->theta0 : lz->ww * tt + lz->theta0 + lz->theta2;
      const double tmpcos = cos(ph), tmpsin = sin(ph);
      const double tmpex = -(pos[0] * (c[1] / 2 + c[3] * r2 / 4) * tmpcos);
      const double tmpey = -(pos[1] * (c[1] / 2 + c[3] * r2 / 4) * tmpcos);
      const double tmpez = (c[0] + c[2] * r2) * tmpcos;
      const double tmpbx = pos[1] * lz->xlrep / lz->clite * (c[0] / 2 + c[2] * r2 / 4) * tmpsin;
      const double tmpby =
          -(pos[0] * lz->xlrep / lz->clite * (c[0] / 2 + c[2] * r2 / 4) * tmpsin);
      f[0] = f[0] + tmpex;
      f[1] = f[1] + tmpey;
      f[2] = f[2] + tmpez;
      f[3] = f[3] + tmpbx;
      f[4] = f[4] + tmpby;
    }
    if (lz->on2 && lz->e->type == 105) {
      const double bscale = lz->e->val[10];
      const double ez1 = lz->sol[0], ezp1 = lz->sol[1], ezpp1 = lz->sol[2], ezppp = lz->sol[3];
      f[3] = f[3] - bscale * ezp1 / 2 * pos[0] + bscale * ezppp * pos[0] * r2 / 16;
      f[4] = f[4] - bscale * ezp1 / 2 * pos[1] + bscale * ezppp * pos[1] * r2 / 16;
      f[5] = f[5] + bscale * ez1 - bscale * ezpp1 * r2 / 4;
    }
  }
}

/* scatter2's ez0: the element's Ez on axis at the reference time */
static double lz_ez0(const lorentz_kick *lz) {
  if (lz->e->type == 110) return lz_emfld_ez0(lz);
  const double pos[4] = {0.0, 0.0, lz->z, lz->tg};
  double f[6];
  lz_getfld(lz, pos, f);
  return f[2];
}

/* the implicit Lorentz update of scatter2/scatter20 (BeamBunch.f90:3019-3065
 * and 3478-3531) for a space-charge field (exn, eyn, ezn) [grid units] and
 * the element's field at the particle, plus scatter2wake's wake (wx, wy, wz)
 * at the particle (BeamBunch.f90:5634-5636, 5885-5887); p = one particle's
 * Pts1 */
static void lorentz_update(double *p, double exn, double eyn, double ezn, double gam, double tau,
                           double mass, double chrg, double ez0, const lorentz_kick *lz,
                           double wx, double wy, double wz) {
  const double xl = PC.Scxl, Clight = PC.Clight;
  const double tmpscale2 = Clight * Clight * (double)1.0e-7f;
  const double beta0 = sqrt(gam * gam - 1.0) / gam;
  const double qmcc = chrg / mass;
  const double tmpgamma0 = gam + 0.5 * tau * qmcc * ez0;
  const double pos[4] = {p[0] * xl, p[2] * xl, lz->z, p[4] + lz->tg};
  double extfld[6];
  lz_getfld(lz, pos, extfld);
  const double ex = tmpscale2 * exn + extfld[0] + wx;
  const double ey = tmpscale2 * eyn + extfld[1] + wy;
  const double ez = tmpscale2 * ezn + extfld[2] + wz;
  const double bx = -(beta0 / Clight * tmpscale2 * eyn) + extfld[3];
  const double by = beta0 / Clight * tmpscale2 * exn + extfld[4];
  const double bz = extfld[5];
  const double r7 = p[6];  /* rays(7,n): the particle's q/m (multiple charge states) */
  const double tmp12 = -tau * Clight * bz * r7 / 2;
  const double tmp13 = tau * ex * r7 / 2;
  const double tmp23 = tau * ey * r7 / 2;
  const double tmp1 = tmpgamma0 * ex * tau * r7;
  const double tmp2 = Clight * by * tau * r7;
  const double tmp3 = tmpgamma0 * ey * tau * r7;
  const double tmp4 = Clight * bx * tau * r7;
  const double tmp5 = (ez0 * qmcc - ez * r7) * tau;
  double pz = sqrt((gam - p[5]) * (gam - p[5]) - 1.0 - p[1] * p[1] - p[3] * p[3]);
  const double p1 = p[1], p2 = p[3], p3 = p[5];
  for (int ii = 1; ii <= 2; ii++) {
    const double a12 = tmp12 / pz, a13 = tmp13 / pz, a23 = tmp23 / pz;
    const double b1 = p1 - a12 * p2 - a13 * p3 + tmp1 / pz - tmp2;
    const double b2 = a12 * p1 + p2 - a23 * p3 + tmp3 / pz + tmp4;
    const double b3 = -(a13 * p1) - a23 * p2 + p3 + tmp5;
    const double det = 1 + a12 * a12 - a13 * a13 - a23 * a23;
    const double s11 = 1 - a23 * a23, s12 = -a12 + a13 * a23, s13 = a12 * a23 - a13;
    const double s21 = a12 + a13 * a23, s22 = 1 - a13 * a13, s23 = -a23 - a13 * a12;
    const double s31 = -(a12 * a23) - a13, s32 = -a23 + a12 * a13, s33 = 1 + a12 * a12;
    p[1] = (s11 * b1 + s12 * b2 + s13 * b3) / det;
    p[3] = (s21 * b1 + s22 * b2 + s23 * b3) / det;
    p[5] = (s31 * b1 + s32 * b2 + s33 * b3) / det;
    const double tmpgamma00 = gam + tau * qmcc * ez0;
    const double tmpsq2 =
        (tmpgamma00 - p[5]) * (tmpgamma00 - p[5]) - 1.0 - p[1] * p[1] - p[3] * p[3];
    if (tmpsq2 > 0.0) pz = 0.5 * pz + 0.5 * sqrt(tmpsq2);
  }
}

/* kick2_BeamBunch (BeamBunch.f90:2187-2508) with scatter2, one rank,
 * Flagbc=1, or kick2wake with scatter2wake when wraw (the per-plane wake
 * {Ex, Ey, Ez}[nz] of the wake routines) is given; returns the new
 * gamma0 = gam + tau qmcc ez0 (refptcl(6) = -it) */
double orc_kick2(double *pts, int n, const double *phi, const int mesh[3], const double range[6],
                 const double msize[3], double gam, double curr, double tau, double mass,
                 double chrg, const orc_elem *e, double zedge, double z, double tg, double qmi,
                 const double *wraw) {
  lorentz_kick lz = lz_make(e, zedge, z, tg, qmi);
  lz.wraw = wraw;
  kick_common(pts, n, phi, mesh, range, msize, gam, curr, tau, mass, chrg, NULL, NULL, &lz);
  const double g = gam + tau * (chrg / mass) * lz_ez0(&lz);
  free(lz.plane);
  return g;
}

/* kick2_BeamBunch without current: scatter20 (BeamBunch.f90:3075-3531),
 * the element's field alone on the stored coordinates; returns the new
 * gamma0 */
double orc_lorentz_nosc(double *pts, int n, double gam, double tau, double mass, double chrg,
                        const orc_elem *e, double zedge, double z, double tg, double qmi) {
  const lorentz_kick lz = lz_make(e, zedge, z, tg, qmi);
  const double ez0 = lz_ez0(&lz);
  for (int q = 0; q < n; q++)
    lorentz_update(&P(q, 0), 0.0, 0.0, 0.0, gam, tau, mass, chrg, ez0, &lz, 0.0, 0.0, 0.0);
  free(lz.plane);
  return gam + tau * (chrg / mass) * ez0;
}

static void kick_common(double *pts, int n, const double *phi, const int mesh[3],
                        const double range[6], const double msize[3], double gam, double curr,
                        double tau, double mass, double chrg, double *eg, const double *wfield,
                        const lorentz_kick *lz) {
  if (curr < 1.0e-20) return;
  const double lz_ez0v = lz ? lz_ez0(lz) : 0.0;
  const int nx = mesh[0], ny = mesh[1], nz = mesh[2];
  const size_t G = (size_t)nx * ny * nz;
  double *egx = eg ? eg : (double *)malloc(3 * G * sizeof(double));
  double *egy = egx + G, *egz = egy + G;
  const double hxi = 1.0 / msize[0], hyi = 1.0 / msize[1], hzi = 1.0 / msize[2];
  const double hx = msize[0], hy = msize[1], hz = msize[2];
#define IDX(i, j, k) (((i)-1) + (size_t)nx * (((j)-1) + (size_t)ny * ((k)-1)))
#define PHI(i, j, k) phi[IDX(i, j, k)]
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++) {
      egx[IDX(1, j, k)] = hxi * (PHI(1, j, k) - PHI(2, j, k));
      for (int i = 2; i <= nx - 1; i++)
        egx[IDX(i, j, k)] = 0.5 * hxi * (PHI(i - 1, j, k) - PHI(i + 1, j, k));
      egx[IDX(nx, j, k)] = hxi * (PHI(nx - 1, j, k) - PHI(nx, j, k));
    }
  for (int k = 1; k <= nz; k++) {
    for (int i = 1; i <= nx; i++) egy[IDX(i, 1, k)] = hyi * (PHI(i, 1, k) - PHI(i, 2, k));
    for (int j = 2; j <= ny - 1; j++)
      for (int i = 1; i <= nx; i++)
        egy[IDX(i, j, k)] = 0.5 * hyi * (PHI(i, j - 1, k) - PHI(i, j + 1, k));
    for (int i = 1; i <= nx; i++)
      egy[IDX(i, ny, k)] = hyi * (PHI(i, ny - 1, k) - PHI(i, ny, k));
  }
  for (int j = 1; j <= ny; j++)
    for (int i = 1; i <= nx; i++) egz[IDX(i, j, 1)] = hzi * (PHI(i, j, 1) - PHI(i, j, 2));
  for (int k = 2; k <= nz - 1; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++)
        egz[IDX(i, j, k)] = 0.5 * hzi * (PHI(i, j, k - 1) - PHI(i, j, k + 1));
  for (int j = 1; j <= ny; j++)
    for (int i = 1; i <= nx; i++)
      egz[IDX(i, j, nz)] = hzi * (PHI(i, j, nz - 1) - PHI(i, j, nz));
  if (wfield)
    for (int k = 1; k <= nz; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
          egx[IDX(i, j, k)] = egx[IDX(i, j, k)] + wfield[k - 1];
          egy[IDX(i, j, k)] = egy[IDX(i, j, k)] + wfield[nz + k - 1];
          egz[IDX(i, j, k)] = egz[IDX(i, j, k)] + wfield[2 * nz + k - 1];
        }

  /* scatter1_BeamBunch constants (BeamBunch.f90:2066-2084) */
  const double tmpscale = curr / PC.Scfreq;
  const double twopi = 2.0 * PC.Pi;
  const double fpei = PC.Clight * PC.Clight * (double)1.0e-7f;
  const double xk = 1 / PC.Scxl;
  const double bet = sqrt(gam * gam - 1.0) / gam;
  const double bbyk = bet / xk;
  const double gambet = gam * bet;
  const double brho = gambet / (PC.Clight * chrg) * mass;
  const double vz0 = bet * PC.Clight;
  const double perv0 = 2.0 * curr * fpei / (brho * vz0 * vz0 * gam * gam);
  const double xycon = 0.5 * perv0 * gambet * bbyk * twopi / tmpscale;
  const double tcon = bet * xycon * (gam * gam);
  const double xmin = range[0], ymin = range[2], zmin = range[4];
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads)
  for (int q = 0; q < n; q++) {
    int ix = (int)((P(q, 0) - xmin) * hxi + 1);
    double ab = ((xmin - P(q, 0)) + ix * hx) * hxi;
    int jx = (int)((P(q, 2) - ymin) * hyi + 1);
    double cd = ((ymin - P(q, 2)) + jx * hy) * hyi;
    int kx = (int)((P(q, 4) - zmin) * hzi + 1);
    double ef = ((zmin - P(q, 4)) + kx * hz) * hzi;
    int ix1 = ix + 1, jx1 = jx + 1, kx1 = kx + 1;
    double E[3];
    const double *grids[3] = {egx, egy, egz};
    for (int c = 0; c < 3; c++) {
      const double *e = grids[c];
      E[c] = e[IDX(ix, jx, kx)] * ab * cd * ef + e[IDX(ix, jx1, kx)] * ab * (1. - cd) * ef +
             e[IDX(ix, jx1, kx1)] * ab * (1. - cd) * (1.0 - ef) +
             e[IDX(ix, jx, kx1)] * ab * cd * (1.0 - ef) +
             e[IDX(ix1, jx, kx1)] * (1.0 - ab) * cd * (1.0 - ef) +
             e[IDX(ix1, jx1, kx1)] * (1.0 - ab) * (1.0 - cd) * (1.0 - ef) +
             e[IDX(ix1, jx1, kx)] * (1.0 - ab) * (1.0 - cd) * ef +
             e[IDX(ix1, jx, kx)] * (1.0 - ab) * cd * ef;
    }
    double exn = E[0] * gam, eyn = E[1] * gam, ezn = E[2];
    double rcpgammai = 1.0 / (-P(q, 5) + gam);
    double tmpsq = 1.0 - rcpgammai * rcpgammai * ((1 + P(q, 1) * P(q, 1)) + P(q, 3) * P(q, 3));
    double betai = sqrt(tmpsq);
    if (lz) {
      /* scatter2wake's wake at the particle: linear in z over the gather
       * cell's planes (BeamBunch.f90:5634-5636) */
      double wx = 0.0, wy = 0.0, wz = 0.0;
      if (lz->wraw) {
        const double *w = lz->wraw;
        wx = w[kx - 1] * ef + w[kx1 - 1] * (1.0 - ef);
        wy = w[nz + kx - 1] * ef + w[nz + kx1 - 1] * (1.0 - ef);
        wz = w[2 * nz + kx - 1] * ef + w[2 * nz + kx1 - 1] * (1.0 - ef);
      }
      /* back from t to z (BeamBunch.f90:2766-2771), then the element's field
       * at the particle and the implicit Lorentz update iterated twice
       * (BeamBunch.f90:3019-3065) */
      P(q, 4) = P(q, 4) * xk / (-gam * betai);
      P(q, 0) = P(q, 0) * xk;
      P(q, 2) = P(q, 2) * xk;
      lorentz_update(&P(q, 0), exn, eyn, ezn, gam, tau, mass, chrg, lz_ez0v, lz, wx, wy, wz);
      continue;
    }
    P(q, 0) = P(q, 0) * xk;
    P(q, 1) = P(q, 1) + tau * xycon * exn;
    P(q, 2) = P(q, 2) * xk;
    P(q, 3) = P(q, 3) + tau * xycon * eyn;
    P(q, 4) = P(q, 4) * xk / (-(gam * betai));
    P(q, 5) = P(q, 5) - tau * tcon * ezn;
  }
#undef PHI
#undef IDX
  if (!eg) free(egx);
}

/* ------------------------------------------------------------------ */
/* diagnostic1_Output moment sums (Output.f90:133-234) */
void orc_moment_sums(const double *pts, int n, double raw[ORC_RAW_LEN]) {
  double s[37];
  double mx[6], rmax;
  memset(s, 0, sizeof(s));
  if (n != 0) {
    for (int c = 0; c < 6; c++) mx[c] = fabs(P(0, c));
    rmax = P(0, 0) * P(0, 0) + P(0, 2) * P(0, 2);
  } else {
    for (int c = 0; c < 6; c++) mx[c] = 0.0;
    rmax = 0.0;
  }
  for (int i = 0; i < n; i++) {
    double x = P(i, 0), px = P(i, 1), y = P(i, 2), py = P(i, 3), z = P(i, 4), pz = P(i, 5);
    s[0] += x;                           /* x0lc  */
    s[6] += x * x;                       /* sqsum1 */
    s[15] += x * x * x;                  /* x0lc3 */
    s[16] += x * x * x * x;              /* x0lc4 */
    s[12] += x * px;                     /* xpx */
    s[27] += x * px * px;                /* xpx2 */
    s[28] += x * px * px * px;           /* xpx3 */
    s[29] += x * x * px;                 /* x2px */
    s[30] += x * x * px * px;            /* x2px2 */
    s[31] += x * x * x * px;             /* x3px */
    s[1] += px;
    s[7] += px * px;
    s[17] += px * px * px;
    s[18] += px * px * px * px;
    s[2] += y;
    s[8] += y * y;
    s[19] += y * y * y;
    s[20] += y * y * y * y;
    s[13] += y * py;
    s[32] += y * py * py;
    s[33] += y * py * py * py;
    s[34] += y * y * py;
    s[35] += y * y * py * py;
    s[36] += y * y * y * py;
    s[3] += py;
    s[9] += py * py;
    s[21] += py * py * py;
    s[22] += py * py * py * py;
    s[4] += z;
    s[10] += z * z;
    s[23] += fabs(z * z * z);
    s[24] += z * z * z * z;
    s[14] += z * pz;
    s[5] += pz;
    s[11] += pz * pz;
    s[25] += pz * pz * pz;
    s[26] += pz * pz * pz * pz;
    for (int c = 0; c < 6; c++)
      if (mx[c] < fabs(P(i, c))) mx[c] = fabs(P(i, c));
    if (rmax < x * x + y * y) rmax = x * x + y * y;
  }
  memcpy(raw, s, sizeof(s));
  memcpy(raw + 37, mx, sizeof(mx));
  raw[43] = rmax;
}

static double cbrt_f32exp(double v) { return pow(fabs(v), (double)(1.0f / 3.0f)); }

/* diagnostic1_Output rank-0 formulas and write statements (Output.f90:247-352) */
void orc_diag_row(double z, const double raw[ORC_RAW_LEN], int npt, int nlocal,
                  const double refptcl[6], double mass, double row[ORC_DIAG_LEN]) {
  const double *t = raw;
  const double qmc = mass / 1.0e6, xl = PC.Scxl, xt = PC.Rad2deg;
  double den1 = 1.0 / (double)npt;
  double gam = -refptcl[5];
  double gambet = sqrt(gam * gam - 1.0);
  double bet = sqrt(gam * gam - 1.0) / gam;
  double energy = (gam - 1.) * qmc;
  double x0 = t[0] * den1, px0 = t[1] * den1, y0 = t[2] * den1, py0 = t[3] * den1;
  double z0 = t[4] * den1, pz0 = t[5] * den1;
  double sqx = t[6] * den1, sqsum1 = sqx - x0 * x0;
  double sqpx = t[7] * den1, sqsum2 = sqpx - px0 * px0;
  double sqy = t[8] * den1, sqsum3 = sqy - y0 * y0;
  double sqpy = t[9] * den1, sqsum4 = sqpy - py0 * py0;
  double sqz = t[10] * den1, sqsum5 = sqz - z0 * z0;
  double sqpz = t[11] * den1, sqsum6 = sqpz - pz0 * pz0;
  double xpx = t[12] * den1 - x0 * px0;
  double ypy = t[13] * den1 - y0 * py0;
  double zpz = t[14] * den1 - z0 * pz0;
  double cubx = t[15] * den1, fthx = t[16] * den1;
  double x03 = cbrt_f32exp(cubx - 3 * sqx * x0 + 2 * x0 * x0 * x0);
  double x04 = sqrt(sqrt(fabs(fthx - 4 * cubx * x0 + 6 * sqx * x0 * x0 - 3 * x0 * x0 * x0 * x0)));
  double cubpx = t[17] * den1, fthpx = t[18] * den1;
  double px03 = cbrt_f32exp(cubpx - 3 * sqpx * px0 + 2 * px0 * px0 * px0);
  double px04 = sqrt(sqrt(fabs(fthpx - 4 * cubpx * px0 + 6 * sqpx * px0 * px0 -
                               3 * px0 * px0 * px0 * px0)));
  double cuby = t[19] * den1, fthy = t[20] * den1;
  double y03 = cbrt_f32exp(cuby - 3 * sqy * y0 + 2 * y0 * y0 * y0);
  double y04 = sqrt(sqrt(fabs(fthy - 4 * cuby * y0 + 6 * sqy * y0 * y0 - 3 * y0 * y0 * y0 * y0)));
  double cubpy = t[21] * den1, fthpy = t[22] * den1;
  double py03 = cbrt_f32exp(cubpy - 3 * sqpy * py0 + 2 * py0 * py0 * py0);
  double py04 = sqrt(sqrt(fabs(fthpy - 4 * cubpy * py0 + 6 * sqpy * py0 * py0 -
                               3 * py0 * py0 * py0 * py0)));
  double cubz = t[23] * den1, fthz = t[24] * den1;
  double z03 = cbrt_f32exp(cubz - 3 * sqz * z0 + 2 * z0 * z0 * z0);
  double z04 = sqrt(sqrt(fabs(fthz - 4 * cubz * z0 + 6 * sqz * z0 * z0 - 3 * z0 * z0 * z0 * z0)));
  double cubpz = t[25] * den1, fthpz = t[26] * den1;
  double pz03 = cbrt_f32exp(cubpz - 3 * sqpz * pz0 + 2 * pz0 * pz0 * pz0);
  double pz04 = sqrt(sqrt(fabs(fthpz - 4 * cubpz * pz0 + 6 * sqpz * pz0 * pz0 -
                               3 * pz0 * pz0 * pz0 * pz0)));
  double epsx2 = sqsum1 * sqsum2 - xpx * xpx;
  double epsy2 = sqsum3 * sqsum4 - ypy * ypy;
  double epsz2 = sqsum5 * sqsum6 - zpz * zpz;
  double epx = sqrt(fmax(epsx2, 0.0)), epy = sqrt(fmax(epsy2, 0.0)), epz = sqrt(fmax(epsz2, 0.0));
  double xrms = sqrt(sqsum1), pxrms = sqrt(sqsum2), yrms = sqrt(sqsum3);
  double pyrms = sqrt(sqsum4), zrms = sqrt(sqsum5), pzrms = sqrt(sqsum6);
  const double *gm = raw + 37;
  row[0] = z;
  row[1] = refptcl[4]; row[2] = gam; row[3] = energy; row[4] = bet; row[5] = sqrt(raw[43]) * xl;
  row[6] = x0 * xl; row[7] = xrms * xl; row[8] = px0 / gambet; row[9] = pxrms / gambet;
  row[10] = -xpx / epx; row[11] = epx * xl;
  row[12] = y0 * xl; row[13] = yrms * xl; row[14] = py0 / gambet; row[15] = pyrms / gambet;
  row[16] = -ypy / epy; row[17] = epy * xl;
  row[18] = z0 * xt; row[19] = zrms * xt; row[20] = pz0 * qmc; row[21] = pzrms * qmc;
  row[22] = -zpz / epz; row[23] = epz * qmc * xt;
  row[24] = gm[0] * xl; row[25] = gm[1] / gambet; row[26] = gm[2] * xl; row[27] = gm[3] / gambet;
  row[28] = gm[4] * xt; row[29] = gm[5] * qmc;
  row[30] = nlocal; row[31] = nlocal; row[32] = npt;
  row[33] = x03 * xl; row[34] = px03 / gambet; row[35] = y03 * xl; row[36] = py03 / gambet;
  row[37] = z03 * xt; row[38] = pz03 * qmc;
  row[39] = x04 * xl; row[40] = px04 / gambet; row[41] = y04 * xl; row[42] = py04 / gambet;
  row[43] = z04 * xt; row[44] = pz04 * qmc;
}

/* ------------------------------------------------------------------ */
/* Read-in wakefield (type -41 elements, AccSimulator.f90:959-978).  The
 * table is read1wk_Data's (Data.f90:559-633): columns z, longitudinal,
 * x and y wake, z shifted to start at 0; the module arrays hold Ndataini =
 * 5000 rows and are zero beyond the rows read, which the table lookup below
 * reproduces by reading zero past the last row. */
static struct {
  int read, flag;       /* flagwakeread, flagwake of run_AccSimulator */
  int transverse, ntab; /* flagbtw != 2; table rows */
  double scale, hwk;
  double *ew, *epw, *eppw;
  double aa, gg, leng;  /* aawk, ggwk, lengwk of the last 105/106 element */
} WK;

void orc_wake_off(void) {
  WK.read = 0;
  WK.flag = 0;
  WK.scale = 1.0;
}

/* The wake switch at each element (AccSimulator.f90:865-875): a type 105
 * or 106 structure turns the wake on when its Param(15) (period length)
 * is positive, with the analytic wake of Param(13..15) unless a read-in
 * wake is on, and off otherwise; any other element turns off a wake that
 * is not a read-in one. */
void orc_wake_elem(int bitype, const double *val) {
  if (bitype == 105 || bitype == 106) {
    WK.aa = val[11];
    WK.gg = val[12];
    WK.leng = val[13];
    WK.flag = WK.leng > 0.0;
  } else if (!WK.read) {
    WK.flag = 0;
  }
}

int orc_wake_set(const double *z, const double *ew, const double *epw, const double *eppw,
                 int ntab, double scale, int transverse) {
  if (ntab < 2) return -1;
  double *t = (double *)realloc(WK.ew, 3 * (size_t)ntab * sizeof(double));
  if (!t) return -2;
  WK.ew = t;
  WK.epw = t + ntab;
  WK.eppw = t + 2 * (size_t)ntab;
  memcpy(WK.ew, ew, ntab * sizeof(double));
  memcpy(WK.epw, epw, ntab * sizeof(double));
  memcpy(WK.eppw, eppw, ntab * sizeof(double));
  /* zdatwk(i) = zdatwk(i) - zdatwk(1); hwk = zdatwk(2) - zdatwk(1) */
  WK.hwk = (z[1] - z[0]) - (z[0] - z[0]);
  WK.ntab = ntab;
  WK.scale = scale;
  WK.transverse = transverse;
  WK.read = 1;
  WK.flag = 1;
  return 0;
}

static double wk_at(const double *e, int idx1) { /* 1-based, zero past the table */
  return (idx1 >= 1 && idx1 <= WK.ntab) ? e[idx1 - 1] : 0.0;
}

/* greenwake of wakefieldread_FieldQuant (Field.f90:818-830): the table at
 * zz = j*hz with the reference's interpolation weight ab = iwk*hwk - zwk
 * (not divided by hwk) */
static double wk_green(const double *e, int j, double hz) {
  const double zz = j * hz;
  const double zwk = zz - 0.0;
  const int iwk = (int)(zwk / WK.hwk + 1);
  const double ab = iwk * WK.hwk - zwk;
  /* row iwk + 1, written without overflowing iwk + 1 */
  const double e1 = (iwk >= 0 && iwk < WK.ntab) ? e[iwk] : 0.0;
  return wk_at(e, iwk) * ab + e1 * (1.0 - ab);
}

/* line density and transverse moments on the z grid
 * (AccSimulator.f90:1279-1296), particles in the conv1st frame */
void orc_wake_line(const double *pts, int n, int nz, const double range[6], double *densz,
                   double *xsum, double *ysum) {
  const double hzwake = (range[5] - range[4]) / (nz - 1);
  memset(densz, 0, nz * sizeof(double));
  memset(xsum, 0, nz * sizeof(double));
  memset(ysum, 0, nz * sizeof(double));
  for (int q = 0; q < n; q++) {
    const int iizz = (int)((P(q, 4) - range[4]) / hzwake + 1);
    const int iizz1 = iizz + 1;
    const double ab = ((range[4] - P(q, 4)) + iizz * hzwake) / hzwake;
    if (iizz < 1 || iizz1 > nz) continue; /* cannot happen inside update_CompDom's range */
    xsum[iizz - 1] = xsum[iizz - 1] + P(q, 0) * ab;
    xsum[iizz1 - 1] = xsum[iizz1 - 1] + P(q, 0) * (1.0 - ab);
    ysum[iizz - 1] = ysum[iizz - 1] + P(q, 2) * ab;
    ysum[iizz1 - 1] = ysum[iizz1 - 1] + P(q, 2) * (1.0 - ab);
    densz[iizz - 1] = densz[iizz - 1] + ab;
    densz[iizz1 - 1] = densz[iizz1 - 1] + 1.0 - ab;
  }
}

/* The wake fields of one step in grid-field units, added per plane to the
 * node fields by kick1wake (BeamBunch.f90:5015-5033).  The reference
 * convolves on a doubled grid by FFT (wakefieldread_FieldQuant,
 * Field.f90:783-1001); its greenwake has 0.5*W(0) at 0, zeros at 1..Nz-1
 * and W((2Nz-k)hz) above, so for k < Nz the circular convolution is
 *   conv_z(k) = 0.5 W(0) d(k) + sum_{m>k} d(m) W((m-k) hz),
 * evaluated here as that direct sum (the FFT's own rounding aside), and the
 * transverse ones (greenwake zero at 0 too)
 *   conv_x(k) = sum_{m>k} d(m) xbar(m) Wx((m-k) hz).
 * d is recvdensz (AccSimulator.f90:1297-1322).  out = {dEx, dEy, dEz}[nz]. */
static void wake_field(int nz, const double *densz, const double *xsum, const double *ysum,
                       const double range[6], double gam, double curr, int npt, double mass,
                       double chrg, int analytic, double *out, double *raw);

void orc_wake_field(int nz, const double *densz, const double *xsum, const double *ysum,
                    const double range[6], double gam, double curr, int npt, double mass,
                    double chrg, double *out) {
  wake_field(nz, densz, xsum, ysum, range, gam, curr, npt, mass, chrg, 0, out, NULL);
}

/* The analytic wake of wakefield_FieldQuant (Field.f90:590-782), the short-
 * range wakes of a periodic structure of iris radius aa, gap gg and period
 * leng: W_L(z) = Z0 c exp(-sqrt(z/z0)) / (pi aa^2) and
 * W_T(z) = 4 Z0 c z1 / (pi aa^4) (1 - (1 + sqrt(z/z1)) exp(-sqrt(z/z1))),
 * with z0, z1 the fits of Field.f90:627-629 and 694-695 (their literals in
 * default real precision, as the reference writes them).  The same causal
 * sums as the read-in wake, the transverse wakes always on. */
void orc_wake_field_analytic(int nz, const double *densz, const double *xsum,
                             const double *ysum, const double range[6], double gam, double curr,
                             int npt, double mass, double chrg, double aa, double gg,
                             double leng, double *out) {
  const double s_aa = WK.aa, s_gg = WK.gg, s_leng = WK.leng;
  WK.aa = aa;
  WK.gg = gg;
  WK.leng = leng;
  wake_field(nz, densz, xsum, ysum, range, gam, curr, npt, mass, chrg, 1, out, NULL);
  WK.aa = s_aa;
  WK.gg = s_gg;
  WK.leng = s_leng;
}

typedef struct {
  double z0l, z0t, coef1, zc, Z0, pilc, aa;
} analytic_wake;

static analytic_wake analytic_of(double aa, double gg, double leng) {
  analytic_wake w;
  w.pilc = 2 * asin(1.0);
  w.aa = aa;
  w.z0l = (double)0.41f * pow(aa / leng, (double)0.8f) * pow(gg / leng, (double)1.6f) * aa;
  const double Z0 = 120 * w.pilc;
  w.Z0 = Z0;
  w.zc = Z0 * PC.Clight;
  w.z0t = (double)0.169f * aa * pow(aa / leng, (double)1.17f) * pow(gg / aa, (double)0.38f);
  w.coef1 = 4 * Z0 * PC.Clight * w.z0t / (w.pilc * aa * aa * aa * aa);
  return w;
}

static double analytic_wl(const analytic_wake *w, int j, double hz) {
  const double zz = j * hz;
  return w->zc * exp(-sqrt(zz / w->z0l)) / (w->pilc * w->aa * w->aa);
}

static double analytic_wt(const analytic_wake *w, int j, double hz) {
  const double zz = j * hz;
  return w->coef1 * (1.0 - (1. + sqrt(zz / w->z0t)) * exp(-sqrt(zz / w->z0t)));
}

/* out: the per-plane field in grid-field units (kick1wake); raw (or NULL):
 * the wake itself, {Ex, Ey, Ez}[nz], as kick2wake takes it */
static void wake_field(int nz, const double *densz, const double *xsum, const double *ysum,
                       const double range[6], double gam, double curr, int npt, double mass,
                       double chrg, int analytic, double *out, double *raw) {
  const analytic_wake aw = analytic ? analytic_of(WK.aa, WK.gg, WK.leng) : (analytic_wake){0};
  const int tr = analytic || WK.transverse;
  const double scale = analytic ? 1.0 : WK.scale;
  double *d = (double *)malloc(3 * (size_t)nz * sizeof(double));
  double *dx = d + nz, *dy = d + 2 * (size_t)nz;
  double hzwake = (range[5] - range[4]) / (nz - 1);
  hzwake = hzwake / gam;
  for (int k = 0; k < nz; k++) {
    d[k] = densz[k] * curr / PC.Scfreq / npt / hzwake * chrg / fabs(chrg);
    double xw = 0.0, yw = 0.0;
    if (densz[k] != 0.0) {
      xw = xsum[k] / densz[k];
      yw = ysum[k] / densz[k];
    }
    dx[k] = d[k] * xw;
    dy[k] = d[k] * yw;
  }
  /* kick1wake's constants (BeamBunch.f90:4989-5006) */
  const double twopi = 2.0 * PC.Pi;
  const double tmpscale = curr / PC.Scfreq;
  const double fpei = PC.Clight * PC.Clight * (double)1.0e-7f;
  const double xk = 1 / PC.Scxl;
  const double bet = sqrt(gam * gam - 1.0) / gam;
  const double bbyk = bet / xk;
  const double gambet = gam * bet;
  const double brho = gambet / (PC.Clight * chrg) * mass;
  const double vz0 = bet * PC.Clight;
  const double perv0 = 2.0 * curr * fpei / (brho * vz0 * vz0 * gam * gam);
  const double xycon = 0.5 * perv0 * gambet * bbyk * twopi / tmpscale;
  const double tcon = bet * xycon * (gam * gam);
  /* greenwake(1): 0.5 W(0), written as the reference writes each form */
  const double g0 = analytic ? 0.5 * aw.Z0 * PC.Clight * exp(-sqrt(0.0 / aw.z0l)) /
                                   (aw.pilc * aw.aa * aw.aa)
                             : 0.5 * wk_green(WK.ew, 0, hzwake);
  for (int k = 0; k < nz; k++) {
    double cz = d[k] * g0, cx = 0.0, cy = 0.0;
    for (int m = k + 1; m < nz; m++) {
      if (analytic) {
        cz = cz + d[m] * analytic_wl(&aw, m - k, hzwake);
        const double wt = analytic_wt(&aw, m - k, hzwake);
        cx = cx + dx[m] * wt;
        cy = cy + dy[m] * wt;
      } else {
        cz = cz + d[m] * wk_green(WK.ew, m - k, hzwake);
        if (tr) {
          cx = cx + dx[m] * wk_green(WK.epw, m - k, hzwake);
          cy = cy + dy[m] * wk_green(WK.eppw, m - k, hzwake);
        }
      }
    }
    const double ezwake = scale * (-cz * hzwake);
    const double exwake = scale * (cx * hzwake);
    const double eywake = scale * (cy * hzwake);
    out[k] = chrg * exwake / xycon / mass / bet / gam;
    out[nz + k] = chrg * eywake / xycon / mass / bet / gam;
    out[2 * nz + k] = chrg * ezwake / tcon / mass;
    if (raw) {
      raw[k] = exwake;
      raw[nz + k] = eywake;
      raw[2 * nz + k] = ezwake;
    }
  }
  free(d);
}

/* ------------------------------------------------------------------ */
/* 1D CSR wake with integrated Green functions, steady state and transients
 * (csrwakeTrIGF_FieldQuant, Field.f90:1003-1251, with IcsrCaseA..D at
 * Field.f90:1253-1303).  Case D's retarded angle is the root of the quartic
 * of funcd (Field.f90:1370-1388), found by Newton-Raphson with bisection
 * safeguard in a bracket, the published "rtsafe" method (Numerical Recipes
 * 9.4) as the reference's `root` (Field.f90:1305-1368) applies it: a
 * bracket end within xacc of a root is returned as is; no bracket or no
 * convergence in maxit steps returns the last iterate. */
static double csr_caseA(double phih, double ssh, double xk2) {
  const double p2 = phih * phih, p3 = p2 * phih, p4 = p3 * phih;
  const double bb = 2 * phih + p3 / 3 - 2 * ssh;
  const double cc = p2 + p4 / 12 - 2 * ssh * phih;
  const double yh = (-bb + sqrt(bb * bb - 4 * cc)) / 2;
  const double phpy = phih + yh;
  return xk2 * (-(2 * phpy + p3) / (phpy * phpy + p4 / 4) + 1.0 / ssh);
}

static double csr_caseB(double ssh, double xk2) {
  const double aa = sqrt(64.0 + 144.0 * (ssh * ssh));
  const double uuh = pow(aa + 12 * ssh, 1.0 / 3.0) - pow(aa - 12 * ssh, 1.0 / 3.0);
  const double u2 = uuh * uuh;
  return xk2 * (-4 * uuh * (u2 + 8) / ((u2 + 4.0) * (u2 + 12.0)));
}

static double csr_caseC(double phimh, double xxbarh, double ssh, double xk2) {
  const double p2 = phimh * phimh, p3 = p2 * phimh;
  const double bb = 2 * (phimh + xxbarh) - 2 * ssh + p3 / 3 + p2 * xxbarh;
  const double cc = (phimh + xxbarh) * (phimh + xxbarh) +
                    p2 * (p2 + 4 * phimh * xxbarh) / 12 - 2 * ssh * (phimh + xxbarh);
  const double yh = (-bb + sqrt(bb * bb - 4 * cc)) / 2;
  const double pa = phimh + xxbarh + yh;
  const double pb = phimh * xxbarh + phimh * phimh / 2.0;
  return xk2 * (-2.0 * (pa + phimh * pb) / (pa * pa + pb * pb) + 1.0 / ssh);
}

static void csr_quartic(double psi, double xxh, double ds, double *f, double *df) {
  const double p2 = psi * psi, p3 = p2 * psi, p4 = p3 * psi;
  *f = p4 / 12 + xxh * p3 / 3 + p2 + (2 * xxh - 2 * ds) * psi - 2 * ds * xxh + xxh * xxh;
  *df = p3 / 3 + xxh * p2 + 2 * psi + 2 * xxh - 2 * ds;
}

static double csr_root(double x1, double x2, double xacc, int maxit, double ds, double xxh) {
  double fl, fh, f, df, xl, xh;
  csr_quartic(x1, xxh, ds, &fl, &df);
  csr_quartic(x2, xxh, ds, &fh, &df);
  if (fabs(fl) < xacc) return x1;
  if (fabs(fh) < xacc) return x2;
  if (fl < 0.0) { xl = x1; xh = x2; } else { xh = x1; xl = x2; }
  double rts = 0.5 * (x1 + x2);
  double dxold = fabs(x2 - x1), dx = dxold;
  csr_quartic(rts, xxh, ds, &f, &df);
  for (int j = 1; j <= maxit; j++) {
    if (((rts - xh) * df - f) * ((rts - xl) * df - f) > 0.0 || fabs(2.0 * f) > fabs(dxold * df)) {
      dxold = dx;
      dx = 0.5 * (xh - xl);
      rts = xl + dx;
      if (xl == rts) return rts;
    } else {
      dxold = dx;
      dx = f / df;
      const double temp = rts;
      rts = rts - dx;
      if (temp == rts) return rts;
    }
    if (fabs(dx) < xacc) return rts;
    csr_quartic(rts, xxh, ds, &f, &df);
    if (f < 0.0) xl = rts; else xh = rts;
  }
  return rts;
}

static double csr_caseD(double xxbarh, double psimax, double ssh, double xk2, double epstol,
                        int nmax) {
  const double psi = csr_root(-epstol, psimax * (1.0 + epstol), epstol, nmax, ssh, xxbarh);
  const double pa = psi + xxbarh;
  const double pb = psi * (xxbarh + psi / 2.0);
  return xk2 * (-2.0 * (pa + psi * pb) / (pa * pa + pb * pb) + 1.0 / ssh);
}

void orc_csr_wake(int nx, double r0, double ptmin, double hx, double blength,
                  const double *rho, double gam, double *ez) {
  const double epstol = 2.0e-9;
  const int nmax = 100;
  const double pilc = 2 * asin(1.0);
  const double phim = blength / r0;
  const double xconst = 1.0 / (4 * pilc * 8.854187817e-12);
  const double xk2 = gam / r0;
  const double g3 = gam * gam * gam;
#define RHO(j) rho[(j)-1]
#define SSH(xxp) ((xx - (xxp)) * g3 / r0)
  ez[0] = 0.0;
  for (int i = 2; i <= nx; i++) {
    const double xx = ptmin + (i - 1) * hx;
    const double t = xx / r0;
    const double xxl = t * t * t * r0 / 24;
    const int ni = i;
    double e = 0.0;
    if (xx <= 0) {
    } else if (xx <= blength) {
      const double xslp = (xx / r0) * r0 / 2 / gam / gam + xxl;
      const int islp0 = (int)((xx - xslp - ptmin) / hx);
      const int islp1 = islp0 + 1;
      const double phih = xx / r0 * gam;
      /* Case A (entrance transient) */
      for (int j = 2; j <= islp1 - 1; j++) {
        const double c2 = csr_caseA(phih, SSH(ptmin + (j - 1) * hx + hx / 2), xk2);
        const double c1 = csr_caseA(phih, SSH(ptmin + (j - 1) * hx - hx / 2), xk2);
        e = e + RHO(j) * (c1 - c2);
      }
      if (islp1 >= 2) {
        double c2 = csr_caseA(phih, SSH(xx - xslp), xk2);
        double c1 = csr_caseA(phih, SSH(ptmin + (islp1 - 1) * hx - hx / 2), xk2);
        e = e + RHO(islp1) * (c1 - c2);
        c2 = csr_caseA(phih, SSH(ptmin + hx / 2), xk2);
        c1 = csr_caseA(phih, SSH(ptmin), xk2);
        e = e + RHO(1) * (c1 - c2);
      } else if (islp1 == 1) {
        const double c2 = csr_caseA(phih, SSH(xx - xslp), xk2);
        const double c1 = csr_caseA(phih, SSH(ptmin + (islp1 - 1) * hx), xk2);
        e = e + RHO(islp1) * (c1 - c2);
      }
      /* Case B (steady state) */
      const int jstart = islp1 > 1 ? islp1 : 1;
      for (int j = jstart + 2; j <= ni - 1; j++) {
        const double c2 = csr_caseB(SSH(ptmin + (j - 1) * hx + hx / 2), xk2);
        const double c1 = csr_caseB(SSH(ptmin + (j - 1) * hx - hx / 2), xk2);
        e = e + RHO(j) * (c1 - c2);
      }
      if (jstart <= ni - 2) {
        double c2 = csr_caseB(SSH(ptmin + (ni - 1) * hx), xk2);
        double c1 = csr_caseB(SSH(ptmin + (ni - 1) * hx - hx / 2), xk2);
        e = e + RHO(ni) * (c1 - c2);
        if (islp1 < 1) {
          const int j = 1;
          c2 = csr_caseB(SSH(ptmin + (j - 1) * hx + hx / 2), xk2);
          c1 = csr_caseB(SSH(ptmin + (j - 1) * hx), xk2);
          e = e + RHO(j) * (c1 - c2);
        } else {
          const int j = islp1 + 1;
          c2 = csr_caseB(SSH(ptmin + (j - 1) * hx + hx / 2), xk2);
          c1 = csr_caseB(SSH(xx - xslp), xk2);
          e = e + RHO(j) * (c1 - c2);
        }
      } else if (jstart == ni - 1) {
        const int j = ni;
        const double c2 = csr_caseB(SSH(ptmin + (j - 1) * hx), xk2);
        const double c1 = csr_caseB(SSH(xx - xslp), xk2);
        e = e + RHO(j) * (c1 - c2);
      }
    } else {
      const double xxbar = xx - blength;
      const double rp = r0 * phim;
      const double xslp = (rp + xxbar) / 2 / gam / gam +
                          r0 * (phim * phim * phim) / 24 * (rp + 4 * xxbar) / (rp + xxbar);
      const int islp0 = (int)((xx - xslp - ptmin) / hx);
      const int islp1 = islp0 + 1;
      const double xslpN = xxbar / 2.0 / gam / gam;
      const int islpN = (int)((xx - xslpN - ptmin) / hx);
      const int islpN1 = islpN + 1;
      /* Case C (exit transient, source in the bend) */
      const double xxbarh = xxbar * gam / r0;
      const double phimh = phim * gam;
      for (int j = 2; j <= islp1 - 1; j++) {
        const double c2 = csr_caseC(phimh, xxbarh, SSH(ptmin + (j - 1) * hx + hx / 2), xk2);
        const double c1 = csr_caseC(phimh, xxbarh, SSH(ptmin + (j - 1) * hx - hx / 2), xk2);
        e = e + RHO(j) * (c1 - c2);
      }
      if (islp1 >= 2) {
        double c2 = csr_caseC(phimh, xxbarh, SSH(xx - xslp), xk2);
        double c1 = csr_caseC(phimh, xxbarh, SSH(ptmin + (islp1 - 1) * hx - hx / 2), xk2);
        e = e + RHO(islp1) * (c1 - c2);
        c2 = csr_caseC(phimh, xxbarh, SSH(ptmin + hx / 2), xk2);
        c1 = csr_caseC(phimh, xxbarh, SSH(ptmin), xk2);
        e = e + RHO(1) * (c1 - c2);
      } else if (islp1 == 1) {
        const double c2 = csr_caseC(phimh, xxbarh, SSH(xx - xslp), xk2);
        const double c1 = csr_caseC(phimh, xxbarh, SSH(ptmin), xk2);
        e = e + RHO(islp1) * (c1 - c2);
      }
      /* Case D (exit transient, source before the exit) */
      const double psimax = phim * gam;
      const int jstart = islp1 > 0 ? islp1 : 0;
      for (int j = jstart + 2; j <= islpN1 - 1; j++) {
        const double c2 = csr_caseD(xxbarh, psimax, SSH(ptmin + (j - 1) * hx + hx / 2), xk2,
                                    epstol, nmax);
        const double c1 = csr_caseD(xxbarh, psimax, SSH(ptmin + (j - 1) * hx - hx / 2), xk2,
                                    epstol, nmax);
        e = e + RHO(j) * (c1 - c2);
      }
      if (islpN1 >= jstart + 2) {
        double c2 = csr_caseD(xxbarh, psimax, xslpN * g3 / r0, xk2, epstol, nmax);
        double c1 = csr_caseD(xxbarh, psimax, SSH(ptmin + (islpN1 - 1) * hx - hx / 2), xk2,
                              epstol, nmax);
        e = e + RHO(islpN1) * (c1 - c2);
        c2 = csr_caseD(xxbarh, psimax, SSH(ptmin + jstart * hx + hx / 2), xk2, epstol, nmax);
        c1 = csr_caseD(xxbarh, psimax, xslp * g3 / r0, xk2, epstol, nmax);
        e = e + RHO(jstart + 1) * (c1 - c2);
      } else if (islpN1 == jstart + 1) {
        const double c2 = csr_caseD(xxbarh, psimax, xslpN * g3 / r0, xk2, epstol, nmax);
        const double c1 = csr_caseD(xxbarh, psimax, xslp * g3 / r0, xk2, epstol, nmax);
        e = e + RHO(jstart + 1) * (c1 - c2);
      }
    }
    ez[i - 1] = e * xconst;
  }
#undef SSH
#undef RHO
}

/* The CSR glue of one step (AccSimulator.f90:1344-1390) and kick1wake's
 * addition (BeamBunch.f90:5015-5033): densz from orc_wake_line, s0 the
 * distance of the step from the bend entrance, blen the bend length; out =
 * {0, 0, dEz}[nz]. */
static void csr_field(int nz, const double *densz, const double range[6], double gam,
                      double curr, int npt, double mass, double chrg, double r0, double s0,
                      double blen, double *out, double *raw);

void orc_csr_field(int nz, const double *densz, const double range[6], double gam,
                   double curr, int npt, double mass, double chrg, double r0, double s0,
                   double blen, double *out) {
  csr_field(nz, densz, range, gam, curr, npt, mass, chrg, r0, s0, blen, out, NULL);
}

/* raw (or NULL): the wake itself, {0, 0, Ez}[nz], as kick2wake takes it */
static void csr_field(int nz, const double *densz, const double range[6], double gam,
                      double curr, int npt, double mass, double chrg, double r0, double s0,
                      double blen, double *out, double *raw) {
  double *d = (double *)malloc(2 * (size_t)nz * sizeof(double));
  double *ez = d + nz;
  double hzwake = (range[5] - range[4]) / (nz - 1);
  hzwake = hzwake / gam;
  for (int k = 0; k < nz; k++)
    d[k] = densz[k] * curr / PC.Scfreq / npt / hzwake * chrg / fabs(chrg);
  const double zwkmin = range[4] / gam + s0;
  orc_csr_wake(nz, r0, zwkmin, hzwake, blen, d, gam, ez);
  /* kick1wake's constants (BeamBunch.f90:4989-5006) */
  const double twopi = 2.0 * PC.Pi;
  const double tmpscale = curr / PC.Scfreq;
  const double fpei = PC.Clight * PC.Clight * (double)1.0e-7f;
  const double xk = 1 / PC.Scxl;
  const double bet = sqrt(gam * gam - 1.0) / gam;
  const double bbyk = bet / xk;
  const double gambet = gam * bet;
  const double brho = gambet / (PC.Clight * chrg) * mass;
  const double vz0 = bet * PC.Clight;
  const double perv0 = 2.0 * curr * fpei / (brho * vz0 * vz0 * gam * gam);
  const double xycon = 0.5 * perv0 * gambet * bbyk * twopi / tmpscale;
  const double tcon = bet * xycon * (gam * gam);
  for (int k = 0; k < nz; k++) {
    out[k] = 0.0;
    out[nz + k] = 0.0;
    out[2 * nz + k] = chrg * ez[k] / tcon / mass;
    if (raw) {
      raw[k] = 0.0;
      raw[nz + k] = 0.0;
      raw[2 * nz + k] = ez[k];
    }
  }
  free(d);
}

/* ------------------------------------------------------------------ */
/* Laser heater of a type -52 element (AccSimulator.f90:982-1006), one rank */
void orc_laser_heater(double *pts, int n, int npt, double rsig, double wavelength, double ez,
                      double mass) {
  double xygl[2] = {0.0, 0.0};
  for (int i = 0; i < n; i++) {
    xygl[0] = xygl[0] + P(i, 0);
    xygl[1] = xygl[1] + P(i, 0) * P(i, 0);
  }
  xygl[0] = xygl[0] / npt;
  xygl[1] = xygl[1] / npt;
  const double sigx2 = (xygl[1] - xygl[0] * xygl[0]) * PC.Scxl * PC.Scxl;
  const double tmp1 = sqrt(2 * (sigx2 + rsig * rsig) / (rsig * rsig));
  const double freqlaser = PC.Clight / wavelength;
  const double harm = freqlaser / PC.Scfreq;
  const double tmp2 = 4 * rsig * rsig / PC.Scxl / PC.Scxl;
  const double ezlaser = ez / mass;
  for (int i = 0; i < n; i++) {
    const double rr = (P(i, 0) * P(i, 0) + P(i, 2) * P(i, 2)) / tmp2;
    P(i, 5) = P(i, 5) - tmp1 * ezlaser * sin(-harm * P(i, 4)) * exp(-rr);
  }
}

/* ------------------------------------------------------------------ */
/* element 110 as the Lorentz integrator carries it: discrete data
 * (Param(13) = 1) on the x-y-z grid (Param(14) = 2) of read4_Data.  Its
 * other forms read data the driver never loads for it under Flagmap=2
 * (the r-z tables of read2_Data and the Fourier coefficients of
 * read3_Data, AccSimulator.f90:836-846). */
static int emfld_ok(const orc_elem *e) {
  if (e->type != 110 || !e->zdat || !e->edat) return 0;
  if ((int)(0.1 + e->val[11]) != 1 || (int)(0.1 + e->val[12]) != 2) return 0;
  const int nx = (int)(e->zdat[2] + 0.1), ny = (int)(e->zdat[5] + 0.1), nz = (int)(e->zdat[8] + 0.1);
  return nx >= 2 && ny >= 2 && nz >= 2 && e->ndata == (nx + 1) * (ny + 1) * (nz + 1);
}

static double pipe_radius(const orc_elem *e) {
  /* getradius_BeamLineElem (BeamLineElem.f90:500-552): Param index per type */
  switch (e->type) {
    case 0: return e->val[0];  /* DriftTube Param(2) */
    case 1: return e->val[2];  /* Quadrupole Param(4) */
    case 2: return e->val[3];  /* ConstFoc Param(5) */
    case 3: return e->val[2];  /* Sol Param(4) */
    case 4: return e->val[3];  /* Dipole Param(5) */
    case 5: return e->val[3];  /* Multipole Param(5) */
    default: return e->val[4]; /* RF gaps Param(6) */
  }
}

/* run_AccSimulator element/segment loop (AccSimulator.f90:742-1504) for
 * Flagmap=1, Flagbc=1, Flagerr=0, Flagsubstep=0, one rank; the read-in wake
 * of orc_wake_set applies to every space-charge kick while it is on, the
 * CSR wake inside bends with dparam(4) > 200 and after bends with
 * dparam(4) > 500 (bend state carried in the beam between calls). */
int orc_run(const orc_elem *elems, int nelem, orc_beam *beam, const int mesh[3],
            double *rows, int maxrows) {
  const double Scxl = PC.Scxl;
  const double bcurr = beam->current;
  const size_t G = (size_t)mesh[0] * mesh[1] * mesh[2];
  double *rho = (double *)malloc(G * sizeof(double));
  double raw[ORC_RAW_LEN];
  int nrows = 0;
  double z = beam->z;
  if (!rho) return -2;
#define DIAG()                                                                    \
  do {                                                                            \
    if (nrows < maxrows) {                                                        \
      orc_moment_sums(beam->pts, beam->nlocal, raw);                              \
      orc_diag_row(z, raw, beam->npt, beam->nlocal, beam->refptcl, beam->mass,    \
                   rows + (size_t)ORC_DIAG_LEN * nrows);                          \
    }                                                                             \
    if (nrows < g_chg.maxrows)                                                    \
      memcpy(g_chg.out + (size_t)g_chg.nchrg * nrows, g_chg.cur,                  \
             (size_t)g_chg.nchrg * sizeof(int));                                  \
    nrows++;                                                                      \
  } while (0)
  DIAG();
  for (int ie = 0; ie < nelem; ie++) {
    const orc_elem *e = &elems[ie];
    const double blength = e->length;
    const int bnseg = e->nseg, bitype = e->type;
    double piperad = pipe_radius(e), piperad2 = piperad;
    if (bitype == 110) piperad2 = e->val[5]; /* EMfld: Param(7) (BeamLineElem.f90:538-540) */
    if (bitype < 0) { free(rho); return -3; }
    const int lorentz = beam->flagmap == 2;
    /* Lorentz integrator: drifts, quadrupoles (not 0 < Param(3) <= 1e-5,
     * where getfld_Quadrupole reads G', G'' it never set), constant
     * focusing, solenoids and the RF cavities 101..106 over Fourier
     * coefficients */
    if (lorentz && !(bitype == 0 || bitype == 2 || bitype == 3 || emfld_ok(e) ||
                     (bitype == 1 && (e->val[1] <= 0.0 || e->val[1] > 1.0e-5)) ||
                     (bitype >= 101 && bitype <= 104 && e->zdat && e->ndata >= 1) ||
                     ((bitype == 105 || bitype == 106) && e->zdat && e->ndata >= 5) ||
                     (bitype == 5 && (int)(e->val[0] + 0.1) >= 2 &&
                      (int)(e->val[0] + 0.1) <= 4 &&
                      (e->val[2] <= 0.0 || (e->zdat && e->edat && e->ndata >= 2))))) {
      free(rho);
      return -10;
    }
    const double lz_zedge = z;
    orc_wake_elem(bitype, e->val);
    if (bitype == 4) { piperad = 100.0; piperad2 = 100.0; }
    double tau1 = 0.0;
    if (bitype >= 0) tau1 = 0.5 * blength / bnseg;
    double tau2 = 2.0 * tau1;
    double zedge = z;
    /* bend entry (AccSimulator.f90:1032-1094) */
    double gamma0 = 0, beta0 = 0, hd0 = 0, hd1 = 0, hB = 0, tanphiB = 0, tanphiBb = 0;
    double psi2 = 0, angB = 0, qm0 = beam->charge / beam->mass;
    if (bitype == 4) {
      const double *dp = e->val - 2; /* dparam(k) = val[k-2] */
      gamma0 = -beam->refptcl[5];
      beta0 = sqrt(1.0 - 1.0 / gamma0 / gamma0);
      beam->refptcl[4] = beam->refptcl[4] + blength / (Scxl * beta0);
      double hgap = 2 * dp[5];
      piperad2 = dp[5];
      double ang0 = dp[2];
      hd1 = dp[3];
      double angF = dp[6];
      angB = dp[7];
      double hF = dp[8];
      hB = dp[9];
      double dstr1 = dp[10], dstr2 = dstr1;
      hd0 = ang0 / blength;
      /* CSR bookkeeping of the bend entry (AccSimulator.f90:1032-1051, 1088) */
      beam->r0 = fabs(1.0 / hd0);
      if (bcurr > 0.0 && dp[4] > 500) {
        beam->flagbendcsr = 1;
        beam->bendlencsr = blength;
        beam->sentr = 0.0;
      } else {
        beam->flagbendcsr = 0;
      }
      double tanphiF = tan(angF);
      double psi1 = hd0 * hgap * dstr1 * (1.0 + sin(angF) * sin(angF)) / cos(angF);
      double tanphiFb = tan(angF - psi1);
      tanphiB = tan(angB);
      psi2 = hd0 * hgap * dstr2 * (1.0 + sin(angB) * sin(angB)) / cos(angB);
      tanphiBb = tan(angB - psi2);
      orc_fpol(hd0, hF, tanphiF, tanphiFb, hd1, psi1, beam->pts, angF, beam->nlocal,
               gamma0, qm0);
    }
    int ihlf = 0;
    for (int j = 1; j <= bnseg; j++) {
      /* first half map */
      for (int half = 0; half < 2; half++) {
        if (half == 1) {
          /* space charge between the two half maps */
          if (!(bcurr < 1.0e-10)) {
            double ptrange[6], range[6], msize[3];
            beam->nlocal = orc_conv1st(beam->pts, beam->nlocal, &beam->current, &beam->npt,
                                       beam->refptcl, piperad, piperad2, ptrange);
            orc_chgupdate(beam->pts, beam->nlocal); /* AccSimulator.f90:1130 */
            orc_update_compdom(ptrange, mesh, range, msize);
            orc_deposit(beam->pts, beam->nlocal, mesh, range, msize, rho, NULL, NULL);
            if (orc_poisson_open(mesh[0], mesh[1], mesh[2], msize[0], msize[1], msize[2], rho)) {
              free(rho);
              return -5;
            }
            double *wf = NULL;
            /* CSR inside a bend with dparam(4) > 200, and downstream of a
             * bend with dparam(4) > 500 (AccSimulator.f90:1131-1138) */
            int flagcsr = 0;
            if (bitype == 4) {
              if (e->val[2] > 200) flagcsr = 1;
            } else if (beam->flagbendcsr) {
              flagcsr = 1;
            }
            if (flagcsr) { /* AccSimulator.f90:1344-1390: replaces any read-in wake */
              const int nz = mesh[2];
              wf = (double *)calloc(9 * (size_t)nz, sizeof(double));
              double *line = wf + 3 * (size_t)nz;
              orc_wake_line(beam->pts, beam->nlocal, nz, range, line, line + nz,
                            line + 2 * (size_t)nz);
              const double s0 = bitype == 4 ? z - beam->zbleng : z - beam->zbleng + beam->sentr;
              csr_field(nz, line, range, -beam->refptcl[5], beam->current, beam->npt,
                        beam->mass, beam->charge, beam->r0, s0,
                        bitype == 4 ? blength : beam->bendlencsr, wf, wf + 6 * (size_t)nz);
            } else if (WK.flag) { /* AccSimulator.f90:1273-1340 */
              const int nz = mesh[2];
              wf = (double *)malloc(9 * (size_t)nz * sizeof(double));
              double *line = wf + 3 * (size_t)nz;
              orc_wake_line(beam->pts, beam->nlocal, nz, range, line, line + nz,
                            line + 2 * (size_t)nz);
              wake_field(nz, line, line + nz, line + 2 * (size_t)nz, range, -beam->refptcl[5],
                         beam->current, beam->npt, beam->mass, beam->charge, !WK.read, wf,
                         wf + 6 * (size_t)nz);
            }
            orc_cvbkforth1st(beam->pts, beam->nlocal, beam->refptcl);
            if (lorentz)
              beam->refptcl[5] = -orc_kick2(beam->pts, beam->nlocal, rho, mesh, range, msize,
                                            -beam->refptcl[5], beam->current, tau2, beam->mass,
                                            beam->charge, e, lz_zedge, z, beam->refptcl[4],
                                            beam->nlocal ? beam->pts[6] : 0.0,
                                            wf ? wf + 6 * (size_t)mesh[2] : NULL);
            else {
              double *egp = NULL;
              if (g_probe.step < g_probe.maxsteps) {
                if (g_probe.phi)
                  memcpy(g_probe.phi + G * (size_t)g_probe.step, rho, G * sizeof(double));
                if (g_probe.eg) egp = g_probe.eg + 3 * G * (size_t)g_probe.step;
                g_probe.step++;
              }
              orc_kick1w(beam->pts, beam->nlocal, rho, mesh, range, msize, -beam->refptcl[5],
                         beam->current, tau2, beam->mass, beam->charge, egp, wf);
            }
            free(wf);
          }
        }
        if (lorentz && half == 1 && bcurr < 1.0e-10)
          /* kick2 without current: scatter20 (BeamBunch.f90:3075-3531) */
          beam->refptcl[5] = -orc_lorentz_nosc(beam->pts, beam->nlocal, -beam->refptcl[5], tau2,
                                               beam->mass, beam->charge, e, lz_zedge, z,
                                               beam->refptcl[4],
                                               beam->nlocal ? beam->pts[6] : 0.0);
        if (lorentz) {
          /* map1_BeamBunch(Bpts,z,tau2): drift2 by tau2/2 (AccSimulator.f90:1109-1116) */
          orc_drift2(beam->pts, beam->nlocal, beam->refptcl, tau2);
          z = z + 0.5 * tau2;
        } else if (bitype == 4) {
          orc_sector(tau1, beta0, hd0, hd1, beam->pts, beam->nlocal, qm0);
          z = z + tau1;
        } else if (bitype == 0) {
          orc_drift_exact(beam->pts, beam->nlocal, beam->refptcl, tau1);
          z = z + tau1;
          ihlf++;
        } else if (bitype == 1) {
          double x3 = e->val[1];
          if (x3 < -10.0) {
            orc_undulator(tau1, e->val[0], beam->refptcl, beam->pts, beam->nlocal);
          } else if (x3 < -1.0e-6) {
            orc_transfmapK(tau1, e->val[0], beam->refptcl, beam->pts, beam->nlocal, qm0);
          } else if (x3 > 1.0e-5) {
            /* the gradient profile of read1_Data (AccSimulator.f90:853-863) */
            if (e->ndata < 2) { free(rho); return -7; }
            double xm[36];
            orc_maplinear_quad_fringe(z, tau1, xm, beam->refptcl, zedge, e->mapstp,
                                      beam->charge, beam->mass, e->ndata, e->zdat, e->edat);
            orc_apply_xm(beam->pts, beam->nlocal, xm);
          } else {
            double xm[36];
            orc_maplinear_quad(z, tau1, xm, beam->refptcl, e->val[0], e->mapstp,
                               beam->charge, beam->mass);
            orc_apply_xm(beam->pts, beam->nlocal, xm);
          }
          z = z + tau1;
          ihlf++;
        } else if (bitype == 2) {
          if (e->val[3] < 0.0) { free(rho); return -8; } /* ideal-gap test: left out */
          double xm[36];
          orc_maplinear_constfoc(z, tau1, xm, beam->refptcl, e->val, e->mapstp);
          orc_apply_xm(beam->pts, beam->nlocal, xm);
          z = z + tau1;
          ihlf++;
        } else if (bitype == 3) {
          if (e->val[3] < 0.0) { free(rho); return -8; } /* ideal-gap test: left out */
          double xm[36];
          orc_maplinear_sol(z, tau1, xm, beam->refptcl, e->val[0], e->mapstp, beam->charge,
                            beam->mass);
          orc_apply_xm(beam->pts, beam->nlocal, xm);
          z = z + tau1;
          ihlf++;
        } else if (bitype >= 101 && bitype <= 106) {
          if (e->val[3] < 0.0) {
            orc_ideal_rf(beam->pts, beam->nlocal, beam->refptcl, beam->mass, tau1,
                         e->val[0], e->val[1], e->val[2], j, bnseg, ihlf);
          } else if (bitype == 105 && e->ndata >= 5) {
            double xm[36];
            orc_maplinear_solrf(z, tau1, xm, beam->refptcl, zedge, e->val[0], e->val[1],
                                e->val[2], e->mapstp, beam->charge, beam->mass, blength,
                                e->val[10], e->ndata, e->zdat);
            orc_apply_xm(beam->pts, beam->nlocal, xm);
          } else if (bitype == 106 && e->ndata >= 9) {
            double xm[36];
            orc_maplinear_tws(z, tau1, xm, beam->refptcl, zedge, e->val[0], e->val[1], e->val[2],
                              e->mapstp, beam->charge, beam->mass, blength, e->val[10],
                              e->ndata, e->zdat);
            orc_apply_xm(beam->pts, beam->nlocal, xm);
          } else if (bitype <= 104 && e->ndata > 1) {
            /* DTL, CCDTL, CCL, SC linear maps (maplinear_BeamLineElem,
             * BeamLineElem.f90:776-800) */
            double xm[36];
            const double dtlq[5] = {blength, e->val[5], e->val[6], e->val[7], e->val[8]};
            maplinear_rf(z, tau1, xm, beam->refptcl, zedge, e->val[0], e->val[1], e->val[2],
                         e->mapstp, beam->charge, beam->mass, e->ndata, e->zdat, e->edat,
                         e->epdat, e->eppdat, bitype == 101 ? dtlq : NULL);
            orc_apply_xm(beam->pts, beam->nlocal, xm);
          } else {
            free(rho);
            return -8;
          }
          z = z + tau1;
          ihlf++;
        } else {
          free(rho);
          return -9;
        }
      }
      DIAG();
    }
    if (bitype == 4)
      orc_bpol(hd0, hB, tanphiB, tanphiBb, hd1, psi2, beam->pts, angB, beam->nlocal, gamma0,
               qm0);
    beam->zbleng = beam->zbleng + blength; /* AccSimulator.f90:1498-1499 */
    beam->sentr = beam->sentr + blength;
  }
#undef DIAG
  beam->z = z;
  free(rho);
  return nrows;
}
