// impz_host.cpp -- host-side builders for the B200 step pipeline.
//
// Everything here runs once per element or step on the host: the linear
// maps integrated by RK6, the per-element constants the device map ops use,
// the compilation of a lattice into a step table, and the diagnostic
// formulas.  Built with -ffp-contract=off so the arithmetic rounds like the
// reference's x86-64 build; expressions keep the reference's left-to-right
// evaluation order (cited per routine).
#include "impz_host.h"

#include <cmath>
#include <cstring>

namespace impz {

Phys make_phys(double freq) {
  // PhysConst.f90:29-34
  Phys P;
  P.Clight = 299792458.0;
  P.Pi = 2 * std::asin(1.0);
  P.Scxl = P.Clight / (2 * P.Pi * freq);
  P.Rad2deg = 180.0 / P.Pi;
  P.Scfreq = freq;
  return P;
}

// ---------------------------------------------------------------------
// 8-stage RK6 of the reference's rk6i_* routines (Quadrupole.f90:202-252)
namespace {
const int NV = 18;

template <int NV = 18, typename RHS>
void rk6(double h, int ns, double t, double* y, RHS rhs) {
  double yt[NV], a[NV], b[NV], c[NV], d[NV], e[NV], f[NV], g[NV], o[NV], p[NV];
  const double tint = t;
  double tt;
  for (int i = 1; i <= ns; i++) {
    rhs(t, y, f);
    for (int v = 0; v < NV; v++) a[v] = h * f[v];
    for (int v = 0; v < NV; v++) yt[v] = y[v] + a[v] / 9.0;
    tt = t + h / 9.0;
    rhs(tt, yt, f);
    for (int v = 0; v < NV; v++) b[v] = h * f[v];
    for (int v = 0; v < NV; v++) yt[v] = y[v] + (a[v] + 3.0 * b[v]) / 24.0;
    tt = t + h / 6.0;
    rhs(tt, yt, f);
    for (int v = 0; v < NV; v++) c[v] = h * f[v];
    for (int v = 0; v < NV; v++) yt[v] = y[v] + (a[v] - 3.0 * b[v] + 4.0 * c[v]) / 6.0;
    tt = t + h / 3.0;
    rhs(tt, yt, f);
    for (int v = 0; v < NV; v++) d[v] = h * f[v];
    for (int v = 0; v < NV; v++)
      yt[v] = y[v] + (278.0 * a[v] - 945.0 * b[v] + 840.0 * c[v] + 99.0 * d[v]) / 544.0;
    tt = t + .5 * h;
    rhs(tt, yt, f);
    for (int v = 0; v < NV; v++) e[v] = h * f[v];
    for (int v = 0; v < NV; v++)
      yt[v] = y[v] +
              (-106.0 * a[v] + 273.0 * b[v] - 104.0 * c[v] - 107.0 * d[v] + 48.0 * e[v]) / 6.0;
    tt = t + 2.0 * h / 3.0;
    rhs(tt, yt, f);
    for (int v = 0; v < NV; v++) g[v] = h * f[v];
    for (int v = 0; v < NV; v++)
      yt[v] = y[v] + (110974.0 * a[v] - 236799.0 * b[v] + 68376.0 * c[v] + 103803.0 * d[v] -
                      10240.0 * e[v] + 1926.0 * g[v]) /
                         45648.0;
    tt = t + 5.0 * h / 6.0;
    rhs(tt, yt, f);
    for (int v = 0; v < NV; v++) o[v] = h * f[v];
    for (int v = 0; v < NV; v++)
      yt[v] = y[v] + (-101195.0 * a[v] + 222534.0 * b[v] - 71988.0 * c[v] - 26109.0 * d[v] -
                      2.e4 * e[v] - 72.0 * g[v] + 22824.0 * o[v]) /
                         25994.0;
    tt = t + h;
    rhs(tt, yt, f);
    for (int v = 0; v < NV; v++) p[v] = h * f[v];
    for (int v = 0; v < NV; v++)
      y[v] = y[v] + (41.0 * a[v] + 216.0 * c[v] + 27.0 * d[v] + 272.0 * e[v] + 27.0 * g[v] +
                     216.0 * o[v] + 41.0 * p[v]) /
                        840.0;
    t = tint + i * h;
  }
}

// linear part of every intfunc1_* (Quadrupole.f90:291-304)
void lin_rhs(double Scxl, const double* y, double* f, double s11, double s33, double s55) {
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

void y_start(double* y, const double refpt[6]) {
  std::memset(y, 0, NV * sizeof(double));
  y[4] = refpt[4];
  y[5] = refpt[5];
  y[6] = 1.0; y[9] = 1.0; y[10] = 1.0; y[13] = 1.0; y[14] = 1.0; y[17] = 1.0;
}

// the xm(6,6) assembly of maplinear_* (Quadrupole.f90:183-198)
void xm_from_y(double xm[36], const double* y, double squi, double squf, double sqi3,
               double sqf3, double dlti, double dltf, double thli, double thlf) {
  std::memset(xm, 0, 36 * sizeof(double));
  auto X = [&](int j, int k) -> double& { return xm[(j - 1) + 6 * (k - 1)]; };
  const double* Y = y - 1;
  X(1, 1) = Y[7] * squi / squf + Y[9] * squi / squf * dlti;
  X(2, 1) = (Y[8] - Y[7] * dltf) * squi * squf + (Y[10] - Y[9] * dltf) * squi * squf * dlti;
  X(1, 2) = Y[9] / (squi * squf);
  X(2, 2) = (Y[10] - Y[9] * dltf) * squf / squi;
  X(3, 3) = Y[11] * squi / squf + Y[13] * squi / squf * dlti;
  X(4, 3) = (Y[12] - Y[11] * dltf) * squi * squf + (Y[14] - Y[13] * dltf) * squi * squf * dlti;
  X(3, 4) = Y[13] / (squi * squf);
  X(4, 4) = (Y[14] - Y[13] * dltf) * squf / squi;
  X(5, 5) = Y[15] * sqi3 / sqf3 + Y[17] * sqi3 / sqf3 * thli;
  X(6, 5) = (Y[16] - Y[15] * thlf) * sqi3 * sqf3 + (Y[18] - Y[17] * thlf) * sqi3 * sqf3 * thli;
  X(5, 6) = Y[17] / (sqi3 * sqf3);
  X(6, 6) = (Y[18] - Y[17] * thlf) * sqf3 / sqi3;
}

void uvals(double g, double& u, double& squ, double& sq3) {
  const double beta = std::sqrt(g * g - 1.) / g;
  u = g * beta;
  squ = std::sqrt(u);
  const double s = std::sqrt(u);
  sq3 = s * s * s;
}
}  // namespace

void maplinear_quad(const Phys& P, double t, double tau, double xm[36], double refpt[6],
                    double gradient, int mapstp, double chg, double mass,
                    const impz_elem_t* fringe, double zedge) {
  // maplinear_Quadrupole (Quadrupole.f90:120-200), intfunc1 (254-305); a
  // fringe-field quadrupole takes its gradient from the profile table
  // (getfldfrg_Quadrupole, Quadrupole.f90:404-430: bisection and linear
  // interpolation at t - zedge)
  auto grad_at = [&](double tt) {
    if (!fringe) return gradient;
    const double zz = tt - zedge;
    const double* zd = fringe->zdat - 1;
    const double* gd = fringe->edat - 1;
    int klo = 1, khi = fringe->ndata;
    while (khi - klo > 1) {
      const int k = (khi + klo) / 2;
      if (zd[k] > zz) khi = k;
      else klo = k;
    }
    const double hstep = zd[khi] - zd[klo];
    const double slope = (gd[khi] - gd[klo]) / hstep;
    return gd[klo] + slope * (zz - zd[klo]);
  };
  double y[NV];
  y_start(y, refpt);
  const double h = tau / mapstp;
  double ui, squi, sqi3, uf, squf, sqf3;
  uvals(-refpt[5], ui, squi, sqi3);
  const double qmcc = chg / mass;
  rk6(h, mapstp, t, y, [&](double tt, const double* yy, double* f) {
    const double bgrad = grad_at(tt);
    f[0] = 0.0; f[1] = 0.0; f[2] = 0.0; f[3] = 0.0;
    const double gamma0 = -yy[5];
    const double beta0 = std::sqrt(gamma0 * gamma0 - 1.) / gamma0;
    const double gbet = std::sqrt((gamma0 - 1.0) * (gamma0 + 1.0));
    f[4] = 1.0 / (beta0 * P.Scxl);
    f[5] = 0.0;
    const double brho = gbet / P.Clight / qmcc;
    const double s11 = bgrad / brho * P.Scxl;
    const double s33 = -(bgrad / brho * P.Scxl);
    lin_rhs(P.Scxl, yy, f, s11, s33, 0.0);
  });
  refpt[4] = y[4];
  refpt[5] = y[5];
  uvals(-refpt[5], uf, squf, sqf3);
  xm_from_y(xm, y, squi, squf, sqi3, sqf3, 0.0, 0.0, 0.0, 0.0);
}

namespace {
// getaxfldE_CCL (CCL.f90:331-365): bisection and linear interpolation
void ccl_field(const impz_elem_t& e, double zedge, double z, double& ez1, double& ezp1,
               double& ezpp1) {
  const double escale = e.val[0];
  const double zz = z - zedge;
  int klo = 1, khi = e.ndata;
  const double* zd = e.zdat - 1;
  const double* ed = e.edat - 1;
  const double* epd = e.epdat - 1;
  const double* eppd = e.eppdat - 1;
  while (khi - klo > 1) {
    const int k = (khi + klo) / 2;
    if (zd[k] > zz) khi = k;
    else klo = k;
  }
  const double hstep = zd[khi] - zd[klo];
  double slope = (ed[khi] - ed[klo]) / hstep;
  ez1 = ed[klo] + slope * (zz - zd[klo]);
  slope = (epd[khi] - epd[klo]) / hstep;
  ezp1 = epd[klo] + slope * (zz - zd[klo]);
  slope = (eppd[khi] - eppd[klo]) / hstep;
  ezpp1 = eppd[klo] + slope * (zz - zd[klo]);
  ez1 = ez1 * escale;
  ezp1 = ezp1 * escale;
  ezpp1 = ezpp1 * escale;
}
}  // namespace

namespace {
// the transverse blocks of a solenoid's map with its rotation
// y(19..22) (SolRF.f90:216-235, Sol.f90:181-200), each entry written as the
// reference writes it
void rotate_blocks(double xm[36], const double* y, double squi, double squf, double dlti,
                   double dltf) {
  auto X = [&](int j, int k) -> double& { return xm[(j - 1) + 6 * (k - 1)]; };
  const double* Y = y - 1;
  for (int r = 0; r < 2; r++) {  // rows 1,2 from the x block, 3,4 from y
    const int a = r == 0 ? 7 : 11;          // first y index of the block
    const double ca = Y[r == 0 ? 19 : 21];  // factor for the x columns
    const double cb = Y[r == 0 ? 20 : 22];  // factor for the y columns
    const int j = 2 * r + 1;
    const double m1 = Y[a] * squi / squf + Y[a + 2] * squi / squf * dlti;
    const double m2 = (Y[a + 1] - Y[a] * dltf) * squi * squf +
                      (Y[a + 3] - Y[a + 2] * dltf) * squi * squf * dlti;
    X(j, 1) = ca * m1;
    X(j + 1, 1) = ca * m2;
    X(j, 2) = ca * Y[a + 2] / (squi * squf);
    X(j + 1, 2) = ca * (Y[a + 3] - Y[a + 2] * dltf) * squf / squi;
    X(j, 3) = cb * m1;
    X(j + 1, 3) = cb * m2;
    X(j, 4) = cb * Y[a + 2] / (squi * squf);
    X(j + 1, 4) = cb * (Y[a + 3] - Y[a + 2] * dltf) * squf / squi;
  }
}

// getaxfldE_SolRF (SolRF.f90:355-466): the on-axis field as the Fourier
// series of read3_Data's coefficients F (F(1) their count, F(2..4) the
// series' start, end and period within the element, then the constant,
// cosine and sine terms), zero outside the element and the series' range
void solrf_field(const Phys& P, const impz_elem_t& e, double zedge, double z, double& ez1,
                 double& ezp1) {
  const double escale = e.val[0];
  const double len = e.length;
  const double epstol = (double)1.0e-10f;
  const double* F = e.zdat - 1;  // F(1..ndata)
  ez1 = 0.0;
  ezp1 = 0.0;
  if (!((z >= zedge && z <= zedge + len) || std::fabs(z - zedge) <= epstol ||
        std::fabs(z - zedge - len) <= epstol))
    return;
  const double zlc = z - zedge;
  const int numpar1 = (int)(F[1] + 0.1);
  const double zstart1 = F[2], zend1 = F[3], zlength1 = F[4];
  if (!((zlc >= zstart1 && zlc <= zend1) || std::fabs(zlc - zstart1) <= epstol ||
        std::fabs(zlc - zend1) <= epstol))
    return;
  const double zmid = zlength1 / 2;
  const double zz = z - zedge - zstart1 - zmid;
  const double zlen = zlength1;
  const int ntmp = 4;
  ez1 = F[ntmp + 1] / 2;
  for (int i = 2; i <= (numpar1 - 1) / 2 + 1; i++) {
    const double arg = (i - 1) * 2 * P.Pi * zz / zlen;
    const double c = std::cos(arg), s = std::sin(arg);
    ez1 = ez1 + F[2 * i - 2 + ntmp] * c + F[2 * i - 1 + ntmp] * s;
    ezp1 = ezp1 + (i - 1) * 2 * P.Pi / zlen * (-F[2 * i - 2 + ntmp] * s + F[2 * i - 1 + ntmp] * c);
  }
  ez1 = ez1 * escale;
  ezp1 = ezp1 * escale;
}
}  // namespace

void maplinear_constfoc(const Phys& P, double t, double tau, double xm[36], double refpt[6],
                        const double k2[3], int mapstp) {
  // maplinear_ConstFoc / intfunc1_ConstFoc (ConstFoc.f90): constant
  // focusing kx0^2, ky0^2, kz0^2 = Param(2..4)
  const double Scxl = P.Scxl;
  double y[NV];
  y_start(y, refpt);
  const double h = tau / mapstp;
  double ui, squi, sqi3;
  uvals(-refpt[5], ui, squi, sqi3);
  rk6(h, mapstp, t, y, [&](double, const double* yy, double* f) {
    f[0] = 0.0; f[1] = 0.0; f[2] = 0.0; f[3] = 0.0;
    const double gamma0 = -yy[5];
    const double beta0 = std::sqrt(gamma0 * gamma0 - 1.) / gamma0;
    f[4] = 1.0 / (beta0 * Scxl);
    f[5] = 0.0;
    lin_rhs(Scxl, yy, f, k2[0] * Scxl, k2[1] * Scxl, k2[2] * Scxl);
  });
  refpt[4] = y[4];
  refpt[5] = y[5];
  double uf, squf, sqf3;
  uvals(-refpt[5], uf, squf, sqf3);
  xm_from_y(xm, y, squi, squf, sqi3, sqf3, 0.0, 0.0, 0.0, 0.0);
}

void maplinear_sol(const Phys& P, double t, double tau, double xm[36], double refpt[6],
                   double b0, int mapstp, double chg, double mass) {
  // maplinear_Sol (Sol.f90:120-210), intfunc1_Sol (264-316): a constant
  // solenoid field b0 = Param(2), its focusing s11 = s33 = (b0/2/brho)^2 and
  // its rotation in four more variables
  const double Scxl = P.Scxl;
  const double qmcc = chg / mass;
  double y[22];
  y_start(y, refpt);
  y[18] = 1.0; y[19] = 0.0; y[20] = 0.0; y[21] = 1.0;
  const double h = tau / mapstp;
  double ui, squi, sqi3;
  uvals(-refpt[5], ui, squi, sqi3);
  rk6<22>(h, mapstp, t, y, [&](double, const double* yy, double* f) {
    f[0] = 0.0; f[1] = 0.0; f[2] = 0.0; f[3] = 0.0;
    const double gamma0 = -yy[5];
    const double beta0 = std::sqrt(gamma0 * gamma0 - 1.) / gamma0;
    const double gbet = std::sqrt((gamma0 - 1.0) * (gamma0 + 1.0));
    f[4] = 1.0 / (beta0 * Scxl);
    f[5] = 0.0;
    const double brho = gbet / P.Clight / qmcc;
    const double sol = 0.5 * b0 / brho;
    const double s11 = (sol * sol) * Scxl;
    lin_rhs(Scxl, yy, f, s11, s11, 0.0);
    const double c2alpha = -b0 / brho / 2;
    f[18] = -c2alpha * yy[20];
    f[19] = -c2alpha * yy[21];
    f[20] = c2alpha * yy[18];
    f[21] = c2alpha * yy[19];
  });
  refpt[4] = y[4];
  refpt[5] = y[5];
  double uf, squf, sqf3;
  uvals(-refpt[5], uf, squf, sqf3);
  xm_from_y(xm, y, squi, squf, sqi3, sqf3, 0.0, 0.0, 0.0, 0.0);
  rotate_blocks(xm, y, squi, squf, 0.0, 0.0);
}

bool solrf_table_ok(const impz_elem_t& e) {
  if (e.ndata < 5 || !e.zdat) return false;
  const int numpar1 = (int)(e.zdat[0] + 0.1);
  // the series reads F(5 .. numpar1+4)
  return numpar1 >= 1 && numpar1 + 4 <= e.ndata && e.zdat[3] != 0.0;
}

void maplinear_solrf(const Phys& P, double t, double tau, double xm[36], double refpt[6],
                     double zedge, const impz_elem_t& e, double chg, double mass) {
  // maplinear_SolRF (SolRF.f90:126-233), intfunc1_SolRF (287-353): the RF
  // gap's map plus a constant solenoid b0 = Param(12) = val[10], its
  // focusing in s11 = s33 and its rotation in four more variables
  const double Scxl = P.Scxl;
  const double ww = e.val[1] / P.Scfreq;
  const double theta0 = e.val[2] * (double)std::asin(1.0f) / 90;
  const double qmcc = chg / mass;
  const double b0 = e.val[10];
  double y[22];
  y_start(y, refpt);
  y[18] = 1.0; y[19] = 0.0; y[20] = 0.0; y[21] = 1.0;
  const double h = tau / e.mapstp;
  const double gi = -refpt[5];
  const double betai = std::sqrt(gi * gi - 1.) / gi;
  double ui, squi, sqi3;
  uvals(gi, ui, squi, sqi3);
  double ein, e1in;
  solrf_field(P, e, zedge, t, ein, e1in);
  const double sinthi = std::sin(ww * refpt[4] + theta0);
  const double costhi = std::cos(ww * refpt[4] + theta0);
  const double uprimi = qmcc * ein / betai * costhi;
  const double qpwi = 0.5 * qmcc * Scxl / (ui * ww);
  const double dlti = Scxl * (0.5 * uprimi / ui - qpwi * e1in * sinthi);
  const double thli = 1.5 * Scxl * (uprimi / ui);
  rk6<22>(h, e.mapstp, t, y, [&](double tt, const double* yy, double* f) {
    double ez1, ezp1;
    solrf_field(P, e, zedge, tt, ez1, ezp1);
    f[0] = 0.0; f[1] = 0.0; f[2] = 0.0; f[3] = 0.0;
    const double gamma0 = -yy[5];
    const double beta0 = std::sqrt(gamma0 * gamma0 - 1.) / gamma0;
    const double gbet = std::sqrt((gamma0 - 1.0) * (gamma0 + 1.0));
    const double sinphi = std::sin(ww * yy[4] + theta0);
    const double cosphi = std::cos(ww * yy[4] + theta0);
    const double rfdsgn = ez1 * cosphi;
    f[4] = 1.0 / (beta0 * Scxl);
    f[5] = -(qmcc * rfdsgn);
    const double brho = gbet / P.Clight / qmcc;
    const double q = qmcc * rfdsgn / (beta0 * beta0) / (gamma0 * gamma0);
    const double s11tmp =
        0.5 * (1.0 + 0.5 * (gamma0 * gamma0)) * (q * q) +
        qmcc * 0.5 / ((beta0 * beta0) * beta0) / ((gamma0 * gamma0) * gamma0) * ez1 * sinphi *
            ww / Scxl;
    const double sol = 0.5 * b0 / brho;
    const double s11 = (s11tmp + sol * sol / 2) * Scxl;
    double s55 = -(1.5 * qmcc / (beta0 * beta0) / gamma0 * ezp1 * cosphi) +
                 ((beta0 * beta0) + 0.5) / ((beta0 * beta0) * beta0) / gamma0 * qmcc * ez1 *
                     sinphi * ww / Scxl +
                 1.5 * (1.0 - 0.5 * (gamma0 * gamma0)) * (q * q);
    s55 = Scxl * s55;
    lin_rhs(Scxl, yy, f, s11, s11, s55);
    const double c2alpha = -b0 / brho / 2;
    f[18] = -c2alpha * yy[20];
    f[19] = -c2alpha * yy[21];
    f[20] = c2alpha * yy[18];
    f[21] = c2alpha * yy[19];
  });
  refpt[4] = y[4];
  refpt[5] = y[5];
  const double gf = -refpt[5];
  const double betaf = std::sqrt(gf * gf - 1.) / gf;
  double uf, squf, sqf3;
  uvals(gf, uf, squf, sqf3);
  double ef, e1f;
  solrf_field(P, e, zedge, t + tau, ef, e1f);
  const double sinthf = std::sin(ww * refpt[4] + theta0);
  const double costhf = std::cos(ww * refpt[4] + theta0);
  const double uprimf = qmcc * ef / betaf * costhf;
  const double qpwf = 0.5 * qmcc * Scxl / (uf * ww);
  const double dltf = Scxl * (0.5 * uprimf / uf - qpwf * e1f * sinthf);
  const double thlf = 1.5 * Scxl * (uprimf / uf);
  xm_from_y(xm, y, squi, squf, sqi3, sqf3, dlti, dltf, thli, thlf);
  rotate_blocks(xm, y, squi, squf, dlti, dltf);
}

namespace {
// one Fourier series of getaxfldE_TWS (TWS.f90:350-466): count, start, end
// and period at F(k0+1..k0+4), terms from F(k0+5); pi is the routine's own
// default-real 2*asin(1.0)
void tws_series(const double* F, int k0, double pi, double zedge, double z, double zlc,
                double epstol, double& ez, double& ezp) {
  const int numpar = (int)(F[k0 + 1] + 0.1);
  const double zstart = F[k0 + 2], zend = F[k0 + 3], zlength = F[k0 + 4];
  if (!((zlc >= zstart && zlc <= zend) || std::fabs(zlc - zstart) <= epstol ||
        std::fabs(zlc - zend) <= epstol))
    return;
  const double zmid = zlength / 2;
  const double zz = z - zedge - zstart - zmid;
  const double zlen = zlength;
  const int ntmp = k0 + 4;
  ez = F[ntmp + 1] / 2;
  for (int i = 2; i <= (numpar - 1) / 2 + 1; i++) {
    const double arg = (i - 1) * 2 * pi * zz / zlen;
    const double c = std::cos(arg), s = std::sin(arg);
    ez = ez + F[2 * i - 2 + ntmp] * c + F[2 * i - 1 + ntmp] * s;
    ezp = ezp + (i - 1) * 2 * pi / zlen * (-F[2 * i - 2 + ntmp] * s + F[2 * i - 1 + ntmp] * c);
  }
}

void tws_field(const impz_elem_t& e, double zedge, double z, double& ez1, double& ezp1,
               double& ez12, double& ezp12) {
  const double pi = (double)(2 * std::asin(1.0f));
  const double epstol = (double)1.0e-10f;
  const double escale = e.val[0];
  const double len = e.length;
  const double* F = e.zdat - 1;
  ez1 = ezp1 = ez12 = ezp12 = 0.0;
  if (!((z >= zedge && z <= zedge + len) || std::fabs(z - zedge) <= epstol ||
        std::fabs(z - zedge - len) <= epstol))
    return;
  const double zlc = z - zedge;
  tws_series(F, 0, pi, zedge, z, zlc, epstol, ez1, ezp1);
  ez1 = ez1 * escale;
  ezp1 = ezp1 * escale;
  const int numpar1 = (int)(F[1] + 0.1);
  tws_series(F, numpar1 + 4, pi, zedge, z, zlc, epstol, ez12, ezp12);
  ez12 = ez12 * escale;
  ezp12 = ezp12 * escale;
}
}  // namespace

bool tws_table_ok(const impz_elem_t& e) {
  if (e.ndata < 9 || !e.zdat) return false;
  const int n1 = (int)(e.zdat[0] + 0.1);
  if (n1 < 1 || n1 + 8 > e.ndata || e.zdat[3] == 0.0) return false;
  const int n2 = (int)(e.zdat[n1 + 4] + 0.1);
  return n2 >= 1 && n1 + 8 + n2 <= e.ndata && e.zdat[n1 + 7] != 0.0;
}

void maplinear_tws(const Phys& P, double t, double tau, double xm[36], double refpt[6],
                   double zedge, const impz_elem_t& e, double chg, double mass) {
  // maplinear_TWS (TWS.f90:129-229), intfunc1_TWS (231-340): the gap's map
  // over two standing waves, the second shifted by theta2 = Param(12)
  const double Scxl = P.Scxl;
  const double ww = e.val[1] / P.Scfreq;
  const double theta0 = e.val[2] * (double)std::asin(1.0f) / 90;
  const double theta2 = e.val[10] * (double)std::asin(1.0f) / 90;
  const double qmcc = chg / mass;
  double y[NV];
  y_start(y, refpt);
  const double h = tau / e.mapstp;
  const double gi = -refpt[5];
  const double betai = std::sqrt(gi * gi - 1.) / gi;
  double ui, squi, sqi3;
  uvals(gi, ui, squi, sqi3);
  double ein, e1in, ein2, e1in2;
  tws_field(e, zedge, t, ein, e1in, ein2, e1in2);
  const double sinthi = std::sin(ww * refpt[4] + theta0);
  const double costhi = std::cos(ww * refpt[4] + theta0);
  const double sinthi2 = std::sin(ww * refpt[4] + theta0 + theta2);
  const double costhi2 = std::cos(ww * refpt[4] + theta0 + theta2);
  const double uprimi = qmcc * (ein * costhi + ein2 * costhi2) / betai;
  const double qpwi = 0.5 * qmcc * Scxl / (ui * ww);
  const double dlti = Scxl * (0.5 * uprimi / ui - qpwi * (e1in * sinthi + e1in2 * sinthi2));
  const double thli = 1.5 * Scxl * (uprimi / ui);
  rk6(h, e.mapstp, t, y, [&](double tt, const double* yy, double* f) {
    double ez1, ezp1, ez12, ezp12;
    tws_field(e, zedge, tt, ez1, ezp1, ez12, ezp12);
    f[0] = 0.0; f[1] = 0.0; f[2] = 0.0; f[3] = 0.0;
    const double gamma0 = -yy[5];
    const double beta0 = std::sqrt(gamma0 * gamma0 - 1.) / gamma0;
    const double sinphi = std::sin(ww * yy[4] + theta0);
    const double cosphi = std::cos(ww * yy[4] + theta0);
    const double sinphi2 = std::sin(ww * yy[4] + theta0 + theta2);
    const double cosphi2 = std::cos(ww * yy[4] + theta0 + theta2);
    const double rfdsgn = ez1 * cosphi + ez12 * cosphi2;
    f[4] = 1.0 / (beta0 * Scxl);
    f[5] = -(qmcc * rfdsgn);
    const double q = qmcc * rfdsgn / (beta0 * beta0) / (gamma0 * gamma0);
    const double es = ez1 * sinphi + ez12 * sinphi2;
    const double s11tmp =
        0.5 * (1.0 + 0.5 * (gamma0 * gamma0)) * (q * q) +
        qmcc * 0.5 / ((beta0 * beta0) * beta0) / ((gamma0 * gamma0) * gamma0) * es * ww / Scxl;
    double s55 = -(1.5 * qmcc / (beta0 * beta0) / gamma0 * (ezp1 * cosphi + ezp12 * cosphi2)) +
                 ((beta0 * beta0) + 0.5) / ((beta0 * beta0) * beta0) / gamma0 * qmcc * es * ww /
                     Scxl +
                 1.5 * (1.0 - 0.5 * (gamma0 * gamma0)) * (q * q);
    s55 = Scxl * s55;
    lin_rhs(Scxl, yy, f, s11tmp * Scxl, s11tmp * Scxl, s55);
  });
  refpt[4] = y[4];
  refpt[5] = y[5];
  const double gf = -refpt[5];
  const double betaf = std::sqrt(gf * gf - 1.) / gf;
  double uf, squf, sqf3;
  uvals(gf, uf, squf, sqf3);
  double ef, e1f, ef2, e1f2;
  tws_field(e, zedge, t + tau, ef, e1f, ef2, e1f2);
  const double sinthf = std::sin(ww * refpt[4] + theta0);
  const double costhf = std::cos(ww * refpt[4] + theta0);
  const double sinthf2 = std::sin(ww * refpt[4] + theta0 + theta2);
  const double costhf2 = std::cos(ww * refpt[4] + theta0 + theta2);
  const double uprimf = qmcc * (ef * costhf + ef2 * costhf2) / betaf;
  const double qpwf = 0.5 * qmcc * Scxl / (uf * ww);
  const double dltf = Scxl * (0.5 * uprimf / uf - qpwf * (e1f * sinthf + e1f2 * sinthf2));
  const double thlf = 1.5 * Scxl * (uprimf / uf);
  xm_from_y(xm, y, squi, squf, sqi3, sqf3, dlti, dltf, thli, thlf);
}

void maplinear_rfgap(const Phys& P, double t, double tau, double xm[36], double refpt[6],
                     double zedge, const impz_elem_t& e, double chg, double mass) {
  // maplinear_CCL (CCL.f90:122-215), intfunc1_CCL (269-328); CCDTL and SC
  // (CCDTL.f90, SC.f90:122-328) are the same map, DTL (DTL.f90:136-347)
  // adds its drift-tube quadrupoles (getBgradfld_DTL, DTL.f90:395-418:
  // Param(7..10) = val[5..8])
  const double Scxl = P.Scxl;
  const bool dtl = e.type == 101;
  const double ww = e.val[1] / P.Scfreq;
  // theta0 = Param(4)*asin(1.0)/90 with a default-real asin(1.0)
  const double theta0 = e.val[2] * (double)std::asin(1.0f) / 90;
  const double qmcc = chg / mass;
  double y[NV];
  y_start(y, refpt);
  const double h = tau / e.mapstp;
  const double gi = -refpt[5];
  const double betai = std::sqrt(gi * gi - 1.) / gi;
  double ui, squi, sqi3;
  uvals(gi, ui, squi, sqi3);
  double ein, e1in, e2in;
  ccl_field(e, zedge, t, ein, e1in, e2in);
  const double sinthi = std::sin(ww * refpt[4] + theta0);
  const double costhi = std::cos(ww * refpt[4] + theta0);
  const double uprimi = qmcc * ein / betai * costhi;
  const double qpwi = 0.5 * qmcc * Scxl / (ui * ww);
  const double dlti = Scxl * (0.5 * uprimi / ui - qpwi * e1in * sinthi);
  const double thli = 1.5 * Scxl * (uprimi / ui);
  rk6(h, e.mapstp, t, y, [&](double tt, const double* yy, double* f) {
    double ez1, ezp1, ezpp1;
    ccl_field(e, zedge, tt, ez1, ezp1, ezpp1);
    f[0] = 0.0; f[1] = 0.0; f[2] = 0.0; f[3] = 0.0;
    const double gamma0 = -yy[5];
    const double beta0 = std::sqrt(gamma0 * gamma0 - 1.) / gamma0;
    const double sinphi = std::sin(ww * yy[4] + theta0);
    const double cosphi = std::cos(ww * yy[4] + theta0);
    const double rfdsgn = ez1 * cosphi;
    f[4] = 1.0 / (beta0 * Scxl);
    f[5] = -(qmcc * rfdsgn);
    const double q = qmcc * rfdsgn / (beta0 * beta0) / (gamma0 * gamma0);
    const double s11tmp =
        0.5 * (1.0 + 0.5 * (gamma0 * gamma0)) * (q * q) +
        qmcc * 0.5 / ((beta0 * beta0) * beta0) / ((gamma0 * gamma0) * gamma0) * ez1 * sinphi *
            ww / Scxl;
    double s55 = -(1.5 * qmcc / (beta0 * beta0) / gamma0 * ezp1 * cosphi) +
                 ((beta0 * beta0) + 0.5) / ((beta0 * beta0) * beta0) / gamma0 * qmcc * ez1 *
                     sinphi * ww / Scxl +
                 1.5 * (1.0 - 0.5 * (gamma0 * gamma0)) * (q * q);
    s55 = Scxl * s55;
    if (dtl) {
      const double zz = tt - zedge;
      const double bgrad = zz < e.val[5] ? e.val[6] : (zz < e.length - e.val[7] ? 0.0 : e.val[8]);
      const double gbet = std::sqrt((gamma0 - 1.0) * (gamma0 + 1.0));
      const double brho = gbet / P.Clight / qmcc;
      lin_rhs(Scxl, yy, f, (s11tmp + bgrad / brho) * Scxl, (s11tmp - bgrad / brho) * Scxl, s55);
    } else {
      lin_rhs(Scxl, yy, f, s11tmp * Scxl, s11tmp * Scxl, s55);
    }
  });
  refpt[4] = y[4];
  refpt[5] = y[5];
  const double gf = -refpt[5];
  const double betaf = std::sqrt(gf * gf - 1.) / gf;
  double uf, squf, sqf3;
  uvals(gf, uf, squf, sqf3);
  double ef, e1f, e2f;
  ccl_field(e, zedge, t + tau, ef, e1f, e2f);
  const double sinthf = std::sin(ww * refpt[4] + theta0);
  const double costhf = std::cos(ww * refpt[4] + theta0);
  const double uprimf = qmcc * ef / betaf * costhf;
  const double qpwf = 0.5 * qmcc * Scxl / (uf * ww);
  const double dltf = Scxl * (0.5 * uprimf / uf - qpwf * e1f * sinthf);
  const double thlf = 1.5 * Scxl * (uprimf / uf);
  xm_from_y(xm, y, squi, squf, sqi3, sqf3, dlti, dltf, thli, thlf);
}

// ---------------------------------------------------------------------
namespace {
int push_op(MapProgram& prog, const MapOp& op) {
  if (prog.nops >= IMPZ_MAXOPS) return IMPZ_ERR_UNSUPPORTED;
  prog.ops[prog.nops++] = op;
  return IMPZ_OK;
}

MapOp blank(MapKind k) {
  MapOp op;
  std::memset(&op, 0, sizeof(op));
  op.kind = k;
  return op;
}

MapOp op_xm6(const double xm[36]) {
  // block-diagonal maps (every maplinear_* of the path) use the 12-entry op
  bool diag = true;
  for (int j = 0; j < 6 && diag; j++)
    for (int k = 0; k < 6; k++)
      if (xm[j + 6 * k] != 0.0 && (j / 2) != (k / 2)) {
        diag = false;
        break;
      }
  if (diag) {
    MapOp op = blank(MAP_XM2);
    for (int b = 0; b < 3; b++) {
      const int r = 2 * b;
      op.c[4 * b + 0] = xm[r + 6 * r];
      op.c[4 * b + 1] = xm[r + 6 * (r + 1)];
      op.c[4 * b + 2] = xm[(r + 1) + 6 * r];
      op.c[4 * b + 3] = xm[(r + 1) + 6 * (r + 1)];
    }
    return op;
  }
  MapOp op = blank(MAP_XM6);
  unsigned long long mask = 0;
  for (int q = 0; q < 36; q++) {
    op.c[q] = xm[q];
    if (xm[q] != 0.0) mask |= 1ull << q;
  }
  op.flags = (int)(unsigned)(mask & 0xffffffffull);
  op.iparam = (int)(unsigned)(mask >> 32);
  return op;
}

double pipe_radius(const impz_elem_t& e) {
  // getradius_BeamLineElem (BeamLineElem.f90:500-552)
  switch (e.type) {
    case 0: return e.val[0];
    case 1: return e.val[2];
    case 2: return e.val[3];  // ConstFoc: Param(5)
    case 3: return e.val[2];  // Sol: Param(4)
    case 4: return e.val[3];
    case 5: return e.val[3];  // Multipole: Param(5)
    default: return e.val[4];
  }
}
}  // namespace

int half_map_ops(const Phys& P, const impz_elem_t& e, double zedge, double z, double tau,
                 int nst, int ihlf, double refptcl[6], const Species& sp, MapProgram& prog) {
  const double Scxl = P.Scxl;
  if (e.type == 0) {
    // exact drift (BeamBunch.f90:276-298)
    const double gam0 = -refptcl[5];
    const double gambet0 = std::sqrt(gam0 * gam0 - 1.0);
    const double beta0 = gambet0 / gam0;
    MapOp op = blank(MAP_DRIFT);
    op.c[0] = gam0; op.c[1] = beta0; op.c[2] = tau; op.c[3] = Scxl;
    refptcl[4] = refptcl[4] + tau / (Scxl * beta0);
    return push_op(prog, op);
  }
  if (e.type == 1) {
    const double x3 = e.val[1];
    if (x3 < -10.0) {
      // transfUndulator_Quadrupole (Quadrupole.f90:611-665); kqlh = Param(2)
      const double beta0 = std::sqrt(1.0 - 1.0 / (refptcl[5] * refptcl[5]));
      const double kqlh = e.val[0];
      const double argh = tau * std::sqrt(kqlh);
      const double argh2 = argh * argh, argh4 = argh2 * argh2, argh6 = argh4 * argh2;
      const double sincargh = 1 - argh2 / 6 + argh4 / 120 - argh6 / 5040;
      MapOp op = blank(MAP_UNDUL);
      op.c[0] = refptcl[5]; op.c[1] = beta0; op.c[2] = tau; op.c[3] = Scxl;
      op.c[4] = 1.0; op.c[5] = tau; op.c[6] = 0.0; op.c[7] = 1.0;
      op.c[8] = std::cos(tau * std::sqrt(kqlh));
      op.c[9] = tau * sincargh;
      op.c[10] = -std::sin(tau * std::sqrt(kqlh)) * std::sqrt(kqlh);
      op.c[11] = std::cos(tau * std::sqrt(kqlh));
      refptcl[4] = refptcl[4] + tau / beta0 / Scxl;
      return push_op(prog, op);
    }
    if (x3 < -1.0e-6) {
      // transfmapK_Quadrupole (Quadrupole.f90:509-607)
      const double gambet0 = std::sqrt(refptcl[5] * refptcl[5] - 1.0);
      const double beta0 = std::sqrt(1.0 - 1.0 / (refptcl[5] * refptcl[5]));
      MapOp op = blank(MAP_KQUAD);
      op.c[0] = refptcl[5]; op.c[1] = gambet0; op.c[2] = beta0;
      op.c[3] = sp.charge / sp.mass; op.c[4] = e.val[0]; op.c[5] = tau;
      op.c[6] = Scxl; op.c[7] = sp.qmi;
      refptcl[4] = refptcl[4] + tau / beta0 / Scxl;
      return push_op(prog, op);
    }
    // a gradient profile (read1_Data, AccSimulator.f90:853-863) when v2 > 1e-5
    const bool fringe = x3 > 1.0e-5;
    if (fringe && !(e.ndata > 1 && e.zdat && e.edat)) return IMPZ_ERR_UNSUPPORTED;
    if (e.mapstp < 1) return IMPZ_ERR_ARG;
    double xm[36];
    maplinear_quad(P, z, tau, xm, refptcl, e.val[0], e.mapstp, sp.charge, sp.mass,
                   fringe ? &e : nullptr, zedge);
    return push_op(prog, op_xm6(xm));
  }
  if (e.type == 2) {
    // ConstFoc through drift1's generic branch (Param(5), its radius, >= 0)
    if (e.val[3] < 0.0) return IMPZ_ERR_UNSUPPORTED;
    if (e.mapstp < 1) return IMPZ_ERR_ARG;
    double xm[36];
    maplinear_constfoc(P, z, tau, xm, refptcl, e.val, e.mapstp);
    return push_op(prog, op_xm6(xm));
  }
  if (e.type == 3) {
    // drift1_BeamBunch's generic branch: maplinear_Sol unless Param(5) < 0
    // (the ideal-gap test, which a solenoid only meets with a negative x
    // misalignment; left out)
    if (e.val[3] < 0.0) return IMPZ_ERR_UNSUPPORTED;
    if (e.mapstp < 1) return IMPZ_ERR_ARG;
    double xm[36];
    maplinear_sol(P, z, tau, xm, refptcl, e.val[0], e.mapstp, sp.charge, sp.mass);
    return push_op(prog, op_xm6(xm));
  }
  if (e.type >= 101 && e.type <= 106) {
    if (e.val[3] < 0.0) {
      // ideal RF gap (BeamBunch.f90:324-440)
      const double vtmp = e.val[0] / sp.mass;
      const double harm = e.val[1] / P.Scfreq;
      const double phi0lc = e.val[2] * std::asin(1.0) / 90;
      MapOp op = blank(MAP_IDEALRF);
      const int nseg = e.nseg;
      op.flags = ((nst == 1 && ihlf % 2 == 0) ? 1 : 0) | ((nst == nseg && ihlf % 2 == 1) ? 2 : 0);
      op.iparam = 2 * nseg;
      const double gam0 = -refptcl[5];
      const double gambet = std::sqrt(gam0 * gam0 - 1.0);
      double beta0 = gambet / gam0;
      refptcl[4] = refptcl[4] + 0.5 * tau / (Scxl * beta0);
      refptcl[5] = refptcl[5] - tau * vtmp * std::cos(phi0lc);
      const double gam0o = -refptcl[5];
      const double gambet0 = std::sqrt(gam0o * gam0o - 1.0);
      beta0 = gambet0 / gam0o;
      refptcl[4] = refptcl[4] + 0.5 * tau / (Scxl * beta0);
      op.c[0] = vtmp; op.c[1] = harm; op.c[2] = phi0lc; op.c[3] = Scxl; op.c[4] = tau;
      op.c[5] = gam0; op.c[6] = gambet; op.c[7] = gam0o; op.c[8] = std::cos(phi0lc);
      return push_op(prog, op);
    }
    if (e.type <= 104 && e.ndata > 1 && e.zdat && e.edat && e.epdat && e.eppdat) {
      if (e.mapstp < 1) return IMPZ_ERR_ARG;
      double xm[36];
      maplinear_rfgap(P, z, tau, xm, refptcl, zedge, e, sp.charge, sp.mass);
      return push_op(prog, op_xm6(xm));
    }
    if (e.type == 105 && solrf_table_ok(e)) {
      if (e.mapstp < 1) return IMPZ_ERR_ARG;
      double xm[36];
      maplinear_solrf(P, z, tau, xm, refptcl, zedge, e, sp.charge, sp.mass);
      return push_op(prog, op_xm6(xm));
    }
    if (e.type == 106 && tws_table_ok(e)) {
      if (e.mapstp < 1) return IMPZ_ERR_ARG;
      double xm[36];
      maplinear_tws(P, z, tau, xm, refptcl, zedge, e, sp.charge, sp.mass);
      return push_op(prog, op_xm6(xm));
    }
    return IMPZ_ERR_UNSUPPORTED;
  }
  return IMPZ_ERR_UNSUPPORTED;
}

namespace {
MapOp pole_op(const Phys& P, MapKind kind, double h0, double h1, double tanphi, double tanphib,
              double k1, double psi, double ang, double gam0, const Species& sp, double qm0) {
  // preamble of Fpol_Dipole / Bpol_Dipole (Dipole.f90:478-486, 541-550)
  MapOp op = blank(kind);
  const double tanphi2 = tanphi * tanphi;
  const double secphi2 = 1.0 + tanphi2;
  const double secphi = 1.0 / std::cos(ang);
  const double secphi3 = secphi2 * secphi;
  const double secphib2 = 1. + tanphib * tanphib;
  const double beta0 = std::sqrt(1.0 - 1.0 / (gam0 * gam0));
  const double gambet = beta0 * gam0;
  const double c[16] = {h0,      h1,       tanphi,  tanphib, k1,  psi, tanphi2, secphi2,
                        secphi3, secphib2, beta0,   gambet,  gam0, qm0, sp.qmi, P.Scxl};
  std::memcpy(op.c, c, sizeof(c));
  return op;
}
}  // namespace

int bend_entry_ops(const Phys& P, const impz_elem_t& e, double refptcl[6], const Species& sp,
                   BendState& bs, MapProgram& prog) {
  // AccSimulator.f90:1032-1094; dparam(k) = val[k-2]
  const double* dp = e.val - 2;
  if (e.length == 0.0) return IMPZ_ERR_ARG;
  const double blength = e.length;
  bs.active = true;
  bs.gamma0 = -refptcl[5];
  bs.beta0 = std::sqrt(1.0 - 1.0 / bs.gamma0 / bs.gamma0);
  refptcl[4] = refptcl[4] + blength / (P.Scxl * bs.beta0);
  const double hgap = 2 * dp[5];
  const double ang0 = dp[2];
  bs.hd1 = dp[3];
  const double angF = dp[6];
  bs.angB = dp[7];
  const double hF = dp[8];
  bs.hB = dp[9];
  const double dstr1 = dp[10], dstr2 = dstr1;
  bs.hd0 = ang0 / blength;
  const double tanphiF = std::tan(angF);
  const double psi1 =
      bs.hd0 * hgap * dstr1 * (1.0 + std::sin(angF) * std::sin(angF)) / std::cos(angF);
  const double tanphiFb = std::tan(angF - psi1);
  bs.tanphiB = std::tan(bs.angB);
  bs.psi2 = bs.hd0 * hgap * dstr2 * (1.0 + std::sin(bs.angB) * std::sin(bs.angB)) /
            std::cos(bs.angB);
  bs.tanphiBb = std::tan(bs.angB - bs.psi2);
  bs.qm0 = sp.charge / sp.mass;
  return push_op(prog, pole_op(P, MAP_FPOL, bs.hd0, hF, tanphiF, tanphiFb, bs.hd1, psi1, angF,
                               bs.gamma0, sp, bs.qm0));
}

void bend_sector_op(const Phys& P, const BendState& bs, double len, const Species& sp,
                    MapProgram& prog) {
  // Sector_Dipole coefficients (Dipole.f90:709-749)
  const double h0 = bs.hd0, beta0 = bs.beta0;
  const double rho = 1.0 / h0, theta = len * h0;
  const double st = std::sin(theta), ct = std::cos(theta), sh = std::sin(theta / 2.0);
  MapOp op = blank(MAP_SECTOR);
  const double R16 = rho * (1.0 - ct), R26 = st;
  const double T522 = -(0.5 * rho * st);
  const double gambet = beta0 / std::sqrt(1.0 - beta0 * beta0);
  const double gam2 = 1.0 / (1.0 - beta0 * beta0);
  const double gam0 = std::sqrt(gam2);
  const double c[33] = {ct,
                        rho * st,
                        R16,
                        -st / rho,
                        ct,
                        R26,
                        -R26,
                        -R16,
                        rho * (st - (beta0 * beta0) * theta),
                        -(st * st) / (2.0 * rho),
                        st * ct,
                        st * st,
                        rho * ct * (sh * sh),
                        -(rho * st * (-1.0 + ct)),
                        -(rho * (st * st)) / 2.0,
                        rho * (-1.0 + ct) / 2.0,
                        st / rho,
                        -st / 2.0,
                        -st,
                        -st / 2.0,
                        st,
                        2.0 * rho * (sh * sh),
                        rho * (theta - st),
                        T522,
                        T522,
                        rho * (ct - 1.0),
                        len,
                        beta0,
                        gambet,
                        gam0,
                        bs.qm0,
                        sp.qmi,
                        P.Scxl};
  std::memcpy(op.c, c, sizeof(c));
  push_op(prog, op);
}

void bend_exit_op(const Phys& P, const BendState& bs, const Species& sp, MapProgram& prog) {
  push_op(prog, pole_op(P, MAP_BPOL, bs.hd0, bs.hB, bs.tanphiB, bs.tanphiBb, bs.hd1, bs.psi2,
                        bs.angB, bs.gamma0, sp, bs.qm0));
}

namespace {
// getfldfrgAna2_Quadrupole (Quadrupole.f90:456-506): the Enge profile of a
// quadrupole of gradient bb, effective length Param(3) and aperture Param(4)
// at zz from its entrance, and its first two derivatives.
void quad_enge(double bb, double efflen, double radius, double length, double zz, double& g,
               double& gp, double& gpp) {
  const double c1 = -0.00004, c2 = 4.518219;
  const double dd = 2 * radius;
  const double z10 = (length - efflen) / 2;
  const double z20 = length - z10;
  const double z3 = z10 + 1.5 * dd;
  const double z4 = z20 - 1.5 * dd;
  if (zz < z3 || zz > z4) {
    const double tmpz = zz < z3 ? -(zz - z10) / dd : (zz - z20) / dd;
    const double s1 = c1 + c2 * tmpz;
    const double e1 = std::exp(s1);
    const double one = 1.0 + e1;
    g = bb / one;
    const double s2 = zz < z3 ? -c2 / dd : c2 / dd;
    const double tmp1 = e1 * s2;
    gp = -bb * tmp1 / (one * one);
    const double s3 = 0.0;
    const double s4 = e1 * (s3 + s2 * s2);
    gpp = bb * (-s4 / (one * one) + 2 * tmp1 * tmp1 / (one * one * one));
  } else {
    g = bb;
    gp = 0.0;
    gpp = 0.0;
  }
}

// The on-axis part of getfld_DTL / CCDTL / CCL / SC under the Lorentz
// integrator (DTL.f90:769-855, CCL.f90:525-606, CCDTL.f90, SC.f90): Ez and
// its derivatives from read3_Data's Fourier coefficients (zdat, ndata
// values, the count made odd by a trailing zero, Data.f90:348-409) at z
// from the cell's middle, the radial-expansion factors f1, f1', and the
// DTL's drift-tube quadrupole gradient; pi and c are default-real literals
// there.  c = (G, ez1, ez1', f1, f1', w, theta0, xl c); ez0 = Ez on axis
// at time tg.
void rf_fourier_field(const Phys& P, const impz_elem_t& e, double zedge, double z, double tg,
                      double c[8], double& ez0) {
  const double clite = (double)299792458.0f;
  const double pi = (double)(2 * std::asin(1.0f));
  const double escale = e.val[0];
  const double len = e.length;
  const double zmid = zedge + len / 2;
  const double ww = e.val[1] / P.Scfreq;
  const double xl = P.Scxl / ww;
  const double theta0 = e.val[2] * (double)std::asin(1.0f) / 90;
  double bgrad = 0.0;
  if (e.type == 101) {
    const double zz = z - zedge;
    if (zz < e.val[5])
      bgrad = e.val[6];
    else if (zz < len - e.val[7])
      bgrad = 0.0;
    else
      bgrad = e.val[8];
  }
  const double zz = z - zmid;
  const int nd = e.ndata % 2 == 0 ? e.ndata + 1 : e.ndata;
  auto fc = [&](int i) { return i <= e.ndata ? e.zdat[i - 1] : 0.0; };
  double ez1 = fc(1) / 2, ezp1 = 0.0, ezpp1 = 0.0, ezppp = 0.0;
  for (int i = 2; i <= (nd - 1) / 2 + 1; i++) {
    const double a = fc(2 * i - 2), b = fc(2 * i - 1);
    const double arg = (i - 1) * 2 * pi * zz / len;
    const double k = (i - 1) * 2 * pi / len;
    const double sa = std::sin(arg), ca = std::cos(arg);
    ez1 = ez1 + a * ca + b * sa;
    ezp1 = ezp1 + k * (-(a * sa) + b * ca);
    ezpp1 = ezpp1 + k * k * (-(a * ca) - b * sa);
    ezppp = ezppp + k * k * k * (a * sa - b * ca);
  }
  ez1 = ez1 * escale;
  ezp1 = ezp1 * escale;
  ezpp1 = ezpp1 * escale;
  ezppp = ezppp * escale;
  c[0] = bgrad;
  c[1] = ez1;
  c[2] = ezp1;
  c[3] = -((ezpp1 + ez1 / xl / xl) / 4);
  c[4] = -((ezppp + ezp1 / xl / xl) / 4);
  c[5] = ww;
  c[6] = theta0;
  c[7] = xl * clite;
  // getfld at (0, 0, z, tg): (ez1 + f1 0) cos(w tg + theta0)
  ez0 = (ez1 + c[3] * 0.0) * std::cos(ww * tg + theta0);
}

bool solrf_table_ok(const impz_elem_t& e) {
  if (e.ndata < 5 || !e.zdat) return false;
  const int n1 = (int)(e.zdat[0] + 0.1);
  if (n1 < 1 || n1 + 4 > e.ndata || e.zdat[3] == 0.0) return false;
  if (e.ndata < n1 + 8) return true;
  const int n2 = (int)(e.zdat[n1 + 4] + 0.1);
  return n2 < 3 || (n1 + 8 + n2 <= e.ndata && e.zdat[n1 + 7] != 0.0);
}

// One Fourier series of getfld_SolRF / getfld_TWS (SolRF.f90:482-628,
// TWS.f90): terms from F(ntmp+1), npar of them, at zz from the series'
// middle over its period zlen; Ez and three derivatives.
void fourier_axis(const impz_elem_t& e, int ntmp, int npar, double zz, double zlen,
                  double pi, double& ez1, double& ezp1, double& ezpp1, double& ezppp) {
  auto F = [&](int i) { return i >= 1 && i <= e.ndata ? e.zdat[i - 1] : 0.0; };
  ez1 = F(ntmp + 1) / 2;
  ezp1 = 0.0;
  ezpp1 = 0.0;
  ezppp = 0.0;
  for (int i = 2; i <= (npar - 1) / 2 + 1; i++) {
    const double a = F(2 * i - 2 + ntmp), b = F(2 * i - 1 + ntmp);
    const double arg = (i - 1) * 2 * pi * zz / zlen;
    const double k = (i - 1) * 2 * pi / zlen;
    const double sa = std::sin(arg), ca = std::cos(arg);
    ez1 = ez1 + a * ca + b * sa;
    ezp1 = ezp1 + k * (-(a * sa) + b * ca);
    ezpp1 = ezpp1 + k * k * (-(a * ca) - b * sa);
    ezppp = ezppp + k * k * k * (a * sa - b * ca);
  }
}

// getfld_SolRF / getfld_TWS's terms at z (c as LZ_SOLRF / LZ_TWS) and the
// on-axis Ez at time tg.  The field is zero outside zedge < z < zedge+len
// and each series outside its own [zstart, zend].
void rfw_field(const Phys& P, const impz_elem_t& e, double zedge, double z, double tg,
               double c[16], double& ez0) {
  const double clite = (double)299792458.0f;
  const double pi = (double)(2 * std::asin(1.0f));
  const double escale = e.val[0];
  const double len = e.length;
  const bool tws = e.type == 106;
  for (int i = 0; i < 16; i++) c[i] = 0.0;
  ez0 = 0.0;
  if (!(z > zedge && z < zedge + len)) return;
  auto F = [&](int i) { return i >= 1 && i <= e.ndata ? e.zdat[i - 1] : 0.0; };
  const double ww = e.val[1] * 2 * pi;
  const double xlrep = ww / clite;
  const double theta0 = e.val[2] * (double)std::asin(1.0f) / 90;
  const double tsc = 2 * pi * P.Scfreq;
  c[0] = ww;
  c[1] = xlrep;
  c[2] = tsc;
  c[3] = theta0;
  const double zlc = z - zedge;
  const int numpar1 = (int)(F(1) + 0.1);
  const double zstart1 = F(2), zend1 = F(3), zlength1 = F(4);
  double ez1, ezp1, ezpp1, ezppp;
  const double tt = tg / tsc;
  if (zlc >= zstart1 && zlc <= zend1) {
    fourier_axis(e, 4, numpar1, z - zedge - zstart1 - zlength1 / 2, zlength1, pi, ez1, ezp1,
                 ezpp1, ezppp);
    ez1 = ez1 * escale;
    ezp1 = ezp1 * escale;
    ezpp1 = ezpp1 * escale;
    ezppp = ezppp * escale;
    c[4] = ez1;
    c[5] = ezp1;
    c[6] = -((ezpp1 + ez1 * xlrep * xlrep) / 4);
    c[7] = -((ezppp + ezp1 * xlrep * xlrep) / 4);
    ez0 = 0.0 + (c[4] + c[6] * 0.0) * std::cos(ww * tt + theta0);
  }
  const int numpar2 = (int)(F(5 + numpar1) + 0.1);
  const double zstart2 = F(6 + numpar1), zend2 = F(7 + numpar1), zlength2 = F(8 + numpar1);
  if (zlc >= zstart2 && zlc <= zend2) {
    fourier_axis(e, numpar1 + 8, numpar2, z - zedge - zstart2 - zlength2 / 2, zlength2, pi,
                 ez1, ezp1, ezpp1, ezppp);
    if (tws) {
      ez1 = ez1 * escale;
      ezp1 = ezp1 * escale;
      ezpp1 = ezpp1 * escale;
      ezppp = ezppp * escale;
      c[8] = ez1;
      c[9] = ezp1;
      c[10] = -((ezpp1 + ez1 * xlrep * xlrep) / 4);
      c[11] = -((ezppp + ezp1 * xlrep * xlrep) / 4);
      c[12] = e.val[10] * pi / 180;
      ez0 = ez0 + (c[8] + c[10] * 0.0) * std::cos(ww * tt + theta0 + c[12]);
    } else {
      const double bscale = e.val[10];
      c[8] = bscale * ez1;
      c[9] = bscale * ezp1;
      c[10] = bscale * ezpp1;
      c[11] = bscale * ezppp;
    }
  }
  if (tws) c[12] = e.val[10] * pi / 180;
}

// EMfld 110 as the Lorentz integrator carries it: discrete data (Param(13)
// = 1) on read4_Data's x-y-z grid (Param(14) = 2).  zdat: the three header
// records (xmin, xmax, NxIntvRfg, ymin, ymax, NyIntvRfg, zmin, zmax,
// NzIntvRfg), edat: complex Ex, Ey, Ez, Bx, By, Bz per node (twelve
// doubles, x fastest, then y, then z), ndata: the node count
// (Data.f90:415-554).  The reference's other forms of the element read
// data its driver never loads for it under Flagmap=2 (read2_Data's r-z
// tables, read3_Data's coefficients: AccSimulator.f90:836-846).
bool emfld_ok(const impz_elem_t& e) {
  if (e.type != 110 || !e.zdat || !e.edat) return false;
  if ((int)(0.1 + e.val[11]) != 1 || (int)(0.1 + e.val[12]) != 2) return false;
  const int nx = (int)(e.zdat[2] + 0.1), ny = (int)(e.zdat[5] + 0.1), nz = (int)(e.zdat[8] + 0.1);
  return nx >= 2 && ny >= 2 && nz >= 2 && e.ndata == (nx + 1) * (ny + 1) * (nz + 1);
}

// getfld6xyz_EMfld (EMfld.f90:854-916): the field plane at zz = z - zedge,
// linear between the two end planes of the grid, quadratic over three
// planes elsewhere; appended to `out` (twelve doubles per node, x fastest)
void emfld_plane(const impz_elem_t& e, double zz, std::vector<double>& out) {
  const double* hd = e.zdat;
  const int nxi = (int)(hd[2] + 0.1), nyi = (int)(hd[5] + 0.1), nzi = (int)(hd[8] + 0.1);
  const size_t nxp = nxi + 1, nyp = nyi + 1;
  const double hz = (hd[7] - hd[6]) / nzi;
  int iz = (int)(zz / hz + 1);
  if (iz == nzi + 1) iz = iz - 1;
  auto g = [&](int c, size_t i, size_t j, int k) {
    return e.edat[12 * (i + nxp * (j + nyp * (size_t)(k - 1))) + c];
  };
  const bool lin = iz == 1 || iz == nzi;
  const int iz1 = iz + 1;
  int iz2 = iz;
  double w0 = 0, w1 = 0, w2 = 0;
  if (lin) {
    w0 = (iz * hz - zz) / hz;
    w1 = 1.0 - w0;
  } else {
    const double ab = (zz - (iz - 1) * hz) / hz;
    if (ab <= 0.5) {
      iz2 = iz - 1;
      w0 = 0.75 - ab * ab;
      w1 = (0.5 + ab) * (0.5 + ab) / 2;
      w2 = (0.5 - ab) * (0.5 - ab) / 2;
    } else {
      iz2 = iz + 2;
      w0 = (1.5 - ab) * (1.5 - ab) / 2;
      w1 = 0.75 - (1 - ab) * (1 - ab);
      w2 = (ab - 0.5) * (ab - 0.5) / 2;
    }
  }
  for (size_t j = 0; j < nyp; j++)
    for (size_t i = 0; i < nxp; i++)
      for (int c = 0; c < 12; c++)
        out.push_back(lin ? g(c, i, j, iz) * w0 + g(c, i, j, iz1) * w1
                          : g(c, i, j, iz) * w0 + g(c, i, j, iz1) * w1 + g(c, i, j, iz2) * w2);
}

// The external field of element e for a Lorentz kick at z (LzKind):
// getfld_Quadrupole (Quadrupole.f90:369-402), getfld_ConstFoc
// (ConstFoc.f90:297-322), getfld_Sol (Sol.f90:391-435) and no field for a
// drift.  ez0 is its Ez on axis at time tg.  Returns false for an element
// the Lorentz integrator does not carry here.
bool lorentz_field(const Phys& P, const impz_elem_t& e, double zedge, double z, double tg,
                   int& kind, double c[16], double& ez0, std::vector<double>* data) {
  kind = LZ_NONE;
  for (int i = 0; i < 16; i++) c[i] = 0.0;
  ez0 = 0.0;
  const double zz = z - zedge;
  switch (e.type) {
    case 110: {
      if (!emfld_ok(e)) return false;
      // scatter2 with FlagDisc = 1, FlagCart = 2 (BeamBunch.f90:2604-2632,
      // 2794-2880): c = (escale, ww, theta0, xmin, hx, 1/hx, ymin, hy, 1/hy,
      // NxIntvRfg, NyIntvRfg, offset of the plane in the run's field data)
      kind = LZ_EMFLD;
      const double* hd = e.zdat;
      c[0] = e.val[0];
      c[1] = e.val[1] / P.Scfreq;
      c[2] = e.val[2] * (double)std::asin(1.0f) / 90;
      c[3] = hd[0];
      c[4] = (hd[1] - hd[0]) / (int)(hd[2] + 0.1);
      c[5] = 1.0 / c[4];
      c[6] = hd[3];
      c[7] = (hd[4] - hd[3]) / (int)(hd[5] + 0.1);
      c[8] = 1.0 / c[7];
      c[9] = (int)(hd[2] + 0.1);
      c[10] = (int)(hd[5] + 0.1);
      std::vector<double> local;
      std::vector<double>& pl = data ? *data : local;
      c[11] = (double)pl.size();
      emfld_plane(e, zz, pl);
      // ez0: bilinear at x = y = 0 in the plane's Ez, times escale
      // e^{i(ww tg + theta0)}, real part
      const size_t nxp = (size_t)c[9] + 1;
      const double* q = pl.data() + (size_t)c[11];
      const int ix = (int)((0.0 - c[3]) / c[4] + 1), iy = (int)((0.0 - c[6]) / c[7] + 1);
      const double efx = (c[3] - 0.0 + ix * c[4]) / c[4];
      const double efy = (c[6] - 0.0 + iy * c[7]) / c[7];
      auto ez = [&](int i, int j, int part) {
        return q[12 * ((size_t)(i - 1) + nxp * (size_t)(j - 1)) + 4 + part];
      };
      double sr = 0.0, si = 0.0;
      const int ii[4] = {ix, ix, ix + 1, ix + 1}, jj[4] = {iy, iy + 1, iy, iy + 1};
      const double wa[4] = {efx, efx, 1.0 - efx, 1.0 - efx};
      const double wb[4] = {efy, 1.0 - efy, efy, 1.0 - efy};
      if (ix < 1 || ix > (int)c[9] || iy < 1 || iy > (int)c[10]) return false;
      for (int k = 0; k < 4; k++) {
        sr = k ? sr + ez(ii[k], jj[k], 0) * wa[k] * wb[k] : ez(ii[k], jj[k], 0) * wa[k] * wb[k];
        si = k ? si + ez(ii[k], jj[k], 1) * wa[k] * wb[k] : ez(ii[k], jj[k], 1) * wa[k] * wb[k];
      }
      const double ph = c[1] * tg + c[2];
      ez0 = sr * (c[0] * std::cos(ph)) - si * (c[0] * std::sin(ph));
      return true;
    }
    case 0:
      return true;
    case 1:
      if (e.val[1] <= 0.0) {
        kind = LZ_QUAD;
        c[0] = e.val[0];
        return true;
      }
      // 0 < Param(3) <= 1e-5 reads G', G'' that nothing set
      if (!(e.val[1] > 1.0e-5)) return false;
      kind = LZ_QUAD_FRG;
      quad_enge(e.val[0], e.val[1], e.val[2], e.length, zz, c[0], c[1], c[2]);
      return true;
    case 2:
      kind = LZ_CONSTFOC;
      c[0] = e.val[0];
      c[1] = e.val[1];
      c[2] = e.val[2];
      ez0 = c[2] * tg * P.Scxl;
      return true;
    case 3: {
      const double b0 = e.val[0], x02 = 2 * e.val[2];
      kind = LZ_SOL;
      if (zz >= 0.0 && zz < x02) {
        kind = LZ_SOL_FRG;
        c[0] = b0 / x02;
        c[1] = c[0] * zz;
      } else if (zz >= x02 && zz <= e.length - x02) {
        c[1] = b0;
      } else if (zz > e.length - x02 && zz <= e.length) {
        kind = LZ_SOL_FRG;
        c[0] = -b0 / x02;
        c[1] = b0 + c[0] * (zz - (e.length - x02));
      }
      return true;
    }
    case 101:
    case 102:
    case 103:
    case 104:
      if (!e.zdat || e.ndata < 1 || !(e.length > 0.0)) return false;
      kind = LZ_RF;
      rf_fourier_field(P, e, zedge, z, tg, c, ez0);
      return true;
    case 5: {
      // getfld_Multipole (Multipole.f90:403-452): Param(2) the order,
      // Param(3) the strength, or with Param(4) > 0 the profile
      // getfldfrg_Multipole interpolates (Multipole.f90:455-480) from the
      // element's (z, G) table
      const int idpole = (int)(e.val[0] + 0.1);
      if (idpole < 2 || idpole > 4) return false;
      kind = LZ_MULT;
      c[1] = idpole;
      if (e.val[2] > 0.0) {
        if (!e.zdat || !e.edat || e.ndata < 2) return false;
        const double zz = z - zedge;
        int klo = 1, khi = e.ndata;
        const double* zd = e.zdat - 1;
        const double* ed = e.edat - 1;
        while (khi - klo > 1) {
          const int k = (khi + klo) / 2;
          if (zd[k] > zz) khi = k;
          else klo = k;
        }
        const double hstep = zd[khi] - zd[klo];
        const double slope = (ed[khi] - ed[klo]) / hstep;
        c[0] = ed[klo] + slope * (zz - zd[klo]);
      } else {
        c[0] = e.val[1];
      }
      return true;
    }
    case 105:
    case 106:
      // TWS needs both series; SolRF's solenoid series may be absent (the
      // reference then reads its zero-filled coefficient array: no field)
      if (!(e.type == 106 ? tws_table_ok(e) : solrf_table_ok(e)) || !(e.length > 0.0))
        return false;
      kind = e.type == 105 ? LZ_SOLRF : LZ_TWS;
      rfw_field(P, e, zedge, z, tg, c, ez0);
      return true;
    default:
      return false;
  }
}
}  // namespace

// ---------------------------------------------------------------------
int drift2_op(const Phys& P, double tau, double refptcl[6], MapProgram& prog) {
  MapOp op = blank(MAP_DRIFT2);
  const double gamma0 = -refptcl[5];
  const double beta0 = std::sqrt(1.0 - 1.0 / gamma0 / gamma0);
  op.c[0] = gamma0; op.c[1] = beta0; op.c[2] = P.Scxl; op.c[3] = tau;
  refptcl[4] = refptcl[4] + 0.5 * tau / (P.Scxl * beta0);
  return push_op(prog, op);
}

bool lorentz_kick_terms(const Phys& P, const impz_elem_t& e, double zedge, double z, double tau,
                        const Species& sp, double refptcl[6], int& kind, double c[16],
                        double& tg, double& ez0, std::vector<double>* data) {
  tg = refptcl[4];
  if (!lorentz_field(P, e, zedge, z, tg, kind, c, ez0, data)) return false;
  const double gam = -refptcl[5] + tau * (sp.charge / sp.mass) * ez0;
  refptcl[5] = -gam;
  return true;
}

int compile_lattice(const Phys& P, const impz_elem_t* elems, int nelem, double bcurr,
                    const Species& sp, double refptcl[6], double* zio, LoopState& csr,
                    CompiledLattice& out) {
  struct Half {
    MapProgram prog;
  };
  struct Step {
    MapProgram a, b;
    int sc, csr, wake, lorentz;
    double gam, tau, rad;
    double csr_r0, csr_s0, csr_blen;
    double wk_aa, wk_gg, wk_len;
    int lz_kind;
    double lz_c[16], lz_tg, lz_ez0;
    double z;
    double ref[6];
  };
  std::vector<Step> steps;
  std::vector<double> lz_data;
  MapProgram pending;
  std::memset(&pending, 0, sizeof(pending));
  double z = *zio;
  double ref0[6];  // the initial record's reference particle
  std::memcpy(ref0, refptcl, sizeof(ref0));
  const bool sc_on = !(bcurr < 1.0e-10);
  for (int ie = 0; ie < nelem; ie++) {
    const impz_elem_t& e = elems[ie];
    if (e.type < 0) return IMPZ_ERR_UNSUPPORTED;
    if (e.nseg < 1) return IMPZ_ERR_ARG;
    const int bnseg = e.nseg, bitype = e.type;
    double piperad = pipe_radius(e), piperad2 = piperad;
    if (bitype == 110) piperad2 = e.val[5];  // EMfld: Param(7) (BeamLineElem.f90:538-540)
    // the Lorentz integrator covers drifts, quadrupoles, constant focusing,
    // solenoids, multipoles and the RF cavities 101..106, whose fields
    // kick2 applies (lorentz_field)
    const bool lorentz = csr.flagmap == 2;
    if (lorentz) {
      int kind;
      double c[16], ez0;
      if (!lorentz_field(P, e, z, z, 0.0, kind, c, ez0, nullptr)) return IMPZ_ERR_UNSUPPORTED;
    }
    // the wake switch of each element (AccSimulator.f90:865-875)
    if (bitype == 105 || bitype == 106) {
      csr.aawk = e.val[11];
      csr.ggwk = e.val[12];
      csr.lengwk = e.val[13];
      csr.flagwake = csr.lengwk > 0.0 ? 1 : 0;
    } else if (!csr.flagwakeread) {
      csr.flagwake = 0;
    }
    if (bitype == 4) { piperad = 100.0; piperad2 = 100.0; }
    const double tau1 = 0.5 * e.length / bnseg;
    const double tau2 = 2.0 * tau1;
    const double zedge = z;
    BendState bs;
    std::memset(&bs, 0, sizeof(bs));
    if (bitype == 4) {
      int r = bend_entry_ops(P, e, refptcl, sp, bs, pending);
      if (r) return r;
      piperad2 = e.val[3];
      // AccSimulator.f90:1035-1051, 1088: dparam(4) = val[2]
      csr.r0 = std::fabs(1.0 / bs.hd0);
      if (bcurr > 0.0 && e.val[2] > 500) {
        csr.flagbendcsr = 1;
        csr.bendlencsr = e.length;
        csr.sentr = 0.0;
      } else {
        csr.flagbendcsr = 0;
      }
    }
    int ihlf = 0;
    for (int j = 1; j <= bnseg; j++) {
      Step s;
      std::memset(&s, 0, sizeof(s));
      s.a = pending;
      std::memset(&pending, 0, sizeof(pending));
      for (int half = 0; half < 2; half++) {
        MapProgram& prog = half == 0 ? s.a : s.b;
        if (half == 1) {
          s.sc = sc_on ? 1 : 0;
          s.gam = -refptcl[5];
          s.tau = tau2;
          s.rad = (piperad + piperad2) / 2;
          // CSR inside a bend with dparam(4) > 200, after one with > 500
          // (AccSimulator.f90:1131-1138, 1374-1385)
          if (sc_on && (bitype == 4 ? e.val[2] > 200 : csr.flagbendcsr != 0)) {
            s.csr = 1;
            s.csr_r0 = csr.r0;
            s.csr_s0 = bitype == 4 ? z - csr.zbleng : z - csr.zbleng + csr.sentr;
            s.csr_blen = bitype == 4 ? e.length : csr.bendlencsr;
          }
          if (sc_on && csr.flagwake) {
            s.wake = csr.flagwakeread ? 1 : 2;
            s.wk_aa = csr.aawk;
            s.wk_gg = csr.ggwk;
            s.wk_len = csr.lengwk;
          }
          if (lorentz) {
            // kick2_BeamBunch (BeamBunch.f90:2187-2508): the field at the
            // kick's z and tg = refptcl(5); gamma0 += tau qmcc Ez0 after it
            s.lorentz = 1;
            lorentz_kick_terms(P, e, zedge, z, tau2, sp, refptcl, s.lz_kind, s.lz_c, s.lz_tg,
                               s.lz_ez0, &lz_data);
          }
        }
        if (lorentz) {
          // map1_BeamBunch(Bpts,z,tau2): drift2 by tau2/2 (BeamBunch.f90:467-509)
          int r = drift2_op(P, tau2, refptcl, prog);
          if (r) return r;
          ihlf++;
        } else if (bitype == 4) {
          bend_sector_op(P, bs, tau1, sp, prog);
        } else {
          int r = half_map_ops(P, e, zedge, z, tau1, j, ihlf, refptcl, sp, prog);
          if (r) return r;
          ihlf++;
        }
        z = z + tau1;
      }
      s.z = z;
      std::memcpy(s.ref, refptcl, sizeof(s.ref));
      steps.push_back(s);
    }
    if (bitype == 4) bend_exit_op(P, bs, sp, pending);
    csr.zbleng = csr.zbleng + e.length;  // AccSimulator.f90:1498-1499
    csr.sentr = csr.sentr + e.length;
  }
  const int K = (int)steps.size();
  out.nsteps = K;
  out.has_wake = false;
  out.lz_data.swap(lz_data);
  out.steps.assign(K + 2, StepParams());
  for (auto& st : out.steps) std::memset(&st, 0, sizeof(st));
  out.zrec.assign(K + 1, 0.0);
  out.refrec.assign(6 * (K + 1), 0.0);
  // prologue: initial diagnostics, then the first half map of step 1
  out.zrec[0] = *zio;
  std::memcpy(&out.refrec[0], ref0, sizeof(ref0));
  StepParams& p0 = out.steps[0];
  p0.moments = 1;
  p0.gam = 2.0;
  p0.rad = 1e300;
  for (int s = 0; s <= K; s++) {
    StepParams& sp_ = out.steps[s];
    if (s >= 1) {
      const Step& cur = steps[s - 1];
      sp_.post = cur.b;
      sp_.moments = 1;
      sp_.sc = cur.sc;
      sp_.csr = cur.csr;
      sp_.csr_r0 = cur.csr_r0;
      sp_.csr_s0 = cur.csr_s0;
      sp_.csr_blen = cur.csr_blen;
      sp_.wake = cur.wake;
      sp_.wk_aa = cur.wk_aa;
      sp_.wk_gg = cur.wk_gg;
      sp_.wk_len = cur.wk_len;
      sp_.lorentz = cur.lorentz;
      sp_.lz_kind = cur.lz_kind;
      std::memcpy(sp_.lz_c, cur.lz_c, sizeof(sp_.lz_c));
      sp_.lz_tg = cur.lz_tg;
      sp_.lz_ez0 = cur.lz_ez0;
      if (cur.csr || cur.wake) out.has_wake = true;
      sp_.gam = cur.gam;
      sp_.tau = cur.tau;
      sp_.rad = cur.rad;
      out.zrec[s] = cur.z;
      std::memcpy(&out.refrec[6 * s], cur.ref, 6 * sizeof(double));
    }
    if (s < K) {
      sp_.pre_next = steps[s].a;
      sp_.range_next = steps[s].sc;
    } else {
      sp_.pre_next = pending;  // Bpol of a bend that ends the lattice
      sp_.range_next = 0;
    }
  }
  StepParams& sent = out.steps[K + 1];
  sent.gam = 2.0;
  sent.rad = 1e300;
  *zio = z;
  return IMPZ_OK;
}

// ---------------------------------------------------------------------
void diag_row(const Phys& P, double z, const double rec[IMPZ_MOMREC], const double refptcl[6],
              double mass, double row[IMPZ_DIAG_LEN]) {
  // Output.f90:247-352
  const double* t = rec;
  const double qmc = mass / 1.0e6, xl = P.Scxl, xt = P.Rad2deg;
  const double npt = rec[44], nlocal = rec[45];
  const double den1 = 1.0 / npt;
  const double gam = -refptcl[5];
  const double gambet = std::sqrt(gam * gam - 1.0);
  const double bet = std::sqrt(gam * gam - 1.0) / gam;
  const double energy = (gam - 1.) * qmc;
  const double third = (double)(1.0f / 3.0f);  // (1.0/3.0) in default real
  auto m3 = [&](double c3, double s2, double m) {
    return std::pow(std::fabs(c3 - 3 * s2 * m + 2 * m * m * m), third);
  };
  auto m4 = [&](double c4, double c3, double s2, double m) {
    return std::sqrt(std::sqrt(std::fabs(c4 - 4 * c3 * m + 6 * s2 * m * m - 3 * m * m * m * m)));
  };
  double mean[6], sq[6], var[6];
  for (int c = 0; c < 6; c++) {
    mean[c] = t[c] * den1;
    sq[c] = t[6 + c] * den1;
    var[c] = sq[c] - mean[c] * mean[c];
  }
  const double xpx = t[12] * den1 - mean[0] * mean[1];
  const double ypy = t[13] * den1 - mean[2] * mean[3];
  const double zpz = t[14] * den1 - mean[4] * mean[5];
  double c3[6], c4[6];
  for (int c = 0; c < 6; c++) {
    c3[c] = t[15 + 2 * c] * den1;
    c4[c] = t[16 + 2 * c] * den1;
  }
  double o3[6], o4[6];
  for (int c = 0; c < 6; c++) {
    o3[c] = m3(c3[c], sq[c], mean[c]);
    o4[c] = m4(c4[c], c3[c], sq[c], mean[c]);
  }
  const double epsx2 = var[0] * var[1] - xpx * xpx;
  const double epsy2 = var[2] * var[3] - ypy * ypy;
  const double epsz2 = var[4] * var[5] - zpz * zpz;
  const double epx = std::sqrt(std::fmax(epsx2, 0.0));
  const double epy = std::sqrt(std::fmax(epsy2, 0.0));
  const double epz = std::sqrt(std::fmax(epsz2, 0.0));
  double rms[6];
  for (int c = 0; c < 6; c++) rms[c] = std::sqrt(var[c]);
  const double* gm = rec + 37;
  row[0] = z;
  row[1] = refptcl[4]; row[2] = gam; row[3] = energy; row[4] = bet;
  row[5] = std::sqrt(rec[43]) * xl;
  row[6] = mean[0] * xl; row[7] = rms[0] * xl; row[8] = mean[1] / gambet;
  row[9] = rms[1] / gambet; row[10] = -xpx / epx; row[11] = epx * xl;
  row[12] = mean[2] * xl; row[13] = rms[2] * xl; row[14] = mean[3] / gambet;
  row[15] = rms[3] / gambet; row[16] = -ypy / epy; row[17] = epy * xl;
  row[18] = mean[4] * xt; row[19] = rms[4] * xt; row[20] = mean[5] * qmc;
  row[21] = rms[5] * qmc; row[22] = -zpz / epz; row[23] = epz * qmc * xt;
  row[24] = gm[0] * xl; row[25] = gm[1] / gambet; row[26] = gm[2] * xl;
  row[27] = gm[3] / gambet; row[28] = gm[4] * xt; row[29] = gm[5] * qmc;
  row[30] = nlocal; row[31] = nlocal; row[32] = npt;
  row[33] = o3[0] * xl; row[34] = o3[1] / gambet; row[35] = o3[2] * xl;
  row[36] = o3[3] / gambet; row[37] = o3[4] * xt; row[38] = o3[5] * qmc;
  row[39] = o4[0] * xl; row[40] = o4[1] / gambet; row[41] = o4[2] * xl;
  row[42] = o4[3] / gambet; row[43] = o4[4] * xt; row[44] = o4[5] * qmc;
}

}  // namespace impz
