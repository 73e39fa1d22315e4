// impz_particle.cuh -- per-particle kernels of one space-charge step.
//
// This file is compiled twice: once with --fmad=false into namespace
// impz::exact (the plain FP64 form: every FP64 operation in the reference's
// order, no contraction, so single-step results reproduce the Fortran
// arithmetic bit for bit wherever no transcendental function is involved),
// and once with contraction enabled into impz::fast (the FP32-convolution
// form, which gathers an FP32 field and may fuse multiply-adds).
//
// Kernels:
//   k_advance  -- the fused particle pass: [CIC gather + kick + z-frame]
//                 -> second half map -> moments -> next first half map ->
//                 next conv1st range/loss count -> write (sorted by the
//                 deposit cell when a kick ran).  The last block of the
//                 grid reduces moments and range and runs update_CompDom.
//   k_deposit  -- z->t frame + CIC charge deposit into int64 fixed point
//                 (shared-memory tiles, global atomics for sparse chunks)
//                 + per-cell particle counts.
//   k_scan     -- exclusive scan of the per-cell counts (sort cursors).
#pragma once
#include <cuda_runtime.h>
#include <climits>
#include <cstddef>
#include <stdint.h>

#include "impz_common.h"
#include "impz_device.cuh"

#ifndef IMPZ_FASTMATH
#define IMPZ_FASTMATH 0
#endif

#ifndef IMPZ_NS
#error "define IMPZ_NS (exact or fast) before including impz_particle.cuh"
#endif

namespace impz {
namespace IMPZ_NS {

// conv1st's pilc = 2.0*asin(1.0) evaluated in default (single) precision
// (BeamBunch.f90:1268), i.e. the float nearest pi, widened.
__device__ __constant__ const double kPilc = 3.1415927410125732421875;

struct Particle {
  double x, px, y, py, ph, pt;
};

// ---------------------------------------------------------------------
// transfer maps; each follows the cited reference loop body
__device__ __forceinline__ void map_drift(Particle& p, const volatile double* c) {
  // BeamBunch.f90:286-295; c = {gam0, beta0, tau, Scxl}
  const double gam0 = c[0], beta0 = c[1], tau = c[2], Scxl = c[3];
  double d = p.pt - gam0;
#if IMPZ_FASTMATH
  // one reciprocal square root instead of seven divisions
  const double rt = rsqrt(((d * d - 1.0) - p.px * p.px) - p.py * p.py);
  const double ts = tau / Scxl;
  p.x = p.x + p.px * ts * rt;
  p.y = p.y + p.py * ts * rt;
  p.ph = p.ph - (1.0 / beta0 + d * rt) * ts;
#else
  double tmph = sqrt(((d * d - 1.0) - p.px * p.px) - p.py * p.py);
  p.x = p.x + ((p.px * tau) / tmph) / Scxl;
  p.y = p.y + ((p.py * tau) / tmph) / Scxl;
  p.ph = p.ph - ((1.0 / beta0 + (p.pt - gam0) / tmph) * tau) / Scxl;
#endif
}

// drift2_BeamBunch (BeamBunch.f90:467-509): the Lorentz integrator's drift
// by tau/2; c = {gamma0, beta0, Scxl, tau}
__device__ __forceinline__ void map_drift2(Particle& p, const volatile double* c) {
  const double gamma0 = c[0], beta0 = c[1], xl = c[2], tau = c[3];
  const double g = gamma0 - p.pt;
  const double pz = sqrt(((g * g - 1.0) - p.px * p.px) - p.py * p.py);
  p.x = p.x + 0.5 * tau * p.px / (xl * pz);
  p.y = p.y + 0.5 * tau * p.py / (xl * pz);
  p.ph = p.ph + 0.5 * tau * (g / (xl * pz) - 1.0 / (beta0 * xl));
}

__device__ __forceinline__ void map_xm6(Particle& p, const volatile double* xm, int mask_lo,
                                        int mask_hi) {
  // BeamBunch.f90:310-320: temp(j) = sum_k Pts1(k)*xm(j,k) from 0.0; the
  // zero entries of xm only add signed zeros and are skipped.
  double in[6] = {p.x, p.px, p.y, p.py, p.ph, p.pt};
  double out[6];
  unsigned long long mask = (unsigned long long)(unsigned)mask_lo |
                            ((unsigned long long)(unsigned)mask_hi << 32);
#pragma unroll
  for (int j = 0; j < 6; j++) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 6; k++)
      if (mask & (1ull << (j + 6 * k))) s = s + in[k] * xm[j + 6 * k];
    out[j] = s;
  }
  p.x = out[0]; p.px = out[1]; p.y = out[2]; p.py = out[3]; p.ph = out[4]; p.pt = out[5];
}

// the same loop when xm is block diagonal (drift, quadrupole and RF-gap
// linear maps, xm_from_y in the host builder): row j sums its two nonzero
// entries from 0.0 in column order, exactly as the full loop does.
// c = {xm11, xm12, xm21, xm22, xm33, xm34, xm43, xm44, xm55, xm56, xm65, xm66}
__device__ __forceinline__ void map_xm2(Particle& p, const volatile double* c) {
  const double x = p.x, px = p.px, y = p.y, py = p.py, z = p.ph, pz = p.pt;
  p.x = (0.0 + x * c[0]) + px * c[1];
  p.px = (0.0 + x * c[2]) + px * c[3];
  p.y = (0.0 + y * c[4]) + py * c[5];
  p.py = (0.0 + y * c[6]) + py * c[7];
  p.ph = (0.0 + z * c[8]) + pz * c[9];
  p.pt = (0.0 + z * c[10]) + pz * c[11];
}

// qmi: the particle's Pts1(7) (pts(7,i) of the loop; c[7] holds the bunch's)
__device__ __forceinline__ void map_kquad(Particle& p, const volatile double* c,
                                          const double qmi) {
  // Quadrupole.f90:526-600; c = {refpt6, gambet0, beta0, qmass, K, tau, Scxl, qmi}
  const double refpt6 = c[0], gambet0 = c[1], beta0 = c[2], qmass = c[3], K = c[4];
  const double tau = c[5], Scxl = c[6];
  double gam = -refpt6 - p.pt;
  double gambetz = sqrt(((gam * gam - 1.0) - p.px * p.px) - p.py * p.py);
  double betaz = gambetz / gam;
  gambetz = sqrt(gam * gam - 1.0);
  double kstr = qmi / qmass * gambet0 / gambetz * K;
  double rtkstr = sqrt(fabs(kstr));
  double rtkstrzz = rtkstr * tau;
  double xm11, xm12, xm21, xm22, xm33, xm34, xm43, xm44, cs, ss, t;
  if (kstr > 0.0) {
    sincos(rtkstrzz, &ss, &cs);
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
    sincos(rtkstrzz, &ss, &cs);
    xm33 = cs; xm34 = ss / rtkstr; xm43 = -(ss * rtkstr); xm44 = cs;
  } else {
    xm11 = 1.0; xm12 = tau; xm21 = 0.0; xm22 = 1.0;
    xm33 = 1.0; xm34 = tau; xm43 = 0.0; xm44 = 1.0;
  }
  double t1 = xm11 * p.x + xm12 * p.px / gambetz / Scxl;
  double t2 = gambetz * Scxl * xm21 * p.x + xm22 * p.px;
  double t3 = xm33 * p.y + xm34 * p.py / gambetz / Scxl;
  double t4 = gambetz * Scxl * xm43 * p.y + xm44 * p.py;
  double t5 = p.ph + (1.0 / betaz - 1.0 / beta0) * tau / Scxl;
  p.x = t1; p.px = t2; p.y = t3; p.py = t4; p.ph = t5;
}

// transfUndulator_Quadrupole (Quadrupole.f90:611-665): free in x, the
// undulator's natural focusing in y; c = {refpt6, beta0, tau, Scxl, xm11,
// xm12, xm21, xm22, xm33, xm34, xm43, xm44}
__device__ __forceinline__ void map_undul(Particle& p, const volatile double* c) {
  const double refpt6 = c[0], beta0 = c[1], tau = c[2], Scxl = c[3];
  const double xm11 = c[4], xm12 = c[5], xm21 = c[6], xm22 = c[7];
  const double xm33 = c[8], xm34 = c[9], xm43 = c[10], xm44 = c[11];
  const double gam = -refpt6 - p.pt;
  const double gambetz = sqrt(((gam * gam - 1.0) - p.px * p.px) - p.py * p.py);
  const double betaz = gambetz / gam;
  const double t1 = xm11 * p.x + xm12 * p.px / gambetz / Scxl;
  const double t2 = gambetz * Scxl * xm21 * p.x + xm22 * p.px;
  const double t3 = xm33 * p.y + xm34 * p.py / gambetz / Scxl;
  const double t4 = gambetz * Scxl * xm43 * p.y + xm44 * p.py;
  const double t5 = p.ph + (1.0 / betaz - 1.0 / beta0) * tau / Scxl;
  p.x = t1; p.px = t2; p.y = t3; p.py = t4; p.ph = t5;
}

__device__ __forceinline__ void map_idealrf(Particle& p, const volatile double* c, int flags,
                                            int twonseg) {
  // BeamBunch.f90:337-438; c = {vtmp, harm, phi0lc, Scxl, tau, gam0_in,
  //                            gambet_in, gam0_out, cos(phi0lc)}
  const double vtmp = c[0], harm = c[1], phi0lc = c[2], Scxl = c[3], tau = c[4];
  const double gam0 = c[5], gambet = c[6], gam0o = c[7], c0 = c[8];
  if (flags & 1) {  // entrance focusing kick
    double gam = gam0 - p.pt;
    double gambetz = sqrt(((gam * gam - 1.0) - p.px * p.px) - p.py * p.py);
    double phi = p.ph * harm + phi0lc;
    double vg = vtmp * cos(phi) * Scxl;
    p.px = p.px - 0.5 * vg * gambetz / gam * p.x;
    p.py = p.py - 0.5 * vg * gambetz / gam * p.y;
  }
  {
    double gami_1 = gam0 - p.pt;
    double gambeti_1 = sqrt(gami_1 * gami_1 - 1.0);
    double gambetzi_1 = sqrt(((gami_1 * gami_1 - 1.0) - p.px * p.px) - p.py * p.py);
    double phi = p.ph * harm + phi0lc;
    double dgami = tau * vtmp * cos(phi);
    double gami_2 = gami_1 + dgami;
    double gambeti_2 = sqrt(gami_2 * gami_2 - 1.0);
    double fact;
    if (fabs(vtmp) < 1.0e-10)
      fact = tau / Scxl;
    else
      fact = gambeti_1 / dgami * log(gambeti_2 / gambeti_1) * tau / Scxl;
    p.x = p.x + fact * p.px / gambetzi_1;
    p.y = p.y + fact * p.py / gambetzi_1;
    p.ph = p.ph + (tau / Scxl) / (gambet * gambet * gambet) * p.pt;
  }
  if (flags & 2) {  // exit focusing kick and energy correction
    double gam = gam0o - p.pt;
    double gambetz = sqrt(((gam * gam - 1.0) - p.px * p.px) - p.py * p.py);
    double phi = p.ph * harm + phi0lc;
    double vg = vtmp * cos(phi) * Scxl;
    p.px = p.px + 0.5 * vg * gambetz / gam * p.x;
    p.py = p.py + 0.5 * vg * gambetz / gam * p.y;
    phi = p.ph * harm + phi0lc;
    p.pt = p.pt + (double)twonseg * tau * vtmp * (c0 - cos(phi));
  }
}

// Fpol_Dipole / Bpol_Dipole (Dipole.f90:488-524, 551-589).
// c = {h0, h1, tanphi, tanphib, k1, psi, tanphi2, secphi2, secphi3,
//      secphib2, beta0, gambet, gam0, qm0, qmi, Scxl}; the particle's own
// Pts1(7) is passed as qmi (c[14] holds the bunch's)
template <bool EXIT>
__device__ __forceinline__ void map_pole(Particle& p, const volatile double* c, const double qmi) {
  const double h0 = c[0], h1 = c[1], tanphi = c[2], tanphib = c[3], k1 = c[4], psi = c[5];
  const double tanphi2 = c[6], secphi2 = c[7], secphi3 = c[8], secphib2 = c[9];
  const double beta0 = c[10], gambet = c[11], gam0 = c[12], qm0 = c[13];
  const double Scxl = c[15];
  double x = p.x * Scxl;
  double gamn = gam0 - p.pt;
  double gambetz = sqrt(((gamn * gamn - 1.0) - p.px * p.px) - p.py * p.py);
  double xp = p.px / gambetz;
  double y = p.y * Scxl;
  double yp = p.py / gambetz;
  double z5 = -(p.ph * beta0 * Scxl);
  double d = -(p.pt / beta0 / gambet) - (qmi - qm0) / qm0;
  double a0, a1, a2, a3;
  if (!EXIT) {
    a0 = x - 0.5 * h0 * tanphi2 * (x * x) + 0.5 * h0 * secphi2 * (y * y);
    a1 = h0 * tanphi * x + xp + h0 * tanphi2 * x * xp +
         (0.5 * h0 * h1 * secphi3 + k1 * tanphi) * (x * x) -
         (0.5 * h0 * h1 * secphi3 + k1 * tanphi - (h0 * h0) * tanphi * tanphi2 -
          0.5 * (h0 * h0) * tanphi) * (y * y) -
         h0 * tanphi2 * y * yp - h0 * tanphi * x * d;
    a2 = y + h0 * tanphi2 * x * y;
    a3 = -(h0 * tanphib * y) + yp - h0 * tanphi2 * x * yp - h0 * secphi2 * xp * y -
         (h0 * h1 * secphi3 + 2 * k1 * tanphi) * x * y +
         (h0 * tanphi - h0 * psi * secphib2) * y * d;
  } else {
    a0 = x + 0.5 * h0 * tanphi2 * (x * x) - 0.5 * h0 * secphi2 * (y * y);
    a1 = h0 * tanphi * x + xp - h0 * tanphi2 * x * xp +
         (0.5 * h0 * h1 * secphi3 + k1 * tanphi - (h0 * h0) * tanphi2 * tanphi / 2) * (x * x) -
         (0.5 * h0 * h1 * secphi3 + k1 * tanphi + (h0 * h0) * tanphi * tanphi2 / 2) * (y * y) +
         h0 * tanphi2 * y * yp - h0 * tanphi * x * d;
    a2 = y - h0 * tanphi2 * x * y;
    a3 = -(h0 * tanphib * y) + yp + h0 * tanphi2 * x * yp + h0 * secphi2 * xp * y -
         (h0 * h1 * secphi3 + 2 * k1 * tanphi - (h0 * h0) * secphi2 * tanphi) * x * y +
         (h0 * tanphi - h0 * psi * secphib2) * y * d;
  }
  gambetz = sqrt(gamn * gamn - 1.0) / sqrt((a1 * a1 + a3 * a3) + 1);
  p.x = a0 / Scxl;
  p.px = a1 * gambetz;
  p.y = a2 / Scxl;
  p.py = a3 * gambetz;
  p.ph = -z5 / Scxl / beta0;
  p.pt = -(beta0 * gambet * (d + (qmi - qm0) / qm0));
}

// Sector_Dipole second-order map (Dipole.f90:745-786).
// c = {R11,R12,R16,R21,R22,R26,R51,R52,R56, T111,T112,T116,T122,T126,T166,
//      T144,T216,T222,T266,T244,T314,T324,T346,T522,T544,T526,
//      len, beta0, gambet, gam0, qm0, qmi, Scxl}; the particle's own Pts1(7)
// is passed as qmi (c[31] holds the bunch's)
__device__ __forceinline__ void map_sector(Particle& p, const volatile double* c,
                                           const double qmi) {
  const double R11 = c[0], R12 = c[1], R16 = c[2], R21 = c[3], R22 = c[4], R26 = c[5];
  const double R51 = c[6], R52 = c[7], R56 = c[8];
  const double T111 = c[9], T112 = c[10], T116 = c[11], T122 = c[12], T126 = c[13];
  const double T166 = c[14], T144 = c[15], T216 = c[16], T222 = c[17], T266 = c[18];
  const double T244 = c[19], T314 = c[20], T324 = c[21], T346 = c[22], T522 = c[23];
  const double T544 = c[24], T526 = c[25], len = c[26], beta0 = c[27], gambet = c[28];
  const double gam0 = c[29], qm0 = c[30], Scxl = c[32];
  double gami = -p.pt + gam0;
  double gambeti = sqrt(gami * gami - 1.0);
  double gambetz = sqrt((gambeti * gambeti - p.px * p.px) - p.py * p.py);
  double x0 = p.x * Scxl, xp0 = p.px / gambetz, y0 = p.y * Scxl, yp0 = p.py / gambetz;
  double z0 = -(p.ph * beta0 * Scxl);
  double eta = -(p.pt / beta0 / gambet) - (qmi - qm0) / qm0;
  double a0 = R11 * x0 + R12 * xp0 + R16 * eta + T111 * (x0 * x0) + T112 * x0 * xp0 +
              T116 * x0 * eta + T122 * (xp0 * xp0) + T126 * xp0 * eta + T166 * (eta * eta) +
              T144 * (yp0 * yp0);
  double a1 = R21 * x0 + R22 * xp0 + R26 * eta + T216 * x0 * eta + T222 * (xp0 * xp0) +
              T266 * (eta * eta) + T244 * (yp0 * yp0);
  double a2 = y0 + len * yp0 + T314 * x0 * yp0 + T324 * xp0 * yp0 + T346 * yp0 * eta;
  double a3 = yp0;
  double a4 = R51 * x0 + R52 * xp0 + z0 + R56 * eta + T522 * (xp0 * xp0) + T544 * (yp0 * yp0) +
              T526 * xp0 * eta;
  gambetz = gambeti / sqrt((a1 * a1 + a3 * a3) + 1.0);
  p.x = a0 / Scxl;
  p.px = a1 * gambetz;
  p.y = a2 / Scxl;
  p.py = a3 * gambetz;
  p.ph = -a4 / Scxl / beta0;
  p.pt = -(beta0 * gambet * (eta + (qmi - qm0) / qm0));
}

// Map programs are staged in shared memory and read through volatile
// pointers inside the particle loop: the coefficients are re-read (a
// broadcast shared load) per particle instead of being hoisted into
// registers for every map kind the switch could take.
// LIGHT programs hold only drifts and block-diagonal linear maps (the
// drift/quadrupole lattices); the host picks that instantiation when every
// step of a run qualifies, which keeps the other map kinds' code and
// registers out of the particle pass.
// qmi: the particle's Pts1(7), read by the K-map and the bend maps.
template <bool LIGHT>
__device__ __forceinline__ void apply_program(Particle& p, const volatile MapProgram& prog,
                                              const double qmi) {
  const int nops = prog.nops;
  for (int o = 0; o < nops; o++) {
    const volatile MapOp& op = prog.ops[o];
    if (LIGHT) {
      if (op.kind == MAP_DRIFT) map_drift(p, op.c);
      else if (op.kind == MAP_XM2) map_xm2(p, op.c);
      continue;
    }
    switch (op.kind) {
      case MAP_DRIFT: map_drift(p, op.c); break;
      case MAP_XM6: map_xm6(p, op.c, op.flags, op.iparam); break;
      case MAP_KQUAD: map_kquad(p, op.c, qmi); break;
      case MAP_IDEALRF: map_idealrf(p, op.c, op.flags, op.iparam); break;
      case MAP_FPOL: map_pole<false>(p, op.c, qmi); break;
      case MAP_BPOL: map_pole<true>(p, op.c, qmi); break;
      case MAP_SECTOR: map_sector(p, op.c, qmi); break;
      case MAP_XM2: map_xm2(p, op.c); break;
      case MAP_UNDUL: map_undul(p, op.c); break;
      case MAP_DRIFT2: map_drift2(p, op.c); break;
      default: break;
    }
  }
}

// Copies a step's programs into shared memory (whole block).
__device__ __forceinline__ void stage_programs(MapProgram* dst, const StepParams* sp) {
  const int nw = (int)(2 * sizeof(MapProgram) / sizeof(int));
  const int* src0 = reinterpret_cast<const int*>(&sp->post);
  int* d = reinterpret_cast<int*>(dst);
  for (int e = threadIdx.x; e < nw; e += blockDim.x) d[e] = src0[e];
}

// ---------------------------------------------------------------------
// conv1st z->t frame (BeamBunch.f90:1290-1340), without storing the result
struct TFrame {
  double xt, yt, zt;      // t-frame positions [m]
  double tmpx, tmpy;      // z-frame x*Scxl, y*Scxl (they enter the range)
  double ph;              // wrapped phase
  double rcp, tmpbet;     // 1/gamma_i and 1-beta_i^2-ish (before abs)
  bool lost;
};

// Written with explicit round-to-nearest intrinsics: the deposit (plain
// build) and the fused particle pass (either build) must agree bit for bit
// on the loss test and the cell, whatever contraction the build allows.
__device__ __forceinline__ TFrame to_tframe(const Particle& p, double gam, double rad,
                                            double xl) {
  TFrame t;
  if (fabs(p.ph) < kPilc) {
    // |ph/pilc| < 1 truncates to 0 (the quotient cannot round up to 1), and
    // tmp5 - 0*pilc is ph itself: the wrap is the identity, no division
    t.ph = p.ph;
  } else {
    int ntmp5 = (int)(p.ph / kPilc);
    double tmp5 = __dsub_rn(p.ph, __dmul_rn((double)ntmp5, kPilc));
    t.ph = __dsub_rn(tmp5, __dmul_rn((double)(ntmp5 % 2), kPilc));
  }
  t.rcp = 1.0 / __dadd_rn(-p.pt, gam);
  t.tmpbet = __dsub_rn(1.0, __dmul_rn(__dmul_rn(t.rcp, t.rcp),
                                      __dadd_rn(__dadd_rn(1.0, __dmul_rn(p.px, p.px)),
                                                __dmul_rn(p.py, p.py))));
  double betai = sqrt(fabs(t.tmpbet));
  t.tmpx = __dmul_rn(p.x, xl);
  t.xt = __dmul_rn(__dsub_rn(p.x, __dmul_rn(__dmul_rn(p.px, t.ph), t.rcp)), xl);
  t.tmpy = __dmul_rn(p.y, xl);
  t.yt = __dmul_rn(__dsub_rn(p.y, __dmul_rn(__dmul_rn(p.py, t.ph), t.rcp)), xl);
  t.zt = -__dmul_rn(__dmul_rn(__dmul_rn(gam, betai), t.ph), xl);
  // radtest = sqrt(r2) >= rad; the square root is taken only when r2 lies
  // within 1e-12 of rad^2 (sqrt is monotone and correctly rounded)
  const double r2 = __dadd_rn(__dmul_rn(t.xt, t.xt), __dmul_rn(t.yt, t.yt));
  const double rr = rad * rad;
  bool out;
  if (r2 < rr * (1.0 - 4e-12)) out = false;
  else if (r2 > rr * (1.0 + 4e-12)) out = true;
  else out = sqrt(r2) >= rad;
  t.lost = out || (t.tmpbet <= 0.0);
  return t;
}

// The whole-lattice runner stores a particle between two passes as conv1st
// leaves Pts1 (BeamBunch.f90:1296-1340): x_t and y_t [m] in columns 1 and 3,
// z_t in column 5, the momenta unchanged, and a NaN in column 5 for a
// particle conv1st lost.  cvbkforth1st recomputes 1/gamma_i and beta_i from
// the momenta (BeamBunch.f90:1681-1690), so nothing else is needed; the
// values are those to_tframe returned when the pass stored them.
__device__ __forceinline__ double lost_mark() { return __longlong_as_double(0x7ff8000000000000ll); }

__device__ __forceinline__ TFrame stored_tframe(const Particle& p, double gam) {
  TFrame t;
  t.ph = 0.0;
  t.rcp = 1.0 / __dadd_rn(-p.pt, gam);
  t.tmpbet = __dsub_rn(1.0, __dmul_rn(__dmul_rn(t.rcp, t.rcp),
                                      __dadd_rn(__dadd_rn(1.0, __dmul_rn(p.px, p.px)),
                                                __dmul_rn(p.py, p.py))));
  t.xt = p.x;
  t.yt = p.y;
  t.zt = p.ph;
  t.tmpx = 0.0;
  t.tmpy = 0.0;
  t.lost = isnan(p.ph);
  return t;
}

// deposit_BeamBunch cell and weights (BeamBunch.f90:3737-3742)
struct Cell {
  int ix, jx, kx;   // 1-based like the reference
  double ab, cd, ef;
};

template <typename GT>
__device__ __forceinline__ Cell cic_cell(double x, double y, double z, const GT& g) {
  Cell c;
  c.ix = (int)__dadd_rn(__dmul_rn(__dsub_rn(x, g.range[0]), g.hi[0]), 1.0);
  c.ab = __dmul_rn(__dadd_rn(__dsub_rn(g.range[0], x), __dmul_rn((double)c.ix, g.h[0])), g.hi[0]);
  c.jx = (int)__dadd_rn(__dmul_rn(__dsub_rn(y, g.range[2]), g.hi[1]), 1.0);
  c.cd = __dmul_rn(__dadd_rn(__dsub_rn(g.range[2], y), __dmul_rn((double)c.jx, g.h[1])), g.hi[1]);
  c.kx = (int)__dadd_rn(__dmul_rn(__dsub_rn(z, g.range[4]), g.hi[2]), 1.0);
  c.ef = __dmul_rn(__dadd_rn(__dsub_rn(g.range[4], z), __dmul_rn((double)c.kx, g.h[2])), g.hi[2]);
  return c;
}

// deposit_BeamBunch's test ix < 1 .or. ix+1 > nx (BeamBunch.f90:3746-3747),
// written without the +1: a particle far outside the box converts to a
// saturated INT_MAX, and INT_MAX + 1 would wrap to a negative index.
__device__ __forceinline__ bool cell_inside(const Cell& c, int nx, int ny, int nz) {
  return !(c.ix < 1 || c.ix >= nx || c.jx < 1 || c.jx >= ny || c.kx < 1 || c.kx >= nz);
}

// ---------------------------------------------------------------------
// reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// the 37 sums of diagnostic1_Output (Output.f90:133-196), in tmplc order
__device__ __forceinline__ void moment_accumulate(double* s, const Particle& p) {
  const double x = p.x, px = p.px, y = p.y, py = p.py, z = p.ph, pz = p.pt;
  s[0] += x;  s[1] += px; s[2] += y;  s[3] += py; s[4] += z;  s[5] += pz;
  s[6] += x * x; s[7] += px * px; s[8] += y * y; s[9] += py * py;
  s[10] += z * z; s[11] += pz * pz;
  s[12] += x * px; s[13] += y * py; s[14] += z * pz;
  s[15] += x * x * x; s[16] += x * x * x * x;
  s[17] += px * px * px; s[18] += px * px * px * px;
  s[19] += y * y * y; s[20] += y * y * y * y;
  s[21] += py * py * py; s[22] += py * py * py * py;
  s[23] += fabs(z * z * z); s[24] += z * z * z * z;
  s[25] += pz * pz * pz; s[26] += pz * pz * pz * pz;
  s[27] += x * px * px; s[28] += x * px * px * px; s[29] += x * x * px;
  s[30] += x * x * px * px; s[31] += x * x * x * px;
  s[32] += y * py * py; s[33] += y * py * py * py; s[34] += y * y * py;
  s[35] += y * y * py * py; s[36] += y * y * y * py;
  s[37] = fmax(s[37], fabs(x)); s[38] = fmax(s[38], fabs(px));
  s[39] = fmax(s[39], fabs(y)); s[40] = fmax(s[40], fabs(py));
  s[41] = fmax(s[41], fabs(z)); s[42] = fmax(s[42], fabs(pz));
  s[43] = fmax(s[43], x * x + y * y);
}


template <bool F32>
__device__ __forceinline__ void gather_e(const void* ef, const Cell& c, int nx, int ny,
                                         double& ex, double& ey, double& ez);

// scatter1_BeamBunch gather, FP64 field, reference term order (BeamBunch.f90:2128-2155)
template <>
__device__ __forceinline__ void gather_e<false>(const void* ef, const Cell& c, int nx, int ny,
                                                double& ex, double& ey, double& ez) {
  const int sy = nx, sz = nx * ny;  // a grid holds at most 64 x 64 x 4096 nodes
  const int b = (c.ix - 1) + sy * (c.jx - 1) + sz * (c.kx - 1);
  const double ab = c.ab, cd = c.cd, efw = c.ef;
  const double ab1 = 1.0 - ab, cd1 = 1.0 - cd, ef1 = 1.0 - efw;
  const double2* E = reinterpret_cast<const double2*>(ef);
  const int nodes[8] = {b, b + sy, b + sy + sz, b + sz, b + 1 + sz, b + 1 + sy + sz, b + 1 + sy,
                        b + 1};
  double2 A[8], B[8];
#pragma unroll
  for (int q = 0; q < 8; q++) {
    A[q] = __ldg(E + 2 * nodes[q]);
    B[q] = __ldg(E + 2 * nodes[q] + 1);
  }
  // term q: field * w1 * w2 * w3 evaluated left to right like the reference
#define IMPZ_T(q, w1, w2, w3) \
  sx = sx + A[q].x * w1 * w2 * w3; sy_ = sy_ + A[q].y * w1 * w2 * w3; sz_ = sz_ + B[q].x * w1 * w2 * w3;
  double sx = A[0].x * ab * cd * efw, sy_ = A[0].y * ab * cd * efw, sz_ = B[0].x * ab * cd * efw;
  IMPZ_T(1, ab, cd1, efw)
  IMPZ_T(2, ab, cd1, ef1)
  IMPZ_T(3, ab, cd, ef1)
  IMPZ_T(4, ab1, cd, ef1)
  IMPZ_T(5, ab1, cd1, ef1)
  IMPZ_T(6, ab1, cd1, efw)
  IMPZ_T(7, ab1, cd, efw)
#undef IMPZ_T
  ex = sx; ey = sy_; ez = sz_;
}

// FP32 field gather (FP32-convolution form)
template <>
__device__ __forceinline__ void gather_e<true>(const void* ef, const Cell& c, int nx, int ny,
                                               double& ex, double& ey, double& ez) {
  const int sy = nx, sz = nx * ny;
  const int b = (c.ix - 1) + sy * (c.jx - 1) + sz * (c.kx - 1);
  const float ab = (float)c.ab, cd = (float)c.cd, efw = (float)c.ef;
  const float ab1 = 1.0f - ab, cd1 = 1.0f - cd, ef1 = 1.0f - efw;
  const float4* E = reinterpret_cast<const float4*>(ef);
  const int nodes[8] = {b, b + sy, b + sy + sz, b + sz, b + 1 + sz, b + 1 + sy + sz, b + 1 + sy,
                        b + 1};
  const float w[8] = {ab * cd * efw, ab * cd1 * efw, ab * cd1 * ef1, ab * cd * ef1,
                      ab1 * cd * ef1, ab1 * cd1 * ef1, ab1 * cd1 * efw, ab1 * cd * efw};
  float sx = 0.f, sy_ = 0.f, sz_ = 0.f;
#pragma unroll
  for (int q = 0; q < 8; q++) {
    float4 v = __ldg(E + nodes[q]);
    sx += v.x * w[q]; sy_ += v.y * w[q]; sz_ += v.z * w[q];
  }
  ex = sx; ey = sy_; ez = sz_;
}

// scatter1 kick constants (BeamBunch.f90:2066-2084); fpei uses the
// default-real literal 1.0e-7 of the reference.
__device__ __forceinline__ void kick_consts(const Consts& k, double gam, double curr,
                                            double& xycon, double& tcon) {
  const double tmpscale = curr / k.Scfreq;
  const double twopi = 2.0 * k.Pi;
  const double fpei = k.Clight * k.Clight * 1.00000001168609742e-07;
  const double bet = sqrt(gam * gam - 1.0) / gam;
  const double bbyk = bet / k.xk;
  const double gambet = gam * bet;
  const double brho = gambet / (k.Clight * k.charge) * k.mass;
  const double vz0 = bet * k.Clight;
  const double perv0 = 2.0 * curr * fpei / (brho * vz0 * vz0 * gam * gam);
  xycon = 0.5 * perv0 * gambet * bbyk * twopi / tmpscale;
  tcon = bet * xycon * (gam * gam);
}

// update_CompDom, Flagbc=1 (CompDom.f90:545-557, 614-622): eps is the
// default-real 1.0/(Meshnum-3.0)
__device__ __forceinline__ void compdom(Geom& g, int nx, int ny, int nz) {
  const int mesh[3] = {nx, ny, nz};
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double t1 = g.ptrange[2 * k], t2 = g.ptrange[2 * k + 1];
    double eps = (double)(1.0f / ((float)mesh[k] - 3.0f));
    double mn = t1 - eps * (t2 - t1);
    double mx = t2 + eps * (t2 - t1);
    g.range[2 * k] = mn;
    g.range[2 * k + 1] = mx;
    g.h[k] = (mx - mn) / (double)(mesh[k] - 1);
    g.hi[k] = 1.0 / g.h[k];
  }
}

__device__ __forceinline__ bool finite6(const Particle& p) {
  return isfinite(p.x) && isfinite(p.px) && isfinite(p.y) && isfinite(p.py) &&
         isfinite(p.ph) && isfinite(p.pt);
}

__device__ __forceinline__ long long lin_cell(const Cell& c, int nx, int ny) {
  return (long long)(c.ix - 1) + (long long)nx * ((c.jx - 1) + (long long)ny * (c.kx - 1));
}

// Sort key of the cell with lower node (ix, jx, kx) (0-based; grid sides are
// powers of two >= 4): bricks of 4x4x4 cells in x-fastest order, the cells
// of a brick x-fastest.  The particles are kept in this order and the
// per-cell counts indexed by it, so that a deposit chunk of consecutive
// particles covers a compact box of nodes even where the beam is sparse (in
// plain x-fastest order a chunk over a few thousand sparse cells spans whole
// rows and tens of them, more than the shared tile holds).
__device__ __forceinline__ int cell_key(int ix, int jx, int kx, int nx, int ny) {
  const int brick = ((kx >> 2) * (ny >> 2) + (jx >> 2)) * (nx >> 2) + (ix >> 2);
  return (brick << 6) | ((kx & 3) << 4) | ((jx & 3) << 2) | (ix & 3);
}

// ---------------------------------------------------------------------
// The fused particle pass of step s.  Per particle, in the reference's order:
//   [kick]  conv1st z->t, loss test, deposit cell (sort key),
//           cvbkforth1st t->z->gather frame, scatter1 gather + kick + z frame
//   [post]  second half map of step s, then the diagnostic1 sums
//   [pre]   first half map of step s+1 (and pole faces), conv1st range of s+1
//   write   to the sorted slot of the deposit cell (kick) or in place.
// Each thread carries U particles per iteration (U loads in flight).  The
// 37 moment sums and 7 maxima are not held per thread: every iteration each
// warp reduce-scatters them in groups of eight with a shuffle butterfly
// into its own shared-memory accumulators.  The last block to finish
// reduces moments and range in block order (deterministic) and performs
// conv1st's current rescale and update_CompDom.
struct Contrib {  // per-lane particle coordinates feeding the moment sums
  double x, px, y, py, z, pz;
};

// value v (0..43, tmplc order of Output.f90:198-234, then |max| and r^2)
__device__ __forceinline__ double moment_value(const Contrib& c, int v) {
  const double x = c.x, px = c.px, y = c.y, py = c.py, z = c.z, pz = c.pz;
  switch (v) {
    case 0: return x;            case 1: return px;           case 2: return y;
    case 3: return py;           case 4: return z;            case 5: return pz;
    case 6: return x * x;        case 7: return px * px;      case 8: return y * y;
    case 9: return py * py;      case 10: return z * z;       case 11: return pz * pz;
    case 12: return x * px;      case 13: return y * py;      case 14: return z * pz;
    case 15: return x * x * x;   case 16: return x * x * x * x;
    case 17: return px * px * px; case 18: return px * px * px * px;
    case 19: return y * y * y;   case 20: return y * y * y * y;
    case 21: return py * py * py; case 22: return py * py * py * py;
    case 23: return fabs(z * z * z); case 24: return z * z * z * z;
    case 25: return pz * pz * pz; case 26: return pz * pz * pz * pz;
    case 27: return x * px * px; case 28: return x * px * px * px;
    case 29: return x * x * px;  case 30: return x * x * px * px;
    case 31: return x * x * x * px;
    case 32: return y * py * py; case 33: return y * py * py * py;
    case 34: return y * y * py;  case 35: return y * y * py * py;
    case 36: return y * y * y * py;
    case 37: return fabs(x);     case 38: return fabs(px);    case 39: return fabs(y);
    case 40: return fabs(py);    case 41: return fabs(z);     case 42: return fabs(pz);
    case 43: return x * x + y * y;
    default: return 0.0;
  }
}

// Per-warp reduction of the 37 moment sums by a shared-memory transpose:
// every lane writes its sums into its row of a 32 x 37 tile, then lane l
// adds column l over the 32 rows into acc0, and the five columns 32..36 are
// split among all lanes: lane l adds column 32 + l%5 over rows 6*(l/5) ..
// 6*(l/5)+5 into acc1 (the lanes sharing a column cover its 32 rows; they
// are added together once, at the end of the pass, by moment_tail).  Rows
// have an odd length, so the row writes and the column-l reads do not
// conflict.  The seven maxima stay per lane.
#define IMPZ_MSUMS 37
template <int U>
__device__ __forceinline__ void warp_moments(double* tile, const Contrib (&c)[U], int lane,
                                             double& acc0, double& acc1, double (&mx)[7]) {
  double* row = tile + lane * IMPZ_MSUMS;
#pragma unroll
  for (int v = 0; v < IMPZ_MSUMS; v++) {
    double s = 0.0;
#pragma unroll
    for (int u = 0; u < U; u++) s = s + moment_value(c[u], v);
    row[v] = s;
  }
#pragma unroll
  for (int u = 0; u < U; u++)
#pragma unroll
    for (int v = 0; v < 7; v++) mx[v] = fmax(mx[v], moment_value(c[u], 37 + v));
  __syncwarp();
  double s0 = 0.0, s1 = 0.0;
#pragma unroll 8
  for (int r = 0; r < 32; r++) s0 = s0 + tile[r * IMPZ_MSUMS + lane];
  const int c1 = 32 + lane % 5, r1 = 6 * (lane / 5);
#pragma unroll
  for (int j = 0; j < 6; j++)
    if (r1 + j < 32) s1 = s1 + tile[(r1 + j) * IMPZ_MSUMS + c1];
  acc0 = acc0 + s0;
  acc1 = acc1 + s1;
  __syncwarp();
}

// Column 32+m of a warp's sums (m = lane < 5): the acc1 partials of lanes
// m, m+5, m+10, ... added in lane order.
__device__ __forceinline__ double moment_tail(double acc1, int lane) {
  double t = 0.0;
#pragma unroll
  for (int k = 0; k < 7; k++) {
    const int src = 5 * k + lane % 5;
    const double v = __shfl_sync(0xffffffffu, acc1, src & 31);
    if (src < 32) t = t + v;
  }
  return t;
}

// The Lorentz integrator's kick (scatter2_BeamBunch, BeamBunch.f90:
// 2975-3065, the analytic-field branch): the space-charge field exn =
// Ex*gam, eyn = Ey*gam, ezn = Ez of the grid times 1/(4 pi eps0) = c^2 1e-7
// (a default-real literal there), its magnetic part -beta0/c Ey, beta0/c Ex,
// the element's field at the particle, and the implicit momentum update
// iterated twice.  The on-axis Ez0 at the reference time moves gamma0 by
// tau qmcc Ez0 (the host carries that in the step table).
//
// The element's field at (X, Y) [m] and time T of one particle
// (getfld_Quadrupole, Quadrupole.f90:369-402; getfld_Sol, Sol.f90:391-435;
// getfld_ConstFoc, ConstFoc.f90:297-322; getfldpts_DTL, DTL.f90:858-958,
// and the CCDTL, CCL, SC forms; getfld_SolRF, getfld_TWS; getfld_Multipole;
// LzKind), in the reference's expression forms; e = E, b = B.
// scatter2's quadratic weights along one axis of EMfld's x-y grid
// (BeamBunch.f90:2804-2860): node i, i+1 and a third node i2, one-sided at
// the first and the last interval
__device__ __forceinline__ void emfld_weights(int i, double ab, int nint, int& i2, double w[3]) {
  if (i == 1 && ab <= 0.5) {
    i2 = i;
    w[0] = 0.75 - ab * ab;
    w[1] = (0.5 + ab) * (0.5 + ab) / 2;
    w[2] = 0.0;
  } else if (i == nint && ab > 0.5) {
    i2 = i;
    w[0] = (1.5 - ab) * (1.5 - ab) / 2;
    w[1] = 0.75 - (1 - ab) * (1 - ab);
    w[2] = 0.0;
  } else if (ab <= 0.5) {
    i2 = i - 1;
    w[0] = 0.75 - ab * ab;
    w[1] = (0.5 + ab) * (0.5 + ab) / 2;
    w[2] = (0.5 - ab) * (0.5 - ab) / 2;
  } else {
    i2 = i + 2;
    w[0] = (1.5 - ab) * (1.5 - ab) / 2;
    w[1] = 0.75 - (1 - ab) * (1 - ab);
    w[2] = (ab - 0.5) * (ab - 0.5) / 2;
  }
}

__device__ __forceinline__ void lz_field(int kind, const double* __restrict__ c, double X,
                                         double Y, double T, const Consts& k,
                                         const double* __restrict__ data, double& ex,
                                         double& ey, double& ez, double& bx, double& by,
                                         double& bz) {
  ex = 0.0; ey = 0.0; ez = 0.0; bx = 0.0; by = 0.0; bz = 0.0;
  if (kind == LZ_EMFLD) {
    // scatter2, EMfld with discrete x-y-z data (BeamBunch.f90:2794-2880):
    // nine-point quadratic interpolation of the step's complex field plane
    // (data + c[11], twelve doubles per node, x fastest), times escale
    // e^{i(ww T + theta0)}, real part.  Node indices are kept inside the
    // grid (the reference reads outside its arrays there).
    const int nxi = (int)c[9], nyi = (int)c[10];
    int ix = (int)((X - c[3]) * c[5] + 1), iy = (int)((Y - c[6]) * c[8] + 1);
    const double ab = (X - c[3] - (ix - 1) * c[4]) * c[5];
    const double cd = (Y - c[6] - (iy - 1) * c[7]) * c[8];
    int ix2, iy2;
    double wx[3], wy[3];
    emfld_weights(ix, ab, nxi, ix2, wx);
    emfld_weights(iy, cd, nyi, iy2, wy);
    int ii[3] = {ix, ix + 1, ix2}, jj[3] = {iy, iy + 1, iy2};
#pragma unroll
    for (int a = 0; a < 3; a++) {
      ii[a] = min(max(ii[a], 1), nxi + 1);
      jj[a] = min(max(jj[a], 1), nyi + 1);
    }
    double sn, cs;
    sincos(c[1] * T + c[2], &sn, &cs);
    const double tr = c[0] * cs, ti = c[0] * sn;
    const double* q = data + (long long)c[11];
    double f[6];
#pragma unroll
    for (int comp = 0; comp < 6; comp++) {
      double sr = 0.0, si = 0.0;
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
          const double* v = q + 12 * ((ii[a] - 1) + (nxi + 1) * (jj[b] - 1)) + 2 * comp;
          if (a == 0 && b == 0) {
            sr = v[0] * wx[a] * wy[b];
            si = v[1] * wx[a] * wy[b];
          } else {
            sr = sr + v[0] * wx[a] * wy[b];
            si = si + v[1] * wx[a] * wy[b];
          }
        }
      f[comp] = sr * tr - si * ti;
    }
    ex = f[0]; ey = f[1]; ez = f[2]; bx = f[3]; by = f[4]; bz = f[5];
  } else if (kind == LZ_RF) {
    // getfldpts_DTL (DTL.f90:932-956) and its CCDTL, CCL, SC forms
    double sn, cs;
    sincos(c[5] * T + c[6], &sn, &cs);
    const double r2 = X * X + Y * Y;
    const double er = c[2] / 2 + c[4] * r2 / 4;
    const double bt = c[1] / 2 + c[3] * r2 / 4;
    ex = -(X * er * cs);
    ey = -(Y * er * cs);
    ez = (c[1] + c[3] * r2) * cs;
    bx = c[0] * Y + Y / c[7] * bt * sn;
    by = c[0] * X + -(X / c[7] * bt * sn);
  } else if (kind == LZ_SOLRF || kind == LZ_TWS) {
    // getfld_SolRF (SolRF.f90:482-628), getfld_TWS (TWS.f90)
    const double clite = (double)299792458.0f;
    const double tt = T / c[2];
    const double ph = c[0] * tt + c[3];
    double sn, cs;
    sincos(ph, &sn, &cs);
    const double r2 = X * X + Y * Y;
    const double er = c[5] / 2 + c[7] * r2 / 4;
    const double bt = c[4] / 2 + c[6] * r2 / 4;
    ex = 0.0 + -(X * er * cs);
    ey = 0.0 + -(Y * er * cs);
    ez = 0.0 + (c[4] + c[6] * r2) * cs;
    bx = 0.0 + Y * c[1] / clite * bt * sn;
    by = 0.0 + -(X * c[1] / clite * bt * sn);
    if (kind == LZ_TWS) {
      double sn2, cs2;
      sincos(ph + c[12], &sn2, &cs2);
      const double er2 = c[9] / 2 + c[11] * r2 / 4;
      const double bt2 = c[8] / 2 + c[10] * r2 / 4;
      ex = ex + -(X * er2 * cs2);
      ey = ey + -(Y * er2 * cs2);
      ez = ez + (c[8] + c[10] * r2) * cs2;
      bx = bx + Y * c[1] / clite * bt2 * sn2;
      by = by + -(X * c[1] / clite * bt2 * sn2);
    } else {
      bx = bx - c[9] / 2 * X + c[11] * X * r2 / 16;
      by = by - c[9] / 2 * Y + c[11] * Y * r2 / 16;
      bz = bz + c[8] - c[10] * r2 / 4;
    }
  } else if (kind == LZ_MULT) {
    // getfld_Multipole (Multipole.f90:403-452)
    const double g = c[0];
    if (c[1] == 2.0) {
      bx = g * Y * X;
      by = g * (X * X - Y * Y) / 2;
    } else if (c[1] == 3.0) {
      bx = g * (3 * (X * X) * Y - Y * Y * Y) / 6;
      by = g * (X * X * X - 3 * X * (Y * Y)) / 6;
    } else {
      bx = g * (X * X * X * Y - X * (Y * Y * Y)) / 6;
      by = g * ((X * X) * (X * X) - 6 * (X * X) * (Y * Y) + (Y * Y) * (Y * Y)) / 24;
    }
  } else if (kind == LZ_QUAD) {
    bx = c[0] * Y;
    by = c[0] * X;
  } else if (kind == LZ_QUAD_FRG) {
    bx = c[0] * Y - c[2] * (Y * Y * Y + 3 * (X * X) * Y) / 12;
    by = c[0] * X - c[2] * (X * X * X + 3 * X * (Y * Y)) / 12;
    bz = c[1] * X * Y;
  } else if (kind == LZ_SOL) {
    bz = c[1];
  } else if (kind == LZ_SOL_FRG) {
    bx = -(c[0] / 2 * X);
    by = -(c[0] / 2 * Y);
    bz = c[1];
  } else if (kind == LZ_CONSTFOC) {
    ez = c[2] * T * k.Scxl;
    bx = -(c[0] * Y / k.Clight);
    by = c[1] * X / k.Clight;
  }
}

// scatter2's implicit Lorentz update (BeamBunch.f90:3019-3065) of one
// particle in the z frame by the space-charge field (exn, eyn, ezn) [grid
// units] plus the step's element field (lz_*) and scatter2wake's wake at
// the particle (wx, wy, wz; BeamBunch.f90:5885-5887); with no current
// (scatter20, BeamBunch.f90:3478-3531) the space-charge field is zero.
// r7 is the particle's own Pts1(7) (rays(7,n)); qmcc stays the bunch's.
__device__ __forceinline__ void lorentz_kick(Particle& p, double exn, double eyn, double ezn,
                                             double gam, const StepParams* __restrict__ sp,
                                             const Consts& k, double wx, double wy,
                                             double wz, const double* __restrict__ lz_data,
                                             const double r7) {
  const double xl = k.Scxl, Clight = k.Clight;
  const double tau = sp->tau;
  const double tmpscale = Clight * Clight * 1.00000001168609742e-07;
  const double beta0 = sqrt(gam * gam - 1.0) / gam;
  const double qmcc = k.charge / k.mass;
  const double ez0 = sp->lz_ez0;
  const double tmpgamma0 = gam + 0.5 * tau * qmcc * ez0;
  double e1, e2, e3, ext4, ext5, ext6;
  lz_field(sp->lz_kind, sp->lz_c, p.x * xl, p.y * xl, p.ph + sp->lz_tg, k, lz_data, e1, e2, e3,
           ext4, ext5, ext6);
  const double ex = tmpscale * exn + e1 + wx;
  const double ey = tmpscale * eyn + e2 + wy;
  const double ez = tmpscale * ezn + e3 + wz;
  const double bx = -(beta0 / Clight * tmpscale * eyn) + ext4;
  const double by = beta0 / Clight * tmpscale * exn + ext5;
  const double bz = ext6;
  const double tmp12 = -tau * Clight * bz * r7 / 2;
  const double tmp13 = tau * ex * r7 / 2;
  const double tmp23 = tau * ey * r7 / 2;
  const double tmp1 = tmpgamma0 * ex * tau * r7;
  const double tmp2 = Clight * by * tau * r7;
  const double tmp3 = tmpgamma0 * ey * tau * r7;
  const double tmp4 = Clight * bx * tau * r7;
  const double tmp5 = (ez0 * qmcc - ez * r7) * tau;
  double pz = sqrt((gam - p.pt) * (gam - p.pt) - 1.0 - p.px * p.px - p.py * p.py);
  const double p1 = p.px, p2 = p.py, p3 = p.pt;
#pragma unroll
  for (int ii = 1; ii <= 2; ii++) {
    const double a12 = tmp12 / pz, a13 = tmp13 / pz, a23 = tmp23 / pz;
    const double b1 = p1 - a12 * p2 - a13 * p3 + tmp1 / pz - tmp2;
    const double b2 = a12 * p1 + p2 - a23 * p3 + tmp3 / pz + tmp4;
    const double b3 = -(a13 * p1) - a23 * p2 + p3 + tmp5;
    const double det = 1 + a12 * a12 - a13 * a13 - a23 * a23;
    const double s11 = 1 - a23 * a23, s12 = -a12 + a13 * a23, s13 = a12 * a23 - a13;
    const double s21 = a12 + a13 * a23, s22 = 1 - a13 * a13, s23 = -a23 - a13 * a12;
    const double s31 = -(a12 * a23) - a13, s32 = -a23 + a12 * a13, s33 = 1 + a12 * a12;
    p.px = (s11 * b1 + s12 * b2 + s13 * b3) / det;
    p.py = (s21 * b1 + s22 * b2 + s23 * b3) / det;
    p.pt = (s31 * b1 + s32 * b2 + s33 * b3) / det;
    const double tmpgamma00 = gam + tau * qmcc * ez0;
    const double tmpsq2 = (tmpgamma00 - p.pt) * (tmpgamma00 - p.pt) - 1.0 - p.px * p.px -
                          p.py * p.py;
    if (tmpsq2 > 0.0) pz = 0.5 * pz + 0.5 * sqrt(tmpsq2);
  }
}

// The pass of one bunch as block vbx of a grid of vgx blocks: k_advance
// runs it for one bunch (vbx = vbx), k_advance_packed for the bunch
// that owns the block in a launch over many.
// SP: the instantiation for multi-species bunches (the species column, each
// particle's q/m and the per-species counts); without it that code is absent.
template <int BLOCK, bool F32, int U, bool LIGHT, bool SP>
__device__ __forceinline__ void advance_pass(const AdvanceArgs& a, const int vbx, const int vgx) {
  __shared__ double red[BLOCK / 32][IMPZ_RAW_LEN];
  __shared__ double redr[BLOCK / 32][8];
  __shared__ unsigned int s_last;
  __shared__ double fin[8];
  __shared__ MapProgram progs[2];  // post, pre_next
  extern __shared__ __align__(16) double mtile_dyn[];  // [BLOCK/32][32*IMPZ_MSUMS]
  __shared__ Geom sgeom;
  __shared__ int s_spc[IMPZ_MAX_SPECIES];  // particles kept per species (multi-species bunches)
  griddep_wait();  // step state, geometry and field come from earlier kernels
  DevState* st = a.st;
  const int s = a.fixed_step >= 0 ? a.fixed_step : st->step;
  const StepParams* __restrict__ sp = a.steps + s;
  const long long n = st->nlocal;
  static_assert(offsetof(StepParams, pre_next) == sizeof(MapProgram), "program layout");
  stage_programs(progs, sp);
  if (threadIdx.x == 0) sgeom = st->geom;
  const bool species = SP && a.sp_in != nullptr;
  if (SP)
    for (int t = threadIdx.x; t < a.nspecies; t += BLOCK) s_spc[t] = 0;
  __syncthreads();
  // the geometry lives in registers for the whole pass (a volatile shared
  // reference re-read it per particle: 5 % slower)
  const Geom g = sgeom;
  const double xl = a.k.Scxl, xk = a.k.xk;
  const bool kick = a.kick != 0;
  const bool post = a.do_post != 0;
  const bool mom = post && sp->moments;
  const bool pre = a.do_pre != 0;
  const bool rng = pre && sp->range_next;
  const double gam = sp->gam, rad = sp->rad;
  const double gam_n = sp[1].gam, rad_n = sp[1].rad;
  double txy = 0.0, tt = 0.0;
  if (kick) {
    double xycon, tcon;
    kick_consts(a.k, gam, st->current, xycon, tcon);
    txy = sp->tau * xycon;
    tt = sp->tau * tcon;
  }
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const long long G = (long long)nx * ny * nz;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double macc0 = 0.0, macc1 = 0.0;
  double mmax[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};

  double rmn[3] = {1e300, 1e300, 1e300}, rmx[3] = {-1e300, -1e300, -1e300};
  long long nlive = 0, nkept = 0;
  unsigned int err = 0;

  const long long stride = (long long)vgx * BLOCK * U;
  const long long nround = (n + stride - 1) / stride * stride;
  // the next pass's particles are loaded while this pass computes (each
  // thread reads its own slots only; in-place launches write slot i back)
  Particle nxt[U];
  auto fetch = [&](long long ib) {
#pragma unroll
    for (int u = 0; u < U; u++) {
      const long long i = ib + (long long)u * BLOCK;
      if (i < n) {
        nxt[u].x = a.in[0][i]; nxt[u].px = a.in[1][i]; nxt[u].y = a.in[2][i];
        nxt[u].py = a.in[3][i]; nxt[u].ph = a.in[4][i]; nxt[u].pt = a.in[5][i];
      } else {
        nxt[u].x = 0; nxt[u].px = 0; nxt[u].y = 0; nxt[u].py = 0; nxt[u].ph = 0; nxt[u].pt = 0;
      }
    }
  };
#if IMPZ_ADV_PREFETCH
  fetch((long long)vbx * BLOCK * U + threadIdx.x);
#endif
  for (long long i0 = (long long)vbx * BLOCK * U + threadIdx.x; i0 < nround;
       i0 += stride) {
    Particle p[U];
    bool keep[U];
    int key[U];  // deposit cell (a grid holds at most 64 x 64 x 4096 nodes)
    int spi[U];  // species index (0 for a single-species bunch)
#if !IMPZ_ADV_PREFETCH
    fetch(i0);
#endif
#pragma unroll
    for (int u = 0; u < U; u++) {
      const long long i = i0 + (long long)u * BLOCK;
      keep[u] = i < n;
      key[u] = 0;
      p[u] = nxt[u];
      spi[u] = (species && keep[u]) ? (int)a.sp_in[i] : 0;
    }
#if IMPZ_ADV_PREFETCH
    if (i0 + stride < nround) fetch(i0 + stride);
#endif
    Contrib c[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (keep[u] && kick) {
        const TFrame t = a.tframe ? stored_tframe(p[u], gam) : to_tframe(p[u], gam, rad, xl);
        if (t.lost) {
          keep[u] = false;
        } else {
          Cell cd = cic_cell(t.xt, t.yt, t.zt, g);
          key[u] = cell_inside(cd, nx, ny, nz) ? cell_key(cd.ix - 1, cd.jx - 1, cd.kx - 1, nx, ny)
                                                : (int)G;
          // cvbkforth1st (BeamBunch.f90:1681-1699); betai reuses conv1st's
          // tmpbet, the same expression of the same operands
          const double rcp = t.rcp;
#if IMPZ_FASTMATH
          const double rb = rsqrt(t.tmpbet);  // 1/betai
          const double betai = t.tmpbet * rb;
          const double xkg = -xk / gam;
          const double ph1 = t.zt * xkg * rb;
#else
          const double betai = sqrt(t.tmpbet);
          const double ph1 = t.zt * xk / (-(gam * betai));
#endif
          const double x1 = t.xt * xk + p[u].px * ph1 * rcp;
          const double y1 = t.yt * xk + p[u].py * ph1 * rcp;
          const double xg = x1 * xl, yg = y1 * xl;
          const double zg = -(gam * betai * ph1 * xl);
          // scatter1 (BeamBunch.f90:2121-2177); indices clamped into the grid
          Cell cg = cic_cell(xg, yg, zg, g);
          if (!cell_inside(cg, nx, ny, nz)) {
            err |= DERR_OUTSIDE;
            cg.ix = min(max(cg.ix, 1), nx - 1);
            cg.jx = min(max(cg.jx, 1), ny - 1);
            cg.kx = min(max(cg.kx, 1), nz - 1);
          }
          double ex, ey, ez;
          gather_e<F32>(a.efield, cg, nx, ny, ex, ey, ez);
          if (F32) {
            ex = ex * a.efield_scale;
            ey = ey * a.efield_scale;
            ez = ez * a.efield_scale;
          }
          const double exn = ex * gam, eyn = ey * gam, ezn = ez;
          p[u].x = xg * xk;
          p[u].y = yg * xk;
#if IMPZ_FASTMATH
          p[u].ph = zg * xkg * rb;
#else
          p[u].ph = zg * xk / (-(gam * betai));
#endif
          if (!LIGHT && sp->lorentz) {
            // scatter2_BeamBunch (BeamBunch.f90:2766-3065): the same way back
            // to the z frame, then the implicit Lorentz update
            // scatter2wake: the wake's planes kx, kx+1 weighted by the
            // gather cell's ef (BeamBunch.f90:5634-5636)
            double wx = 0.0, wy = 0.0, wz = 0.0;
            if ((sp->csr || sp->wake) && a.wake_raw) {
              const double* w = a.wake_raw + (cg.kx - 1);
              wx = w[0] * cg.ef + w[1] * (1.0 - cg.ef);
              wy = w[nz] * cg.ef + w[nz + 1] * (1.0 - cg.ef);
              wz = w[2 * nz] * cg.ef + w[2 * nz + 1] * (1.0 - cg.ef);
            }
            lorentz_kick(p[u], exn, eyn, ezn, gam, sp, a.k, wx, wy, wz, a.lz_data,
                         species ? __ldg(a.sp_qm + spi[u]) : a.k.qmi);
          } else {
            p[u].px = p[u].px + txy * exn;
            p[u].py = p[u].py + txy * eyn;
            p[u].pt = p[u].pt - tt * ezn;
          }
        }
      }
      // a Lorentz-integrator step without space charge: scatter20's kick by
      // the element's field alone, on the stored coordinates
      // (BeamBunch.f90:3075-3531)
      if (!LIGHT && keep[u] && !kick && post && sp->lorentz)
        lorentz_kick(p[u], 0.0, 0.0, 0.0, gam, sp, a.k, 0.0, 0.0, 0.0, a.lz_data,
                     species ? __ldg(a.sp_qm + spi[u]) : a.k.qmi);
      if (keep[u] && post)
        apply_program<LIGHT>(p[u], progs[0], species ? __ldg(a.sp_qm + spi[u]) : a.k.qmi);
      if (keep[u]) {
        c[u].x = p[u].x; c[u].px = p[u].px; c[u].y = p[u].y;
        c[u].py = p[u].py; c[u].z = p[u].ph; c[u].pz = p[u].pt;
      } else {
        c[u].x = 0; c[u].px = 0; c[u].y = 0; c[u].py = 0; c[u].z = 0; c[u].pz = 0;
      }
    }
    if (mom) warp_moments<U>(mtile_dyn + wid * 32 * IMPZ_MSUMS, c, lane, macc0, macc1, mmax);
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (keep[u]) {
        if (pre)
          apply_program<LIGHT>(p[u], progs[1], species ? __ldg(a.sp_qm + spi[u]) : a.k.qmi);
        if (!finite6(p[u])) err |= DERR_NONFINITE;
        nkept++;
        if (SP && a.sp_cnt) atomicAdd(&s_spc[spi[u]], 1);
        if (rng) {
          const TFrame t = to_tframe(p[u], gam_n, rad_n, xl);
          rmn[0] = fmin(rmn[0], fmin(t.tmpx, t.xt));
          rmx[0] = fmax(rmx[0], fmax(t.tmpx, t.xt));
          rmn[1] = fmin(rmn[1], fmin(t.tmpy, t.yt));
          rmx[1] = fmax(rmx[1], fmax(t.tmpy, t.yt));
          rmn[2] = fmin(rmn[2], t.zt);
          rmx[2] = fmax(rmx[2], t.zt);
          nlive += t.lost ? 0 : 1;
          if (a.tframe) {  // stored as conv1st leaves Pts1 (stored_tframe)
            p[u].x = t.xt;
            p[u].y = t.yt;
            p[u].ph = t.lost ? lost_mark() : t.zt;
          }
        }
      }
      // destination slot
      long long dst = i0 + (long long)u * BLOCK;
      if (kick) {
        const unsigned active = __ballot_sync(0xffffffffu, keep[u]);
        if (keep[u]) {
          const unsigned grp = __match_any_sync(active, key[u]);
          const int leader = __ffs(grp) - 1;
          const int rank = __popc(grp & ((1u << lane) - 1u));
          int base = 0;
          if (lane == leader) base = atomicAdd(a.cursor + key[u], __popc(grp));
          base = __shfl_sync(grp, base, leader);
          dst = (long long)base + rank + a.bsum[key[u] >> IMPZ_SCAN_LOG];
          if (dst < 0 || dst >= a.cap) {  // cannot happen when deposit and pass agree
            err |= DERR_SLOT;
            keep[u] = false;
          }
        }
      }
      if (keep[u]) {
        a.out[0][dst] = p[u].x; a.out[1][dst] = p[u].px; a.out[2][dst] = p[u].y;
        a.out[3][dst] = p[u].py; a.out[4][dst] = p[u].ph; a.out[5][dst] = p[u].pt;
        if (a.id_out) a.id_out[dst] = a.id_in[i0 + (long long)u * BLOCK];
        if (species && a.sp_out) a.sp_out[dst] = (unsigned char)spi[u];
      }
    }
  }

  // ---- block reductions
  if (mom) {
    red[wid][lane] = macc0;
    const double tail = moment_tail(macc1, lane);
    if (lane < IMPZ_MSUMS - 32) red[wid][32 + lane] = tail;
#pragma unroll
    for (int v = 0; v < 7; v++) {
      const double m = warp_max(mmax[v]);
      if (lane == 0) red[wid][IMPZ_MSUMS + v] = m;
    }
  }
  double cnt_l = (double)warp_sum_ll(nlive), cnt_k = (double)warp_sum_ll(nkept);
  double r[6];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    r[2 * d] = warp_min(rmn[d]);
    r[2 * d + 1] = warp_max(rmx[d]);
  }
  err = __reduce_or_sync(0xffffffffu, err);
  if (lane == 0) {
#pragma unroll
    for (int d = 0; d < 6; d++) redr[wid][d] = r[d];
    redr[wid][6] = cnt_l;
    redr[wid][7] = cnt_k;
    if (err) atomicOr(&st->err, err);
  }
  __syncthreads();
  // chgupdate_BeamBunch's count of each charge state (BeamBunch.f90:688-728)
  // after this step's conv1st: integer sums, so the block order is immaterial
  if (SP && a.sp_cnt) {
    int* cnt = a.sp_cnt + (size_t)(a.fixed_step >= 0 ? a.mom_index : s) * a.nspecies;
    for (int t = threadIdx.x; t < a.nspecies; t += BLOCK)
      if (s_spc[t]) atomicAdd(cnt + t, s_spc[t]);
  }
  const int nw = BLOCK / 32;
  if (mom && threadIdx.x < IMPZ_RAW_LEN) {
    const int v = threadIdx.x;
    double x = red[0][v];
    for (int w = 1; w < nw; w++) x = v < 37 ? x + red[w][v] : fmax(x, red[w][v]);
    a.mom_part[(size_t)vbx * IMPZ_RAW_LEN + v] = x;
  }
  if (threadIdx.x < 8) {
    const int v = threadIdx.x;
    double x = redr[0][v];
    for (int w = 1; w < nw; w++) {
      double y = redr[w][v];
      x = (v >= 6) ? x + y : ((v & 1) ? fmax(x, y) : fmin(x, y));
    }
    a.rng_part[(size_t)vbx * 8 + v] = x;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&st->done_range, 1u) == vgx - 1) ? 1u : 0u;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // ---- last block: fixed-order reduction over blocks, then bookkeeping.
  // Warp w reduces blocks [w*nb/nw, (w+1)*nb/nw) of every value (lane l:
  // values l and l+32; 0..43 moments, 44..51 range), then thread v combines
  // the warps' partials in warp order: a fixed order, and the loads of one
  // lane are independent, so they overlap instead of chaining.
  const int nb = vgx;
  const int row = a.fixed_step >= 0 ? a.mom_index : s;
  const int b0 = wid * nb / nw, b1 = (wid + 1) * nb / nw;
  for (int v = lane; v < IMPZ_RAW_LEN + 8; v += 32) {
    const bool isrng = v >= IMPZ_RAW_LEN;
    const int r = v - IMPZ_RAW_LEN;  // range value 0..7
    if (!isrng && !mom) continue;
    // identities: sums 0, maxima of |.| 0, range min +1e300 / max -1e300
    double x = (isrng && r < 6) ? ((r & 1) ? -1e300 : 1e300) : 0.0;
#pragma unroll 4
    for (int b = b0; b < b1; b++) {
      const double y = isrng ? __ldcg(a.rng_part + (size_t)b * 8 + r)
                             : __ldcg(a.mom_part + (size_t)b * IMPZ_RAW_LEN + v);
      if (isrng) x = (r >= 6) ? x + y : ((r & 1) ? fmax(x, y) : fmin(x, y));
      else x = v < IMPZ_MSUMS ? x + y : fmax(x, y);
    }
    if (isrng) redr[wid][r] = x;
    else red[wid][v] = x;
  }
  __syncthreads();
  if (mom && threadIdx.x < IMPZ_RAW_LEN) {
    const int v = threadIdx.x;
    double x = red[0][v];
    for (int w = 1; w < nw; w++) x = v < IMPZ_MSUMS ? x + red[w][v] : fmax(x, red[w][v]);
    a.mom_out[(size_t)row * IMPZ_MOMREC + v] = x;
  }
  if (threadIdx.x < 8) {
    const int v = threadIdx.x;
    double x = redr[0][v];
    for (int w = 1; w < nw; w++) {
      const double y = redr[w][v];
      x = (v >= 6) ? x + y : ((v & 1) ? fmax(x, y) : fmin(x, y));
    }
    fin[v] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const long long kept = (long long)fin[7];
    if (mom) {
      double* m = a.mom_out + (size_t)row * IMPZ_MOMREC;
      m[44] = (double)st->npt;
      m[45] = (double)kept;
      m[46] = st->current;
      m[47] = 0.0;
    }
    st->nlocal = kept;
    if (rng) {
      Geom ng;
      for (int d = 0; d < 6; d++) ng.ptrange[d] = fin[d];
      compdom(ng, nx, ny, nz);
      st->geom = ng;
      const long long nptot = (long long)fin[6];
      // conv1st: Current = Current*nptot/Npt; Npt = nptot
      st->current = st->current * (double)nptot / (double)st->npt;
      st->npt = nptot;
      st->nlive = nptot;
    }
    if (a.fixed_step < 0) st->step = s + 1;
    if (kick) st->parity ^= 1;
    st->done_range = 0;
  }
}

template <int BLOCK, bool F32, int U, bool LIGHT, bool SP>
__global__ void __launch_bounds__(BLOCK, IMPZ_ADV_MINB) k_advance(AdvanceArgs a) {
  advance_pass<BLOCK, F32, U, LIGHT, SP>(a, blockIdx.x, gridDim.x);
}

// The member of a packed launch that owns block `blk`: blocks
// [offs[m], offs[m+1]) belong to member m (binary search, offs[0] = 0).
__device__ __forceinline__ int packed_member(const int* __restrict__ offs, int nmem, int blk) {
  int lo = 0, hi = nmem - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(offs + mid) <= blk) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Copies a launch-argument struct of `bytes` (a multiple of 8) to shared
// memory (whole block).
__device__ __forceinline__ void copy_args(void* dst, const void* src, int bytes) {
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(dst);
  for (int e = threadIdx.x; e < bytes / 8; e += blockDim.x) d[e] = __ldg(s + e);
}

// Every member's pass in one launch: a packed work list of (bunch, block)
// items, each bunch keeping its own block count and last-block reduction.
template <int BLOCK, bool F32, int U, bool LIGHT, bool SP>
__global__ void __launch_bounds__(BLOCK, IMPZ_ADV_MINB)
    k_advance_packed(const AdvanceArgs* __restrict__ args, const int* __restrict__ offs,
                     int nmem) {
  __shared__ __align__(16) AdvanceArgs sa;
  static_assert(sizeof(AdvanceArgs) % 8 == 0, "argument copy in 8-byte words");
  const int m = packed_member(offs, nmem, blockIdx.x);
  copy_args(&sa, args + m, (int)sizeof(AdvanceArgs));
  __syncthreads();
  advance_pass<BLOCK, F32, U, LIGHT, SP>(sa, blockIdx.x - __ldg(offs + m),
                                     __ldg(offs + m + 1) - __ldg(offs + m));
}

// ---------------------------------------------------------------------
// Charge deposit.  Each block takes chunks of BLOCK*U consecutive particles.
// Particles are kept sorted by the previous step's deposit cell, so after the
// grid is refitted a chunk still covers a small box of cells, give or take
// one cell per axis.  Its charge is accumulated in a shared-memory tile over
// that box (the chunk's min..max+1 in each of x, y, z) and every touched node
// is flushed with one 64-bit global reduction; chunks whose box exceeds the
// tile (the sparse tails) reduce straight into the grid.  Sorted particles
// put many lanes of a warp on the same cell, where shared atomics serialize,
// so the tile holds R copies of the box (R = tile / box, at most 32) and
// lane l adds to copy l % R; the copies sit 1 mod 32 words apart so the same
// node of different copies falls in different banks, and the flush adds the
// copies.  Small boxes (the dense core) thus get many copies, large boxes
// (sparse regions, few lanes per cell) few.  Each tile word keeps a node's
// fixed-point sum as two 32-bit halves (the low 20 bits and the rest) so
// that native 32-bit shared atomics suffice: a chunk of at most 2048
// particles cannot overflow either half.  With quanta of at most 2^21 (the
// FP32-convolution form) one word holds a chunk's sum and the high half is
// not used.  Accumulation is in int64 fixed
// point (2^-fixbits of a unit macro-particle charge), so the result does not
// depend on the order of the additions; the corner with the largest weight
// takes 2^fixbits minus the other seven (never negative), so every live
// particle deposits exactly one unit.
#ifndef IMPZ_DEP_RMAX
#define IMPZ_DEP_RMAX 32
#endif
#define IMPZ_DEP_LOBITS 20
#define IMPZ_DEP_FIXBITS_1WORD 21
template <int BLOCK, int U, bool SP>
__device__ __forceinline__ void deposit_pass(const DepositArgs& a, const int vbx, const int vgx) {
  static_assert(BLOCK * U <= 1024, "one-word tile sums sized for chunks of at most 1024");
  extern __shared__ __align__(16) unsigned int tsm[];
  unsigned int* tlo = tsm;                       // [IMPZ_DEP_TILE]
  unsigned int* thi = tsm + IMPZ_DEP_TILE;       // [IMPZ_DEP_TILE]
  unsigned int* tcnt = tsm + 2 * IMPZ_DEP_TILE;  // [IMPZ_DEP_TILE]
  __shared__ int s_box[6];
  __shared__ Geom sg;
  griddep_wait();  // the geometry comes from the previous push
  const DevState* st = a.st;
  const int s = a.fixed_step >= 0 ? a.fixed_step : st->step;
  const double gam = a.steps[s].gam, rad = a.steps[s].rad;
  const long long n = st->nlocal;
  if (threadIdx.x == 0) sg = st->geom;
  for (int e = threadIdx.x; e < IMPZ_DEP_TILE; e += BLOCK) {
    tlo[e] = 0u;
    thi[e] = 0u;
    tcnt[e] = 0u;
  }
  __syncthreads();
  const Geom g = sg;  // in registers: a volatile shared reference measured 6 % slower
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const long long P = (long long)nx * ny;
  const long long G = P * nz;
  const double scale = ldexp(1.0, a.fixbits);
  const unsigned long long unit = 1ull << a.fixbits;
  // round-to-nearest-even of w*2^f (exact below 2^51) by the 1.5*2^52 shift
  const double magic = 6755399441055744.0;
  const long long magic_bits = 0x4338000000000000ll;
  const unsigned lomask = (1u << IMPZ_DEP_LOBITS) - 1u;
  // quanta of at most 2^21: a chunk's sum at one node stays below 2^31 in
  // a single word (species of either sign take the two signed halves)
  const bool species = SP && a.sp_in != nullptr;
  const bool split = a.fixbits > IMPZ_DEP_FIXBITS_1WORD || species;
  const long long chunk = (long long)BLOCK * U;
  const int lane = threadIdx.x & 31;
  for (long long c0 = (long long)vbx * chunk; c0 < n; c0 += (long long)vgx * chunk) {
    int cell[U];
    unsigned pk[U];  // x | y << 10 | z << 20 (nx, ny <= 64, nz <= 4096)
    double wab[U], wcd[U], wef[U];
    int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {-1, -1, -1};
#pragma unroll
    for (int u = 0; u < U; u++) {
      const long long i = c0 + (long long)u * BLOCK + threadIdx.x;
      cell[u] = -1;
      pk[u] = 0u;
      wab[u] = wcd[u] = wef[u] = 0.0;
      if (i < n) {
        double xt, yt, zt;
        bool lost;
        if (a.tframe) {  // stored in conv1st's frame: three columns suffice
          xt = a.in[0][i];
          yt = a.in[2][i];
          zt = a.in[4][i];
          lost = isnan(zt);
        } else {
          Particle p;
          p.x = a.in[0][i]; p.px = a.in[1][i]; p.y = a.in[2][i];
          p.py = a.in[3][i]; p.ph = a.in[4][i]; p.pt = a.in[5][i];
          const TFrame t = to_tframe(p, gam, rad, a.xl);
          xt = t.xt; yt = t.yt; zt = t.zt;
          lost = t.lost;
        }
        if (!lost) {
          Cell c = cic_cell(xt, yt, zt, g);
          if (cell_inside(c, nx, ny, nz)) {
            cell[u] = (int)lin_cell(c, nx, ny);
            pk[u] = (unsigned)(c.ix - 1) | ((unsigned)(c.jx - 1) << 10) |
                    ((unsigned)(c.kx - 1) << 20);
            wab[u] = c.ab; wcd[u] = c.cd; wef[u] = c.ef;
            mn[0] = min(mn[0], c.ix - 1); mx[0] = max(mx[0], c.ix - 1);
            mn[1] = min(mn[1], c.jx - 1); mx[1] = max(mx[1], c.jx - 1);
            mn[2] = min(mn[2], c.kx - 1); mx[2] = max(mx[2], c.kx - 1);
          } else {
            atomicAdd(a.counts + G, 1);  // live but outside: keeps its sort slot
          }
        }
      }
    }
    if (threadIdx.x < 3) { s_box[threadIdx.x] = INT_MAX; s_box[3 + threadIdx.x] = -1; }
    __syncthreads();
#pragma unroll
    for (int d = 0; d < 3; d++) {
      mn[d] = __reduce_min_sync(0xffffffffu, mn[d]);
      mx[d] = __reduce_max_sync(0xffffffffu, mx[d]);
    }
    if (lane == 0 && mx[0] >= 0) {
#pragma unroll
      for (int d = 0; d < 3; d++) {
        atomicMin(&s_box[d], mn[d]);
        atomicMax(&s_box[3 + d], mx[d]);
      }
    }
    __syncthreads();
    // the box of nodes: lower cell corners min..max, plus one
    const bool any = s_box[3] >= 0;
    const int x0 = any ? s_box[0] : 0, y0 = any ? s_box[1] : 0, z0 = any ? s_box[2] : 0;
    const int bx = any ? s_box[3] - x0 + 2 : 0, by = any ? s_box[4] - y0 + 2 : 0;
    const int bz = any ? s_box[5] - z0 + 2 : 0;
    const long long V = (long long)bx * by * bz;
    const int S = (int)(((V + 31) & ~31ll) + 1);  // copy stride, 1 mod 32
    const bool tiled = any && V + 32 <= IMPZ_DEP_TILE;
    const int R = tiled ? min(IMPZ_DEP_RMAX, IMPZ_DEP_TILE / S) : 1;
    const int mycopy = (lane % R) * S;
    const int bxy = bx * by;
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (cell[u] < 0) continue;
      const double ab = wab[u], cd = wcd[u], ef = wef[u];
      // weights in the order of deposit_BeamBunch (BeamBunch.f90:3749-3763)
      const double w8[8] = {ab * cd * ef,
                            ab * (1.0 - cd) * ef,
                            ab * (1.0 - cd) * (1.0 - ef),
                            ab * cd * (1.0 - ef),
                            (1.0 - ab) * cd * (1.0 - ef),
                            (1.0 - ab) * (1.0 - cd) * (1.0 - ef),
                            (1.0 - ab) * (1.0 - cd) * ef,
                            (1.0 - ab) * cd * ef};
      int big = 0;
      double wbig = w8[0];
#pragma unroll
      for (int k = 1; k < 8; k++)
        if (w8[k] > wbig) { wbig = w8[k]; big = k; }
      // a particle of relative weight ws deposits round(ws 2^f) quanta (one
      // unit, 2^f, for the bunch's own species); two's complement for
      // species of the other sign
      double pscale = scale;
      unsigned long long punit = unit;
      if (species) {  // the particle's charge weight relative to the bunch's
        const double ws = __ldg(a.sp_w + a.sp_in[c0 + (long long)u * BLOCK + threadIdx.x]);
        pscale = __dmul_rn(ws, scale);
        punit = (unsigned long long)(__double_as_longlong(__dadd_rn(pscale, magic)) - magic_bits);
      }
      unsigned long long qv[8];
      unsigned long long sum7 = 0;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const double sh = __dadd_rn(__dmul_rn(w8[k], pscale), magic);
        qv[k] = (k == big) ? 0ull : (unsigned long long)(__double_as_longlong(sh) - magic_bits);
        sum7 += qv[k];
      }
#pragma unroll
      for (int k = 0; k < 8; k++)
        if (k == big) qv[k] = punit - sum7;
      if (!tiled) {
        const long long c = cell[u];
        const long long node[8] = {c, c + nx, c + nx + P, c + P, c + 1 + P, c + 1 + nx + P,
                                   c + 1 + nx, c + 1};
#pragma unroll
        for (int k = 0; k < 8; k++) atomicAdd(a.rho + node[k], qv[k]);
        atomicAdd(a.counts + cell_key((int)(pk[u] & 1023u), (int)((pk[u] >> 10) & 1023u),
                                      (int)(pk[u] >> 20), nx, ny), 1);
      } else {
        const int t = mycopy + ((int)(pk[u] & 1023u) - x0) +
                      bx * (((int)((pk[u] >> 10) & 1023u) - y0) + by * ((int)(pk[u] >> 20) - z0));
        const int node[8] = {t, t + bx, t + bx + bxy, t + bxy, t + 1 + bxy, t + 1 + bx + bxy,
                             t + 1 + bx, t + 1};
        if (split) {
#pragma unroll
          for (int k = 0; k < 8; k++) {
            atomicAdd(tlo + node[k], (unsigned)(qv[k] & lomask));
            atomicAdd(thi + node[k], (unsigned)((long long)qv[k] >> IMPZ_DEP_LOBITS));
          }
        } else {
#pragma unroll
          for (int k = 0; k < 8; k++) atomicAdd(tlo + node[k], (unsigned)qv[k]);
        }
        atomicAdd(tcnt + t, 1u);
      }
    }
    __syncthreads();
    if (tiled) {
      // add the copies, flush the box and clear it for the next chunk
      for (int e = threadIdx.x; e < (int)V; e += BLOCK) {
        unsigned long long q = 0ull;
        unsigned int k = 0u;
        for (int r = 0, o = e; r < R; r++, o += S) {
          const unsigned lo = tlo[o], hi = split ? thi[o] : 0u, c = tcnt[o];
          if (lo | hi | c) {
            // the high half is signed (a negative quantum's arithmetic shift)
            q += ((unsigned long long)(long long)(int)hi << IMPZ_DEP_LOBITS) +
                 (unsigned long long)lo;
            k += c;
            tlo[o] = 0u;
            if (split) thi[o] = 0u;
            tcnt[o] = 0u;
          }
        }
        if (q | k) {
          const int lz = e / bxy, r = e - lz * bxy;
          const int ly = r / bx, lx = r - ly * bx;
          const long long gi = (long long)(x0 + lx) + nx * ((long long)(y0 + ly) +
                                                           (long long)ny * (z0 + lz));
          if (q) atomicAdd(a.rho + gi, q);
          if (k) atomicAdd(a.counts + cell_key(x0 + lx, y0 + ly, z0 + lz, nx, ny), (int)k);
        }
      }
    }
    __syncthreads();
  }
}

template <int BLOCK, int U, bool SP>
__global__ void __launch_bounds__(BLOCK, IMPZ_DEP_MINB) k_deposit(DepositArgs a) {
  deposit_pass<BLOCK, U, SP>(a, blockIdx.x, gridDim.x);
}

template <int BLOCK, int U, bool SP>
__global__ void __launch_bounds__(BLOCK, IMPZ_DEP_MINB)
    k_deposit_packed(const DepositArgs* __restrict__ args, const int* __restrict__ offs,
                     int nmem) {
  __shared__ __align__(16) DepositArgs sa;
  static_assert(sizeof(DepositArgs) % 8 == 0, "argument copy in 8-byte words");
  const int m = packed_member(offs, nmem, blockIdx.x);
  copy_args(&sa, args + m, (int)sizeof(DepositArgs));
  __syncthreads();
  deposit_pass<BLOCK, U, SP>(sa, blockIdx.x - __ldg(offs + m), __ldg(offs + m + 1) - __ldg(offs + m));
}

// chgupdate_BeamBunch (BeamBunch.f90:688-728) on the per-step surface: the
// particles of each species that the latest conv1st kept.  test_loss = 1
// between impz_sc_prepare and the kick (conv1st has run, its losses are
// not yet removed: the deposit's loss test of the step decides), 0 when
// every stored particle is live.  counts[nspecies] are added to.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_species_count(DepositArgs a, int test_loss,
                                                         int nspecies, int* counts) {
  __shared__ int hist[IMPZ_MAX_SPECIES];
  for (int t = threadIdx.x; t < nspecies; t += BLOCK) hist[t] = 0;
  __syncthreads();
  const DevState* st = a.st;
  const int s = a.fixed_step >= 0 ? a.fixed_step : st->step;
  const double gam = a.steps[s].gam, rad = a.steps[s].rad;
  const long long n = st->nlocal;
  for (long long i = (long long)blockIdx.x * BLOCK + threadIdx.x; i < n;
       i += (long long)gridDim.x * BLOCK) {
    bool lost = false;
    if (test_loss) {
      if (a.tframe) {
        lost = isnan(a.in[4][i]);
      } else {
        Particle p;
        p.x = a.in[0][i]; p.px = a.in[1][i]; p.y = a.in[2][i];
        p.py = a.in[3][i]; p.ph = a.in[4][i]; p.pt = a.in[5][i];
        lost = to_tframe(p, gam, rad, a.xl).lost;
      }
    }
    if (!lost) atomicAdd(&hist[a.sp_in ? (int)a.sp_in[i] : 0], 1);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nspecies; t += BLOCK)
    if (hist[t]) atomicAdd(counts + t, hist[t]);
}

// Exclusive scan over the block of one value per thread; *total gets the
// block's sum.  wsum: BLOCK/32 ints of shared memory.
template <int BLOCK>
__device__ __forceinline__ int block_exclusive_scan(int x, int* wsum, int* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  __syncthreads();  // wsum may still be read by a previous call
  if (lane == 31) wsum[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    const int w = lane < BLOCK / 32 ? wsum[lane] : 0;
    int wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < BLOCK / 32) wsum[lane] = wi - w;  // exclusive warp offsets
    if (lane == BLOCK / 32 - 1) wsum[BLOCK / 32] = wi;
  }
  __syncthreads();
  *total = wsum[BLOCK / 32];
  return wsum[wid] + incl - x;
}

// Exclusive scan of counts[0..total) into per-block local offsets (cursor)
// and per-block totals (bsum), clearing counts for the next step; the last
// block to finish turns bsum into exclusive block offsets.  Each thread
// takes four consecutive cells (one 16-byte load and store).
template <int BLOCK>
__device__ __forceinline__ void scan_pass(int* counts, int* cursor, int* bsum, long long total,
                                          DevState* st, const int vbx, const int vgx) {
  // each thread owns CPT consecutive cells (CPT/4 16-byte loads and stores)
  constexpr int CPT = (1 << IMPZ_SCAN_LOG) / BLOCK;
  static_assert(CPT % 4 == 0 && CPT * BLOCK == (1 << IMPZ_SCAN_LOG), "cells per thread");
  __shared__ int wsum[BLOCK / 32 + 1];
  __shared__ unsigned int s_last;
  const long long i0 = ((long long)vbx << IMPZ_SCAN_LOG) + (long long)CPT * threadIdx.x;
  int v[CPT];
  const bool full = i0 + CPT - 1 < total;
  if (full) {
#pragma unroll
    for (int q = 0; q < CPT / 4; q++) {
      const int4 c = *reinterpret_cast<const int4*>(counts + i0 + 4 * q);
      v[4 * q] = c.x; v[4 * q + 1] = c.y; v[4 * q + 2] = c.z; v[4 * q + 3] = c.w;
    }
#pragma unroll
    for (int q = 0; q < CPT / 4; q++)
      *reinterpret_cast<int4*>(counts + i0 + 4 * q) = make_int4(0, 0, 0, 0);
  } else {
#pragma unroll
    for (int j = 0; j < CPT; j++) {
      v[j] = (i0 + j < total) ? counts[i0 + j] : 0;
      if (i0 + j < total) counts[i0 + j] = 0;
    }
  }
  int mine = 0;
#pragma unroll
  for (int j = 0; j < CPT; j++) mine += v[j];
  int btotal = 0;
  int run = block_exclusive_scan<BLOCK>(mine, wsum, &btotal);
#pragma unroll
  for (int j = 0; j < CPT; j++) {
    const int x = v[j];
    v[j] = run;  // the exclusive offset of cell j within the block
    run += x;
  }
  if (full) {
#pragma unroll
    for (int q = 0; q < CPT / 4; q++)
      *reinterpret_cast<int4*>(cursor + i0 + 4 * q) =
          make_int4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  } else {
#pragma unroll
    for (int j = 0; j < CPT; j++)
      if (i0 + j < total) cursor[i0 + j] = v[j];
  }
  // the last block reads only the block totals, so only their writer
  // fences (the cursors and the cleared counts reach the next kernels at the
  // launch boundary); a fence in every thread was the kernel's third stall
  // reason under ncu
  if (threadIdx.x == 0) {
    bsum[vbx] = btotal;
    __threadfence();
    s_last = (atomicAdd(&st->done_scan, 1u) == vgx - 1) ? 1u : 0u;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // block totals -> exclusive block offsets, BLOCK at a time with a carry
  const int nb = (int)vgx;
  int carry = 0;
  for (int k0 = 0; k0 < nb; k0 += BLOCK) {
    const int k = k0 + threadIdx.x;
    const int t = k < nb ? __ldcg(bsum + k) : 0;
    int sum = 0;
    const int ex = block_exclusive_scan<BLOCK>(t, wsum, &sum);
    if (k < nb) bsum[k] = carry + ex;
    carry += sum;
  }
  if (threadIdx.x == 0) st->done_scan = 0;
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_scan(int* counts, int* cursor, int* bsum,
                                                long long total, DevState* st) {
  scan_pass<BLOCK>(counts, cursor, bsum, total, st, blockIdx.x, gridDim.x);
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_scan_packed(const ScanArgs* __restrict__ args,
                                                       const int* __restrict__ offs, int nmem) {
  const int m = packed_member(offs, nmem, blockIdx.x);
  const ScanArgs a = args[m];
  scan_pass<BLOCK>(a.counts, a.cursor, a.bsum, a.total, a.st, blockIdx.x - __ldg(offs + m),
                   __ldg(offs + m + 1) - __ldg(offs + m));
}

// ---------------------------------------------------------------------
// Read-in wakefield, step part 1: the line density on the z grid
// (AccSimulator.f90:1279-1296).  Every live particle adds ab and 1-ab to
// planes iizz and iizz+1, with the reference's division by hzwake, and with
// the transverse wake x*ab, x*(1-ab) and the same in y.  The sums are int64
// fixed point: the density in units of 2^-fixbits, the moments in units of
// 2^-fixbits of the smallest power of two above the grid's largest |x|
// (|y|), so they do not depend on the order of the additions.  Sorted
// particles put a warp mostly on one plane: such a warp adds each sum with
// one global atomic, any other warp lane by lane.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_wake_line(WakeArgs a) {
  const DevState* st = a.st;
  const int s = a.fixed_step >= 0 ? a.fixed_step : st->step;
  const StepParams& sp = a.steps[s];
  if (!sp.csr && !sp.wake) return;  // no wake acts in this step
  // the x/y moments feed the transverse wakes: the analytic one always, the
  // read-in one unless the table's transverse columns are off; CSR has none
  const bool tr = !sp.csr && (sp.wake == 2 || (sp.wake == 1 && a.transverse));
  const double gam = a.steps[s].gam, rad = a.steps[s].rad;
  const long long n = st->nlocal;
  const int nz = a.nz;
  const double zmin = st->geom.range[4];
  const double hzw = (st->geom.range[5] - zmin) / (nz - 1);
  const double sc = ldexp(1.0, a.fixbits);
  int ex, ey;
  frexp(fmax(fabs(st->geom.range[0]), fabs(st->geom.range[1])), &ex);
  frexp(fmax(fabs(st->geom.range[2]), fabs(st->geom.range[3])), &ey);
  const double sx = ldexp(1.0, a.fixbits - ex), sy = ldexp(1.0, a.fixbits - ey);
  const int nq = tr ? 6 : 2;
  const int lane = threadIdx.x & 31;
  for (long long base = (long long)blockIdx.x * BLOCK + (threadIdx.x & ~31); base < n;
       base += (long long)gridDim.x * BLOCK) {
    const long long i = base + lane;
    int kz = -1;
    long long q[6] = {0, 0, 0, 0, 0, 0};
    if (i < n) {
      Particle p;
      p.x = a.in[0][i]; p.px = a.in[1][i]; p.y = a.in[2][i];
      p.py = a.in[3][i]; p.ph = a.in[4][i]; p.pt = a.in[5][i];
      const TFrame t = a.tframe ? stored_tframe(p, gam) : to_tframe(p, gam, rad, a.xl);
      if (!t.lost) {
        const int iizz = (int)((t.zt - zmin) / hzw + 1);
        const double ab = ((zmin - t.zt) + iizz * hzw) / hzw;
        if (iizz >= 1 && iizz < nz) {
          kz = iizz - 1;
          q[0] = llrint(ab * sc);
          q[1] = llrint((1.0 - ab) * sc);
          if (tr) {
            q[2] = llrint(t.xt * ab * sx);
            q[3] = llrint(t.xt * (1.0 - ab) * sx);
            q[4] = llrint(t.yt * ab * sy);
            q[5] = llrint(t.yt * (1.0 - ab) * sy);
          }
        }
      }
    }
    const int kmin = __reduce_min_sync(0xffffffffu, kz < 0 ? INT_MAX : kz);
    const int kmax = __reduce_max_sync(0xffffffffu, kz);
    if (kmax < 0) continue;
    if (kmin == kmax) {
      for (int c = 0; c < nq; c++) {
        long long v = q[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0)
          atomicAdd(a.line + (long long)(c >> 1) * nz + kmin + (c & 1), (unsigned long long)v);
      }
    } else if (kz >= 0) {
      for (int c = 0; c < nq; c++)
        atomicAdd(a.line + (long long)(c >> 1) * nz + kz + (c & 1), (unsigned long long)q[c]);
    }
  }
}

// greenwake of wakefieldread_FieldQuant (Field.f90:818-830): the table at
// zz = j*hz with the reference's weight ab = iwk*hwk - zwk (not divided by
// hwk); rows past the table read zero, as the reference's zero-filled module
// arrays do.
__device__ __forceinline__ double wake_green(const double* e, int ntab, double hwk, int j,
                                             double hz) {
  const double zz = j * hz;
  const double zwk = zz - 0.0;
  const int iwk = (int)(zwk / hwk + 1);
  const double ab = iwk * hwk - zwk;
  const double e0 = (iwk >= 1 && iwk <= ntab) ? e[iwk - 1] : 0.0;
  const double e1 = (iwk >= 0 && iwk < ntab) ? e[iwk] : 0.0;  // row iwk + 1
  return e0 * ab + e1 * (1.0 - ab);
}

// 1D CSR wake with integrated Green functions (csrwakeTrIGF_FieldQuant,
// Field.f90:1003-1303): the field at node i of the line density rho on the
// lab-frame grid ptmin + (i-1) hx, for a bend of radius r0 and length
// blength.  Sources within the entrance transient use case A, the steady
// state case B, and past the bend exit cases C and D; case D's retarded
// angle solves a quartic by Newton-Raphson with a bisection safeguard in a
// bracket (the published "rtsafe" method), with the reference's handling
// of the bracket ends and its 100-step limit.  One thread per node.
struct CsrKernel {
  double r0, gam, xk2, g3, epstol;
  __device__ double caseA(double phih, double ssh) const {
    const double p2 = phih * phih, p3 = p2 * phih, p4 = p3 * phih;
    const double bb = 2 * phih + p3 / 3 - 2 * ssh;
    const double cc = p2 + p4 / 12 - 2 * ssh * phih;
    const double yh = (-bb + sqrt(bb * bb - 4 * cc)) / 2;
    const double phpy = phih + yh;
    return xk2 * (-(2 * phpy + p3) / (phpy * phpy + p4 / 4) + 1.0 / ssh);
  }
  __device__ double caseB(double ssh) const {
    const double aa = sqrt(64.0 + 144.0 * (ssh * ssh));
    const double uuh = pow(aa + 12 * ssh, 1.0 / 3.0) - pow(aa - 12 * ssh, 1.0 / 3.0);
    const double u2 = uuh * uuh;
    return xk2 * (-4 * uuh * (u2 + 8) / ((u2 + 4.0) * (u2 + 12.0)));
  }
  __device__ double caseC(double phimh, double xxbarh, double ssh) const {
    const double p2 = phimh * phimh, p3 = p2 * phimh;
    const double bb = 2 * (phimh + xxbarh) - 2 * ssh + p3 / 3 + p2 * xxbarh;
    const double cc = (phimh + xxbarh) * (phimh + xxbarh) +
                      p2 * (p2 + 4 * phimh * xxbarh) / 12 - 2 * ssh * (phimh + xxbarh);
    const double yh = (-bb + sqrt(bb * bb - 4 * cc)) / 2;
    const double pa = phimh + xxbarh + yh;
    const double pb = phimh * xxbarh + phimh * phimh / 2.0;
    return xk2 * (-2.0 * (pa + phimh * pb) / (pa * pa + pb * pb) + 1.0 / ssh);
  }
  __device__ static void quartic(double psi, double xxh, double ds, double& f, double& df) {
    const double p2 = psi * psi, p3 = p2 * psi, p4 = p3 * psi;
    f = p4 / 12 + xxh * p3 / 3 + p2 + (2 * xxh - 2 * ds) * psi - 2 * ds * xxh + xxh * xxh;
    df = p3 / 3 + xxh * p2 + 2 * psi + 2 * xxh - 2 * ds;
  }
  __device__ static double root(double x1, double x2, double xacc, double ds, double xxh) {
    double fl, fh, f, df, xl, xh;
    quartic(x1, xxh, ds, fl, df);
    quartic(x2, xxh, ds, fh, df);
    if (fabs(fl) < xacc) return x1;
    if (fabs(fh) < xacc) return x2;
    if (fl < 0.0) { xl = x1; xh = x2; } else { xh = x1; xl = x2; }
    double rts = 0.5 * (x1 + x2);
    double dxold = fabs(x2 - x1), dx = dxold;
    quartic(rts, xxh, ds, f, df);
    for (int j = 1; j <= 100; j++) {
      if (((rts - xh) * df - f) * ((rts - xl) * df - f) > 0.0 ||
          fabs(2.0 * f) > fabs(dxold * df)) {
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
      quartic(rts, xxh, ds, f, df);
      if (f < 0.0) xl = rts; else xh = rts;
    }
    return rts;
  }
  __device__ double caseD(double xxbarh, double psimax, double ssh) const {
    const double psi = root(-epstol, psimax * (1.0 + epstol), epstol, ssh, xxbarh);
    const double pa = psi + xxbarh;
    const double pb = psi * (xxbarh + psi / 2.0);
    return xk2 * (-2.0 * (pa + psi * pb) / (pa * pa + pb * pb) + 1.0 / ssh);
  }
};

__device__ double csr_node(int i, const double* __restrict__ rho, double r0, double ptmin,
                           double hx, double blength, double gam) {
  const double pilc = 2 * asin(1.0);
  const double phim = blength / r0;
  const double xconst = 1.0 / (4 * pilc * 8.854187817e-12);
  CsrKernel K;
  K.r0 = r0;
  K.gam = gam;
  K.xk2 = gam / r0;
  K.g3 = gam * gam * gam;
  K.epstol = 2.0e-9;
  if (i == 1) return 0.0;
  const double xx = ptmin + (i - 1) * hx;
  const double t = xx / r0;
  const double xxl = t * t * t * r0 / 24;
  const int ni = i;
  double e = 0.0;
#define RHO(j) rho[(j)-1]
#define SSH(xxp) ((xx - (xxp)) * K.g3 / r0)
  if (xx <= 0) {
  } else if (xx <= blength) {
    const double xslp = (xx / r0) * r0 / 2 / gam / gam + xxl;
    const int islp1 = (int)((xx - xslp - ptmin) / hx) + 1;
    const double phih = xx / r0 * gam;
    for (int j = 2; j <= islp1 - 1; j++) {
      const double c2 = K.caseA(phih, SSH(ptmin + (j - 1) * hx + hx / 2));
      const double c1 = K.caseA(phih, SSH(ptmin + (j - 1) * hx - hx / 2));
      e = e + RHO(j) * (c1 - c2);
    }
    if (islp1 >= 2) {
      double c2 = K.caseA(phih, SSH(xx - xslp));
      double c1 = K.caseA(phih, SSH(ptmin + (islp1 - 1) * hx - hx / 2));
      e = e + RHO(islp1) * (c1 - c2);
      c2 = K.caseA(phih, SSH(ptmin + hx / 2));
      c1 = K.caseA(phih, SSH(ptmin));
      e = e + RHO(1) * (c1 - c2);
    } else if (islp1 == 1) {
      const double c2 = K.caseA(phih, SSH(xx - xslp));
      const double c1 = K.caseA(phih, SSH(ptmin + (islp1 - 1) * hx));
      e = e + RHO(islp1) * (c1 - c2);
    }
    const int jstart = islp1 > 1 ? islp1 : 1;
    for (int j = jstart + 2; j <= ni - 1; j++) {
      const double c2 = K.caseB(SSH(ptmin + (j - 1) * hx + hx / 2));
      const double c1 = K.caseB(SSH(ptmin + (j - 1) * hx - hx / 2));
      e = e + RHO(j) * (c1 - c2);
    }
    if (jstart <= ni - 2) {
      double c2 = K.caseB(SSH(ptmin + (ni - 1) * hx));
      double c1 = K.caseB(SSH(ptmin + (ni - 1) * hx - hx / 2));
      e = e + RHO(ni) * (c1 - c2);
      if (islp1 < 1) {
        c2 = K.caseB(SSH(ptmin + hx / 2));
        c1 = K.caseB(SSH(ptmin));
        e = e + RHO(1) * (c1 - c2);
      } else {
        const int j = islp1 + 1;
        c2 = K.caseB(SSH(ptmin + (j - 1) * hx + hx / 2));
        c1 = K.caseB(SSH(xx - xslp));
        e = e + RHO(j) * (c1 - c2);
      }
    } else if (jstart == ni - 1) {
      const double c2 = K.caseB(SSH(ptmin + (ni - 1) * hx));
      const double c1 = K.caseB(SSH(xx - xslp));
      e = e + RHO(ni) * (c1 - c2);
    }
  } else {
    const double xxbar = xx - blength;
    const double rp = r0 * phim;
    const double xslp = (rp + xxbar) / 2 / gam / gam +
                        r0 * (phim * phim * phim) / 24 * (rp + 4 * xxbar) / (rp + xxbar);
    const int islp1 = (int)((xx - xslp - ptmin) / hx) + 1;
    const double xslpN = xxbar / 2.0 / gam / gam;
    const int islpN1 = (int)((xx - xslpN - ptmin) / hx) + 1;
    const double xxbarh = xxbar * gam / r0;
    const double phimh = phim * gam;
    for (int j = 2; j <= islp1 - 1; j++) {
      const double c2 = K.caseC(phimh, xxbarh, SSH(ptmin + (j - 1) * hx + hx / 2));
      const double c1 = K.caseC(phimh, xxbarh, SSH(ptmin + (j - 1) * hx - hx / 2));
      e = e + RHO(j) * (c1 - c2);
    }
    if (islp1 >= 2) {
      double c2 = K.caseC(phimh, xxbarh, SSH(xx - xslp));
      double c1 = K.caseC(phimh, xxbarh, SSH(ptmin + (islp1 - 1) * hx - hx / 2));
      e = e + RHO(islp1) * (c1 - c2);
      c2 = K.caseC(phimh, xxbarh, SSH(ptmin + hx / 2));
      c1 = K.caseC(phimh, xxbarh, SSH(ptmin));
      e = e + RHO(1) * (c1 - c2);
    } else if (islp1 == 1) {
      const double c2 = K.caseC(phimh, xxbarh, SSH(xx - xslp));
      const double c1 = K.caseC(phimh, xxbarh, SSH(ptmin));
      e = e + RHO(islp1) * (c1 - c2);
    }
    const double psimax = phim * gam;
    const int jstart = islp1 > 0 ? islp1 : 0;
    for (int j = jstart + 2; j <= islpN1 - 1; j++) {
      const double c2 = K.caseD(xxbarh, psimax, SSH(ptmin + (j - 1) * hx + hx / 2));
      const double c1 = K.caseD(xxbarh, psimax, SSH(ptmin + (j - 1) * hx - hx / 2));
      e = e + RHO(j) * (c1 - c2);
    }
    if (islpN1 >= jstart + 2) {
      double c2 = K.caseD(xxbarh, psimax, xslpN * K.g3 / r0);
      double c1 = K.caseD(xxbarh, psimax, SSH(ptmin + (islpN1 - 1) * hx - hx / 2));
      e = e + RHO(islpN1) * (c1 - c2);
      c2 = K.caseD(xxbarh, psimax, SSH(ptmin + jstart * hx + hx / 2));
      c1 = K.caseD(xxbarh, psimax, xslp * K.g3 / r0);
      e = e + RHO(jstart + 1) * (c1 - c2);
    } else if (islpN1 == jstart + 1) {
      const double c2 = K.caseD(xxbarh, psimax, xslpN * K.g3 / r0);
      const double c1 = K.caseD(xxbarh, psimax, xslp * K.g3 / r0);
      e = e + RHO(jstart + 1) * (c1 - c2);
    }
  }
#undef SSH
#undef RHO
  return e * xconst;
}

// The analytic wake of wakefield_FieldQuant (Field.f90:590-782), the short-
// range wakes of a periodic structure of iris radius aa, gap gg, period
// leng: W_L(z) = Z0 c exp(-sqrt(z/z0)) / (pi aa^2) and
// W_T(z) = 4 Z0 c z1 / (pi aa^4) (1 - (1 + sqrt(z/z1)) exp(-sqrt(z/z1)));
// the fits z0, z1 (Field.f90:627-629, 694-695) keep the reference's default-
// real literals.
struct AnalyticWake {
  double z0l, z0t, coef1, zc, Z0, pilc, aa;
  __device__ static AnalyticWake of(double aa, double gg, double leng, double clight) {
    AnalyticWake w;
    w.pilc = 2 * asin(1.0);
    w.aa = aa;
    w.z0l = (double)0.41f * pow(aa / leng, (double)0.8f) * pow(gg / leng, (double)1.6f) * aa;
    w.Z0 = 120 * w.pilc;
    w.zc = w.Z0 * clight;
    w.z0t = (double)0.169f * aa * pow(aa / leng, (double)1.17f) * pow(gg / aa, (double)0.38f);
    w.coef1 = 4 * w.Z0 * clight * w.z0t / (w.pilc * aa * aa * aa * aa);
    return w;
  }
  __device__ double wl(int j, double hz) const {
    const double zz = j * hz;
    return zc * exp(-sqrt(zz / z0l)) / (pilc * aa * aa);
  }
  __device__ double wt(int j, double hz) const {
    const double zz = j * hz;
    return coef1 * (1.0 - (1. + sqrt(zz / z0t)) * exp(-sqrt(zz / z0t)));
  }
  __device__ double w0_half(double clight) const {
    return 0.5 * Z0 * clight * exp(-sqrt(0.0 / z0l)) / (pilc * aa * aa);
  }
};

// Wake step part 2: the line charge density recvdensz
// (AccSimulator.f90:1297-1322 and 1360-1368) and from it the per-plane field
// that kick1wake adds to the node fields before the gather
// (BeamBunch.f90:5015-5033).  A step with CSR takes the CSR wake
// (AccSimulator.f90:1344-1390, which replaces any other wake), else the
// step's wake (the read-in table or the analytic one), else zero.  The read-in wake: the reference
// convolves on a doubled grid by FFT (wakefieldread_FieldQuant,
// Field.f90:783-1001) with a Green function that is 0.5 W(0) at 0, zero at
// 1..Nz-1 and W((2Nz-k) hz) above; for k < Nz that circular convolution is
// the causal sum
//   conv_z(k) = 0.5 W(0) d(k) + sum_{m>k} d(m) W((m-k) hz),
// evaluated here directly, and the transverse ones (zero at 0 too)
// conv_x(k) = sum_{m>k} d(m) xbar(m) Wx((m-k) hz).  Every block builds the
// density in shared memory; each thread then owns one plane.  The line sums
// are cleared by the field kernel that follows.
__global__ void __launch_bounds__(256) k_wake_field(WakeArgs a) {
  extern __shared__ double wsm[];
  const int nz = a.nz;
  const DevState* st = a.st;
  const int s = a.fixed_step >= 0 ? a.fixed_step : st->step;
  const StepParams& sp = a.steps[s];
  const int kk = blockIdx.x * blockDim.x + threadIdx.x;
  if (!sp.csr && !sp.wake) {
    if (kk < nz) a.wfield[kk] = a.wfield[nz + kk] = a.wfield[2 * nz + kk] = 0.0;
    return;
  }
  const bool csr = sp.csr != 0;
  const bool analytic = !csr && sp.wake == 2;
  const bool tr = analytic || (!csr && sp.wake == 1 && a.transverse);
  const AnalyticWake aw = AnalyticWake::of(sp.wk_aa, sp.wk_gg, sp.wk_len, a.k.Clight);
  double* d = wsm;
  double* dx = wsm + nz;
  double* dy = wsm + 2 * nz;
  double* gz = wsm + 3 * nz;
  double* gx = wsm + 4 * nz;
  double* gy = wsm + 5 * nz;
  const double gam = sp.gam;
  const double cur = st->current;
  const double npt = (double)st->npt;
  double hzw = (st->geom.range[5] - st->geom.range[4]) / (nz - 1);
  hzw = hzw / gam;
  const double sc = ldexp(1.0, a.fixbits);
  int ex, ey;
  frexp(fmax(fabs(st->geom.range[0]), fabs(st->geom.range[1])), &ex);
  frexp(fmax(fabs(st->geom.range[2]), fabs(st->geom.range[3])), &ey);
  const double sx = ldexp(1.0, a.fixbits - ex), sy = ldexp(1.0, a.fixbits - ey);
  const double chrg = a.k.charge, mass = a.k.mass;
  const int ntab = a.ntab;
  for (int k = threadIdx.x; k < nz; k += blockDim.x) {
    const double dens = (double)(long long)a.line[k] / sc;
    const double dk = dens * cur / a.k.Scfreq / npt / hzw * chrg / fabs(chrg);
    double xw = 0.0, yw = 0.0;
    if (tr && dens != 0.0) {
      xw = ((double)(long long)a.line[nz + k] / sx) / dens;
      yw = ((double)(long long)a.line[2 * nz + k] / sy) / dens;
    }
    d[k] = dk;
    if (analytic) {
      dx[k] = dk * xw;
      dy[k] = dk * yw;
      gz[k] = aw.wl(k, hzw);
      gx[k] = gy[k] = aw.wt(k, hzw);
    } else if (!csr) {
      dx[k] = dk * xw;
      dy[k] = dk * yw;
      gz[k] = wake_green(a.table, ntab, a.hwk, k, hzw);
      gx[k] = tr ? wake_green(a.table + ntab, ntab, a.hwk, k, hzw) : 0.0;
      gy[k] = tr ? wake_green(a.table + 2 * ntab, ntab, a.hwk, k, hzw) : 0.0;
    }
  }
  __syncthreads();
  const int k = kk;
  if (k >= nz) return;
  double xycon, tcon;
  kick_consts(a.k, gam, cur, xycon, tcon);
  if (csr) {
    const double zwkmin = st->geom.range[4] / gam + sp.csr_s0;
    const double ez = csr_node(k + 1, d, sp.csr_r0, zwkmin, hzw, sp.csr_blen, gam);
    a.wfield[k] = 0.0;
    a.wfield[nz + k] = 0.0;
    if (sp.lorentz) {  // kick2wake takes the wake as it is, per particle
      a.wfield[2 * nz + k] = 0.0;
      a.wfield[3 * nz + k] = 0.0;
      a.wfield[4 * nz + k] = 0.0;
      a.wfield[5 * nz + k] = ez;
    } else {
      a.wfield[2 * nz + k] = chrg * ez / tcon / mass / a.unit;
    }
    return;
  }
  const double bet = sqrt(gam * gam - 1.0) / gam;
  // greenwake(1) = 0.5 W(0), in each form as the reference writes it
  const double g0 = analytic ? aw.w0_half(a.k.Clight) : 0.5 * gz[0];
  const double scale = analytic ? 1.0 : a.scale;
  double cz = d[k] * g0, cx = 0.0, cy = 0.0;
  if (tr) {
    for (int m = k + 1; m < nz; m++) {
      cz = cz + d[m] * gz[m - k];
      cx = cx + dx[m] * gx[m - k];
      cy = cy + dy[m] * gy[m - k];
    }
  } else {
    for (int m = k + 1; m < nz; m++) cz = cz + d[m] * gz[m - k];
  }
  const double ezwake = scale * (-cz * hzw);
  const double exwake = scale * (cx * hzw);
  const double eywake = scale * (cy * hzw);
  if (sp.lorentz) {  // kick2wake takes the wake as it is, per particle
    a.wfield[k] = 0.0;
    a.wfield[nz + k] = 0.0;
    a.wfield[2 * nz + k] = 0.0;
    a.wfield[3 * nz + k] = exwake;
    a.wfield[4 * nz + k] = eywake;
    a.wfield[5 * nz + k] = ezwake;
    return;
  }
  a.wfield[k] = chrg * exwake / xycon / mass / bet / gam / a.unit;
  a.wfield[nz + k] = chrg * eywake / xycon / mass / bet / gam / a.unit;
  a.wfield[2 * nz + k] = chrg * ezwake / tcon / mass / a.unit;
}

}  // namespace IMPZ_NS
}  // namespace impz
