// impz_common.h -- types shared by the host runtime and the sm_100a kernels.
//
// Particle state lives on the device as six FP64 structure-of-arrays columns
// (x/Scxl, gamma*beta_x, y/Scxl, gamma*beta_y, phase, gamma0-gamma), the
// first six rows of the reference's Pts1(9,N) (src/Appl/BeamBunch.f90:9-12).
// Rows 7 (q/m) and 8 (charge weight) are per-bunch constants for the single
// species the map integrator supports (BeamBunch.f90:13-14); row 9 (id) is an
// optional int64 column carried through the per-step particle sort.
#pragma once
#include <stdint.h>

#define IMPZ_RAW_LEN 44     // 37 moment sums, 6 |max|, 1 max r^2 (Output.f90:133-245)
#define IMPZ_MAXOPS 4       // map ops per program
#define IMPZ_OPC 40         // coefficients per map op

namespace impz {

// One per-particle transfer map, with every constant the per-particle loop
// of the reference routine needs precomputed on the host.
enum MapKind : int {
  MAP_NONE = 0,
  MAP_DRIFT = 1,     // drift1_BeamBunch bitype 0 (BeamBunch.f90:276-298)
  MAP_XM6 = 2,       // 6x6 linear map loop (BeamBunch.f90:310-320)
  MAP_KQUAD = 3,     // transfmapK_Quadrupole (Quadrupole.f90:509-607)
  MAP_IDEALRF = 4,   // ideal RF gap (BeamBunch.f90:324-440)
  MAP_FPOL = 5,      // Fpol_Dipole (Dipole.f90:466-526)
  MAP_BPOL = 6,      // Bpol_Dipole (Dipole.f90:528-591)
  MAP_SECTOR = 7,    // Sector_Dipole (Dipole.f90:693-788)
  MAP_XM2 = 8,       // 6x6 map with only its three 2x2 diagonal blocks nonzero
  MAP_UNDUL = 9,     // transfUndulator_Quadrupole (Quadrupole.f90:611-665)
  MAP_DRIFT2 = 10,   // drift2_BeamBunch, the Lorentz integrator's drift (BeamBunch.f90:467-509)
};

struct MapOp {
  int kind;
  int flags;   // XM6: bitmask of nonzero entries (36 bits in c[36..]); RF: 1 entrance, 2 exit
  int iparam;  // RF: 2*nseg
  int pad;
  double c[IMPZ_OPC];
};

// The external field (E, B) of a Lorentz-integrator step's element at the
// kick's z (getfld_BeamLineElem, BeamLineElem.f90:827-867), as a function
// of X, Y [m] and the particle's time T = phase + tg; E_x = E_y = 0 for all.
//   LZ_NONE      drift (getfld_DriftTube): 0
//   LZ_QUAD      hard-edge quadrupole, c0 = G: B = (G Y, G X, 0)
//   LZ_QUAD_FRG  Enge fringe (getfldfrgAna2_Quadrupole), c = (G, G', G''):
//                Bx = G Y - G''(Y^3 + 3 X^2 Y)/12, By = G X - G''(X^3 + 3 X Y^2)/12,
//                Bz = G' X Y
//   LZ_SOL       solenoid body or outside (getfld_Sol): B = (0, 0, c1)
//   LZ_SOL_FRG   solenoid ramp, c0 = dBz/dz: B = (-c0/2 X, -c0/2 Y, c1)
//   LZ_CONSTFOC  constant focusing (getfld_ConstFoc), c = (kx, ky, kz):
//                Ez = kz T Scxl, Bx = -kx Y / c, By = ky X / c
//   LZ_RF        RF cavity 101..104 (getfld_DTL / CCDTL / CCL / SC), c =
//                (G, ez1, ez1', f1, f1', w, theta0, xl c) with the on-axis
//                Fourier sums at z; per particle, phi = w T + theta0:
//                E = (-X (ez1'/2 + f1' r^2/4) cos phi, same with Y,
//                (ez1 + f1 r^2) cos phi), B = (G Y + Y/(xl c)(ez1/2 + f1 r^2/4)
//                sin phi, G X - X/(xl c)(...) sin phi, 0); G the DTL's
//                drift-tube quadrupole gradient, 0 for the others
//   LZ_SOLRF     SolRF 105 (getfld_SolRF): t = T / (2 pi Scfreq),
//   LZ_TWS       phi = w t + theta0, r = xlrep, the wave c[4..7] = (ez1,
//                ez1', f1, f1') as LZ_RF but B = (Y r/c (...) sin phi, -X r/c
//                (...) sin phi, 0); c = (w, xlrep, 2 pi Scfreq, theta0, wave,
//                then SolRF's solenoid (bscale times bz, bz', bz'', bz''')
//                B += (-bz'/2 X + bz''' X r^2/16, same with Y, bz - bz'' r^2/4),
//                or TWS 106's second wave (ez1, ez1', f1, f1', theta2) at
//                phi + theta2)
//   LZ_EMFLD     EMfld 110 with discrete x-y-z data (scatter2, FlagDisc 1,
//                FlagCart 2): c = (escale, ww, theta0, xmin, hx, 1/hx, ymin,
//                hy, 1/hy, NxIntvRfg, NyIntvRfg, offset of the step's complex
//                field plane in AdvanceArgs::lz_data); nine-point quadratic
//                interpolation in x, y of each component times escale
//                e^{i(ww T + theta0)}, real part
//   LZ_MULT      multipole 5 (getfld_Multipole, MAD notation), c = (G, id):
//                sextupole (id 2) B = (G X Y, G (X^2 - Y^2)/2, 0), octupole
//                (3) G (3 X^2 Y - Y^3)/6, G (X^3 - 3 X Y^2)/6, decapole (4)
//                G (X^3 Y - X Y^3)/6, G (X^4 - 6 X^2 Y^2 + Y^4)/24
enum LzKind {
  LZ_NONE = 0,
  LZ_QUAD = 1,
  LZ_QUAD_FRG = 2,
  LZ_SOL = 3,
  LZ_SOL_FRG = 4,
  LZ_CONSTFOC = 5,
  LZ_RF = 6,
  LZ_SOLRF = 7,
  LZ_TWS = 8,
  LZ_MULT = 9,
  LZ_EMFLD = 10
};

struct MapProgram {
  int nops;
  int pad;
  MapOp ops[IMPZ_MAXOPS];
};

// Everything one step needs that the host knows in advance.  Entry s of a
// step table describes step s; the particle pass of step s applies `post`,
// records moments, applies `pre_next` and evaluates conv1st for step s+1
// with steps[s+1].gam and steps[s+1].rad.
struct StepParams {
  MapProgram post;     // second half map of this step (after the kick)
  MapProgram pre_next; // first half map of the next step (+ pole faces)
  int sc;              // this step kicks (a deposit and a field solve preceded it)
  int moments;         // record diagnostics after `post`
  int range_next;      // evaluate conv1st of step s+1 after `pre_next`
  int csr;             // this step's kick includes the CSR wake (csr_* below)
  double gam;          // -refptcl(6) during this step's conv1st/kick
  double tau;          // tau2 of the kick
  double rad;          // (piperad+piperad2)/2 for this step's conv1st loss test
  double csr_r0;       // CSR: radius of the bend
  double csr_s0;       // CSR: distance of the kick from the bend entrance (z - zbleng [+ sentr])
  double csr_blen;     // CSR: bend length
  int wake;            // wake of this step's kick: 0 none, 1 read-in table, 2 analytic
  int pad3;
  double wk_aa, wk_gg, wk_len;  // analytic wake: iris radius, gap, period (Param(13..15))
  int lorentz;         // the kick is the Lorentz integrator's (kick2/scatter2)
  int lz_kind;         // LzKind of its element's external field
  double lz_c[16];     // that field's coefficients at the kick's z (LzKind)
  double lz_tg;        // refptcl(5) at the kick (scatter2's tg)
  double lz_ez0;       // the field's Ez on axis at tg (scatter2's ez0)
};

#define IMPZ_MOMREC 48   // per recorded step: 44 raw values, npt, nlocal, current, spare

// update_CompDom output for one step, plus the conv1st range that fed it.
struct Geom {
  double ptrange[6];   // raw particle range (conv1st)
  double range[6];     // xmin,xmax,ymin,ymax,zmin,zmax after padding
  double h[3];         // hx,hy,hz
  double hi[3];        // 1.0/h
};

struct DevState {
  Geom geom;
  double current;      // BeamBunch%Current after the loss rescale
  double xycon, tcon;  // scatter1 kick constants of the current step
  long long npt;       // BeamBunch%Npt
  long long nlocal;    // particles stored in the current buffer
  long long nlive;     // particles that survive the pending conv1st
  int step;            // index of the current step in the step table
  int parity;          // which particle buffer holds the state
  unsigned int err;    // sticky error bits (IMPZ_DERR_*)
  unsigned int done_range, done_mom, done_scan;
  unsigned int pad0;
  double charge_unit;  // FP64 form: weight * 2^-fixbits (grid value per quantum)
  double rhomax;       // unused placeholder for alignment
};

enum DevErr : unsigned int {
  DERR_NONFINITE = 1u,   // a particle coordinate became Inf/NaN
  DERR_OUTSIDE = 2u,     // a live particle fell outside the deposit grid
  DERR_FIXOVF = 4u,      // fixed-point charge grid overflow guard
  DERR_SLOT = 8u,        // a sorted slot fell outside the buffer (deposit/pass mismatch)
};

struct Consts {  // per-bunch constants (PhysConst.f90:25-35 and the species)
  double Scxl, xk, Clight, Pi, Scfreq;
  double mass, charge, qm0, qmi;  // qm0 = Charge/Mass, qmi = Pts1(7,:)
};

// Launch arguments of the fused particle pass.  The step index is either
// fixed by the host or read from DevState::step, so one captured CUDA graph
// can replay every step of a lattice.
struct AdvanceArgs {
  const double* in[6];
  double* out[6];
  const long long* id_in;   // may be null (ids not tracked)
  long long* id_out;
  const StepParams* steps;
  DevState* st;
  int nx, ny, nz;
  int nspecies;             // species of a multi-species bunch (sp_in set), else 0
  long long cap;            // particle capacity of the output buffer
  const void* efield;       // per node {Ex,Ey,Ez,0}: double in the FP64 form, float otherwise
  double efield_scale;      // FP32 form: charge weight (field solved for unit charges)
  int* cursor;              // per-cell sort cursors (scan-block local offsets)
  const int* bsum;          // exclusive offset of each scan block
  double* mom_part;         // [gridDim][IMPZ_RAW_LEN]
  double* rng_part;         // [gridDim][8]
  double* mom_out;          // [records][IMPZ_MOMREC]
  Consts k;
  int fixed_step;           // >= 0: step index; < 0: read and advance DevState::step
  int kick;                 // 1: gather + kick (steps[s].sc must be set)
  int do_post;              // apply steps[s].post (+ moments if steps[s].moments)
  int do_pre;               // apply steps[s].pre_next (+ conv1st of s+1 if range_next)
  int mom_index;            // record row for fixed_step launches
  int tframe;               // 1: conv1st's frame between passes (the whole-lattice runner):
                            //    a kick reads it, a pass with range_next writes it
  const double* wake_raw;   // per-plane wake {Ex,Ey,Ez}[nz] of a Lorentz step (kick2wake), or null
  const double* lz_data;    // field data of the Lorentz kicks (LZ_EMFLD planes), or null
  // multi-species bunches (Pts1 rows 7 and 8 differ between particles):
  // each particle's species index, permuted with the sort like the ids
  const unsigned char* sp_in;  // null for a single-species bunch
  unsigned char* sp_out;
  const double* sp_qm;      // [IMPZ_MAX_SPECIES] Pts1(7) of each species
  int* sp_cnt;              // [records][nspecies] particles kept per species (chgupdate), or null
};

struct DepositArgs {
  const double* in[6];
  const StepParams* steps;
  DevState* st;
  int fixed_step;
  int nx, ny, nz;
  int fixbits;
  int tframe;               // 1: the particles are stored in conv1st's frame (AdvanceArgs)
  unsigned long long* rho;  // G int64 (two's complement) accumulators
  int* counts;              // G+1 per-cell particle counts by sort key (cell_key; slot G:
                            // live but outside)
  double xl;
  const unsigned char* sp_in;  // species index per particle (multi-species bunches), or null
  const double* sp_w;       // [IMPZ_MAX_SPECIES] Pts1(8) of each species / the bunch's weight
};

// Read-in wakefield of type -41 elements: the line density (and, with the
// transverse wake, the x/y moments) on the z grid, then the per-plane field
// added to the node fields before the gather.
struct WakeArgs {
  const double* in[6];
  const StepParams* steps;
  const DevState* st;
  int fixed_step;
  int nz;
  int fixbits;               // fixed-point resolution of the line sums
  int transverse;            // 1: x/y moments and the transverse wakes too
  int ntab;                  // wake table rows
  int tframe;                // 1: the particles are stored in conv1st's frame (AdvanceArgs)
  unsigned long long* line;  // [3][nz] int64 sums (density, x, y), left cleared
  const double* table;       // [3][ntab]: longitudinal, x and y wake columns
  double* wfield;            // [3][nz] out: added to Ex, Ey, Ez of plane k
  double hwk;                // table spacing (second z minus first)
  double scale;              // the element's wake scale (Param(2))
  double unit;               // grid-field unit: 1 (FP64 form) or the charge weight (FP32 form)
  double xl;
  Consts k;
};

// One bunch of a group of bunches with the same grid size and form, for the
// field solve launched once for the whole group (the *_group kernels):
// blockIdx.y or blockIdx.z selects the member.
struct PoissonMember {
  unsigned long long* rho;  // int64 charge (read by the forward pass, cleared by the field)
  double qscale;            // grid value of one fixed-point quantum
  void* spec;               // spectrum (complex T)
  void* ghat;               // G-hat octant (T) / DCT work
  void* phi;                // potential (T)
  void* efield;             // {Ex,Ey,Ez,0} per node (T)
  const void* twx;          // twiddles of length 2nx, 2ny, 2nz (complex T)
  const void* twy;
  const void* twz;
  double* F;                // IGF corners
  DevState* st;
};

// the arguments of one bunch's count scan in a packed launch (k_scan)
struct ScanArgs {
  int* counts;
  int* cursor;
  int* bsum;
  long long total;
  DevState* st;
};

#ifndef IMPZ_MAX_SPECIES
#define IMPZ_MAX_SPECIES 128   // distinct (q/m, weight) pairs of a multi-species bunch
#endif
#define IMPZ_SCAN_LOG 12      // 4096 cells per scan block (1024 threads x 4)
#ifndef IMPZ_DEP_TILE
#define IMPZ_DEP_TILE 4096    // deposit tile entries: two int32 halves + an int32 count (48 KB)
#endif

}  // namespace impz
