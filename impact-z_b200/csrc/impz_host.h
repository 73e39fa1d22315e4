// impz_host.h -- host-side builders: transfer-map constants, the RK6 linear
// maps, the lattice-to-step-table compiler and the diagnostic formulas.
#pragma once
#include <vector>

#include "../../include/impz_b200.h"
#include "impz_common.h"

namespace impz {

struct Phys {  // PhysConst (src/DataStruct/PhysConst.f90:25-35)
  double Pi, Clight, Scxl, Rad2deg, Scfreq;
};
Phys make_phys(double freq);

// maplinear_Quadrupole / maplinear_DriftTube and the RF gaps' linear maps
// over an on-axis field table, maplinear_DTL / CCDTL / CCL / SC (types
// 101..104; RK6 of the 18-variable linear ODE); refpt(5), refpt(6) advance
// like the reference.
void maplinear_quad(const Phys& P, double t, double tau, double xm[36], double refpt[6],
                    double gradient, int mapstp, double chg, double mass,
                    const impz_elem_t* fringe = nullptr, double zedge = 0.0);
void maplinear_rfgap(const Phys& P, double t, double tau, double xm[36], double refpt[6],
                     double zedge, const impz_elem_t& e, double chg, double mass);
// maplinear_SolRF (type 105): zdat holds read3_Data's Fourier coefficients
// (ndata values), val[10] the solenoid field Param(12)
void maplinear_solrf(const Phys& P, double t, double tau, double xm[36], double refpt[6],
                     double zedge, const impz_elem_t& e, double chg, double mass);
bool solrf_table_ok(const impz_elem_t& e);
// maplinear_ConstFoc (type 2): k2 = kx0^2, ky0^2, kz0^2 (Param(2..4))
void maplinear_constfoc(const Phys& P, double t, double tau, double xm[36], double refpt[6],
                        const double k2[3], int mapstp);
// maplinear_Sol (type 3): constant field b0 = Param(2)
void maplinear_sol(const Phys& P, double t, double tau, double xm[36], double refpt[6],
                   double b0, int mapstp, double chg, double mass);
// maplinear_TWS (type 106): zdat holds the two series of read3_Data's
// coefficients, val[10] the second wave's phase Param(12)
void maplinear_tws(const Phys& P, double t, double tau, double xm[36], double refpt[6],
                   double zedge, const impz_elem_t& e, double chg, double mass);
bool tws_table_ok(const impz_elem_t& e);

struct BendState {  // the bend constants AccSimulator.f90:1057-1093 keeps
  bool active;
  double gamma0, beta0, hd0, hd1;
  double hB, tanphiB, tanphiBb, psi2, angB;
  double qm0;
};

struct Species {
  double charge, mass, qmi;  // qmi = Pts1(7,:)
};

// One half step of element e (the drift1_BeamBunch dispatch,
// BeamBunch.f90:250-464); appends its map op to prog, updates refptcl.
int half_map_ops(const Phys& P, const impz_elem_t& e, double zedge, double z, double tau,
                 int nst, int ihlf, double refptcl[6], const Species& sp, MapProgram& prog);
// The Lorentz integrator's pieces (Flagmap=2): drift2_BeamBunch's op by
// tau/2 with refptcl(5) advanced (BeamBunch.f90:467-509), and kick2's
// field terms for a step table entry at z (tg = refptcl(5); LzKind) with
// gamma0 moved by tau qmcc Ez0 (BeamBunch.f90:2187-2508); false for an
// element outside the integrator.
int drift2_op(const Phys& P, double tau, double refptcl[6], MapProgram& prog);
// `data`, when given, receives the per-step field data of the kick (EMfld
// 110: the plane at z), whose offset the coefficients c carry.
bool lorentz_kick_terms(const Phys& P, const impz_elem_t& e, double zedge, double z, double tau,
                        const Species& sp, double refptcl[6], int& kind, double c[16],
                        double& tg, double& ez0, std::vector<double>* data = nullptr);
// Bend entry (refptcl(5) update + Fpol op), Sector op, Bpol op.
int bend_entry_ops(const Phys& P, const impz_elem_t& e, double refptcl[6], const Species& sp,
                   BendState& bs, MapProgram& prog);
void bend_sector_op(const Phys& P, const BendState& bs, double tau, const Species& sp,
                    MapProgram& prog);
void bend_exit_op(const Phys& P, const BendState& bs, const Species& sp, MapProgram& prog);

struct CompiledLattice {
  std::vector<StepParams> steps;  // [0] prologue, [1..K] steps, [K+1] sentinel
  std::vector<double> zrec;       // z of each record (K+1)
  std::vector<double> refrec;     // refptcl of each record, 6 per record
  int nsteps;
  bool has_wake;                  // some step kicks with a wake (read-in, analytic or CSR)
  std::vector<double> lz_data;    // field data of Lorentz kicks (EMfld planes), in device order
};
// The state of run_AccSimulator's element loop that decides where wakes
// act: the bend bookkeeping of CSR (AccSimulator.f90:638-740, 1032-1051,
// 1131-1138, 1498-1499) and the wake switches (flagwake, flagwakeread of
// -41 elements and 105/106 structures, AccSimulator.f90:865-875, 959-978).
struct LoopState {
  double zbleng = 0.0;      // sum of the lengths of the elements passed
  double sentr = 0.0;       // distance from the last CSR bend's entrance
  double bendlencsr = 0.0;  // that bend's length
  double r0 = 0.0;          // radius of the last bend
  int flagbendcsr = 0;      // the last bend had dparam(4) > 500
  int flagwake = 0;         // the kicks include a wake
  int flagwakeread = 0;     // ... the read-in one (-41), else the analytic one
  double aawk = 0.0, ggwk = 0.0, lengwk = 0.0;  // the last 105/106's Param(13..15)
  int flagmap = 1;          // 1 the linear map integrator, 2 the Lorentz integrator (-25)
};
// run_AccSimulator's element/segment loop (AccSimulator.f90:742-1504)
// turned into a step table.  refptcl, z and the CSR state advance to the
// lattice exit.
int compile_lattice(const Phys& P, const impz_elem_t* elems, int nelem, double bcurr,
                    const Species& sp, double refptcl[6], double* z, LoopState& csr,
                    CompiledLattice& out);

// diagnostic1_Output rank-0 formulas (Output.f90:247-352)
void diag_row(const Phys& P, double z, const double rec[IMPZ_MOMREC], const double refptcl[6],
              double mass, double row[IMPZ_DIAG_LEN]);

}  // namespace impz
