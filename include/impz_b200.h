/*
 * impz_b200.h -- C ABI of the B200 space-charge kick and element push.
 *
 * Drop-in for the per-step calls that IMPACT-Z's step loop
 * (src/Contrl/AccSimulator.f90:1099-1488) makes into BeamBunch, CompDom and
 * FieldQuant.  Every entry point takes plain pointers and scalars (a Fortran
 * caller binds them with iso_c_binding; see impact-z_b200/fortran/), returns
 * IMPZ_OK (0) or a negative IMPZ_ERR_* code, and never aborts the caller.
 * Arrays follow the reference's column-major layout:
 *   particles  Pts1(9,n): pts[9*i + c], c = x/Scxl, gbx, y/Scxl, gby, phase,
 *              gamma0-gamma, q/m, charge weight, id   (BeamBunch.f90:9-12)
 *   grids      (nx,ny,nz): g[i + nx*(j + ny*k)]
 *   6x6 maps   xm(6,6): xm[(j-1) + 6*(k-1)]
 * All device work of a bunch runs on that bunch's CUDA stream; the calls
 * are synchronous unless the name says otherwise.  One host thread at a time
 * may use a given handle.
 */
#ifndef IMPZ_B200_H
#define IMPZ_B200_H
#ifdef __cplusplus
extern "C" {
#endif

#define IMPZ_OK 0
#define IMPZ_ERR_ARG (-1)         /* invalid argument */
#define IMPZ_ERR_NOMEM (-2)       /* device or host allocation failed */
#define IMPZ_ERR_CUDA (-3)        /* CUDA runtime error (see impz_last_cuda_error) */
#define IMPZ_ERR_UNSUPPORTED (-4) /* element / option outside the supported path */
#define IMPZ_ERR_NONUNIFORM (-5)  /* q/m or charge weight differ between particles */
#define IMPZ_ERR_STATE (-6)       /* call out of order (e.g. kick before deposit) */
#define IMPZ_ERR_NONFINITE (-7)   /* a particle coordinate became Inf/NaN */
#define IMPZ_ERR_NODEVICE (-8)    /* no CUDA device / extension built without GPU */
#define IMPZ_ERR_BUDGET (-9)      /* admission refused: footprint above budget */
#define IMPZ_ERR_LIMIT (-10)      /* grid above IMPZ_STATIC_MAX_CELLS (impz_deposit_static) */

/* numerical forms */
#define IMPZ_FORM_FP64 0     /* plain: all FP64, reference operation order, no FMA */
#define IMPZ_FORM_FP32CONV 1 /* FP32 FFT convolution and field gather, FP64 elsewhere */

/* bunch creation flags */
#define IMPZ_FLAG_TRACK_IDS 1 /* carry Pts1(9,:) through the per-step particle sort */
#define IMPZ_FLAG_SPECIES 2   /* multi-species bunch: Pts1(7,:) and Pts1(8,:) per particle */
#ifndef IMPZ_MAX_SPECIES
#define IMPZ_MAX_SPECIES 128  /* distinct (Pts1(7), Pts1(8)) pairs of one bunch */
#endif

#define IMPZ_RAW_LEN 44   /* 37 moment sums, 6 |max|, max r^2 */
#define IMPZ_DIAG_LEN 45  /* one row of fort.18/24-30, see impz_diag_row */
#define IMPZ_MOMREC 48    /* raw record: IMPZ_RAW_LEN values, Npt, Nptlocal, Current, 0 */

typedef struct impz_bunch_s* impz_bunch_t;

/* One lattice line of ImpactZ.in: "L nseg mapstp type v1 .. v24 /"
 * (src/Contrl/Input.f90:300-315).  Param(1) of the reference element is
 * zedge, Param(k) = val[k-2] for k >= 2 (AccSimulator.f90:262-330).
 * Supported types: 0 drift, 1 quadrupole (gradient; K map when v2 in
 * (-10,-1e-6); the undulator map when v2 < -10; with v2 > 1e-5 the
 * gradient profile of its rfdataN.in in zdat/edat), 2 constant focusing
 * (kx0^2, ky0^2, kz0^2 = v1..v3), 3 solenoid (constant field v1,
 * maplinear_Sol), 4 dipole (file ID v3 <= 200: no CSR; above 200 CSR
 * inside the bend, above 500 also downstream: impz_run only), 101..106 RF gaps
 * as the ideal-RF model (v4 < 0), and otherwise as RK6 linear maps:
 * 101 DTL (with its drift-tube quadrupoles, v6..v9), 102 CCDTL, 103 CCL and
 * 104 SC over the on-axis table zdat/edat/epdat/eppdat (rfdataN.in,
 * read1_Data); 105 SolRF (solenoid field v11) and 106 TWS (second wave's
 * phase v11) over read3_Data's Fourier coefficients in zdat (ndata values,
 * the other table pointers unused).  Under the Lorentz integrator
 * (impz_set_integrator(b, 2)) types 101..104 also take read3_Data's
 * Fourier coefficients in zdat, as the reference reads them then
 * (AccSimulator.f90:826-848). */
typedef struct {
  int type;
  int nseg;
  int mapstp;
  int ndata;
  double length;
  double val[24];
  const double* zdat;
  const double* edat;
  const double* epdat;
  const double* eppdat;
} impz_elem_t;

/* ---- library ------------------------------------------------------------ */
const char* impz_version(void);
const char* impz_error_string(int code);
const char* impz_last_cuda_error(void);
/* Select the CUDA device for subsequent calls on this host thread. */
int impz_set_device(int device);

/* ---- BeamBunch / FieldQuant / CompDom lifetime ------------------------------ */
/* construct_BeamBunch + setpts (BeamBunch.f90:41-60, 3632-3644) together with
 * construct_CompDom/construct_FieldQuant of one rank: uploads Pts1(9,n) into
 * device SoA state and sizes the nx*ny*nz grid (powers of two, >= 4).
 * freq is Scfreq (PhysConst.f90:25-35).  refptcl[6] as BeamBunch%refptcl. */
int impz_bunch_create(const double* pts, long long n, double current, double mass,
                      double charge, double freq, const double refptcl[6], int nx, int ny,
                      int nz, int form, int flags, impz_bunch_t* out);
/* Pts1 rows 7 (q/m) and 8 (charge weight) are per-bunch constants unless the
 * bunch is created with IMPZ_FLAG_SPECIES; without it, rows that differ
 * from the first particle's are IMPZ_ERR_NONUNIFORM.  With it, each
 * distinct (row 7, row 8) pair is a species (at most IMPZ_MAX_SPECIES, else
 * IMPZ_ERR_LIMIT) carried per particle through the sort: the deposit weights
 * each particle by its row 8 (deposit_BeamBunch, BeamBunch.f90:3749-3763),
 * and the K-map quadrupole, the bend maps and the Lorentz kick use its row 7
 * (Quadrupole.f90:533, Dipole.f90:466-591 and 693-788, BeamBunch.f90:3026-3035), as the
 * reference's multiple charge states do (BeamBunch.f90:13-14: the map
 * integrator's space-charge kick keeps the bunch's charge/mass). */
/* getpts_BeamBunch (BeamBunch.f90:3663-3675): copies the live particles back
 * into pts (capacity cap particles); *n receives the live count.  Without
 * IMPZ_FLAG_TRACK_IDS column 9 is filled with 1..n in the current order. */
int impz_bunch_download(impz_bunch_t b, double* pts, long long cap, long long* n);
int impz_bunch_destroy(impz_bunch_t b);
/* Device bytes a bunch of n particles on an nx*ny*nz grid holds while it runs
 * a lattice of nsteps steps (0: the bunch alone), at the driver's 2 MiB
 * allocation granularity: the bunch is one allocation, the run tables a
 * second, and no other call allocates but impz_wake_set and the first run
 * with CSR steps (the wake table and per-step line buffers, a few 10 KB).
 * The serving loop admits by it.
 * No reference counterpart (the reference allocates per process). */
long long impz_bunch_footprint(long long n, int nx, int ny, int nz, int form, int flags,
                               int nsteps);
/* Bunching factor of the live particles at wavenumber k [1/m]:
 * out[0] + i out[1] = (1/N) sum_j exp(-i k z_j), z_j = -phase_j beta0 Scxl
 * their longitudinal position; |out| is the bunching factor.  No reference
 * counterpart (a diagnostic of the chicane study on this path). */
int impz_bunching(impz_bunch_t b, double wavenumber, double out[2]);
/* Read-in wakefield of a type -41 element (AccSimulator.f90:959-978):
 * impz_wake_set turns it on for every space-charge step that follows, as
 * the reference's flagwake does, with table = ntab rows of (z, longitudinal,
 * x, y wake) as in rfdataN.in (read1wk_Data, Data.f90:559-633; z is
 * shifted to start at 0 here), scale = Param(2) (scwk) and transverse = 0
 * when Param(4) < 10 (flagbtw = 2: no transverse wake).  Each step then
 * forms the line density on the z grid, convolves it with the table
 * (wakefieldread_FieldQuant, Field.f90:783-1001) and adds the per-plane
 * field to the node fields before the gather (kick1wake_BeamBunch,
 * BeamBunch.f90:4694-5046).  Allocates the table and its per-step buffers
 * (outside impz_bunch_footprint).  IMPZ_ERR_ARG for ntab < 2, a
 * non-increasing z, or nz > 4096.  impz_wake_off is Param(4) <= 0.
 * Type 105/106 structures with Param(15) > 0 carry the analytic wake of
 * Param(13..15) (wakefield_FieldQuant, Field.f90:590-782) without a call,
 * and switch a wake as AccSimulator.f90:865-875 does; the switch state
 * carries from one impz_run to the next. */
int impz_wake_set(impz_bunch_t b, const double* table, int ntab, double scale, int transverse);
int impz_wake_off(impz_bunch_t b);
/* The integrator of the runs that follow (Flagmap of the deck, or a -25
 * element): 1 the linear map integrator, 2 the Lorentz integrator
 * (drift2 half steps around kick2/scatter2, BeamBunch.f90:467-509,
 * 2187-3071, or scatter20 without current), here for drifts, quadrupoles
 * (hard edge, or the Enge fringe of getfldfrgAna2_Quadrupole when
 * Param(3) > 1e-5), constant focusing, solenoids, multipoles (type 5:
 * sextupole, octupole, decapole by Param(2); with Param(4) > 0 the
 * gradient profile of the element's (zdat, edat) table), the RF cavities
 * 101..106 over Fourier coefficients (getfld_Quadrupole, getfld_ConstFoc,
 * getfld_Sol, getfld_DTL/CCDTL/CCL/SC, getfld_SolRF with its solenoid
 * series scaled by Param(12), getfld_TWS), with a read-in or CSR wake applied as
 * kick2wake does (BeamBunch.f90:5048-5938); a run with any other element
 * under it, or a quadrupole with 0 < Param(3) <= 1e-5 (whose field reads
 * unset derivatives there), is IMPZ_ERR_UNSUPPORTED.  Bends stay outside:
 * getfld_Dipole takes pole-face coefficients from the last rfdata file read
 * (nothing loads them for a bend) on top of the sector map's bending. */
int impz_set_integrator(impz_bunch_t b, int flagmap);
/* sizeof(StepParams): the bytes per step of the step table a run uploads. */
int impz_step_params_size(void);
/* Autotuner: times nsteps (2..64) space-charge steps of a short drift on
 * this bunch under candidate launch shapes (deposit blocks, push blocks, z
 * lines per block of the convolution), one parameter at a time, keeps the
 * fastest and restores the bunch (particles, state, z, refptcl) before each
 * trial and at the end.  out = {deposit blocks, push blocks, z lines per
 * block (0: the largest that fits), ms per step}.  Call between runs (the
 * last run's records are overwritten); allocates a snapshot of the
 * particles for its duration.  No reference counterpart. */
int impz_autotune(impz_bunch_t b, int nsteps, double out[4]);
/* Laser heater of a type -52 element (AccSimulator.f90:982-1006): the
 * energy kick pt -= A sin(-h phase) exp(-(x^2+y^2)/(4 rsig^2/Scxl^2)) with
 * A = sqrt(2 (sigx^2 + rsig^2) / rsig^2) ez / mass from the beam's rms x,
 * h the laser frequency over Scfreq; rsig = Param(2) [m], wavelength =
 * Param(3) [m], ez = Param(4) [eV].  Applied between runs. */
int impz_laser_heater(impz_bunch_t b, double rsig, double wavelength, double ez);
/* Current, Npt, Nptlocal, refptcl(1..6), z, device bytes (11 doubles). */
int impz_bunch_info(impz_bunch_t b, double info[11]);
/* The computational domain of the last space-charge step (getrange_CompDom
 * and getmsize_CompDom, CompDom.f90), as a checkpoint records it
 * (outpoint_Output, Output.f90:1733-1774); zeros before the first one. */
int impz_bunch_geom(impz_bunch_t b, double range[6], double msize[3]);
/* Sets the position z [m] of the bunch, as a restart from a checkpoint does
 * (inpoint_Output, Output.f90:1371-1437); call it between runs. */
int impz_bunch_set_z(impz_bunch_t b, double z);
/* The bunch's CUDA stream (cudaStream_t) for callers that interleave work. */
void* impz_bunch_stream(impz_bunch_t b);

/* ---- the reference's per-step call surface ---------------------------- */
/* drift1_BeamBunch (BeamBunch.f90:250-464): one half-step map of element e
 * of length tau at position *z; *z += tau, *ihlf += 1.  nst is the segment
 * (1..nseg) for the ideal-RF entrance/exit kicks.  zedge is Param(1). */
int impz_map_half(impz_bunch_t b, const impz_elem_t* e, double zedge, double* z, double tau,
                  int nst, int* ihlf);
/* Fpol_Dipole at a bend entrance with the constants of AccSimulator.f90:
 * 1057-1093, after refptcl(5) += L/(Scxl*beta0) (AccSimulator.f90:1063).
 * IMPZ_ERR_UNSUPPORTED for a CSR bend (file ID v3 > 200): the whole-lattice
 * runner carries the CSR wake. */
int impz_bend_entry(impz_bunch_t b, const impz_elem_t* e);
/* Sector_Dipole(tau) inside the bend entered last (Dipole.f90:693-788); *z += tau. */
int impz_bend_sector(impz_bunch_t b, double* z, double tau);
/* Bpol_Dipole at the exit of the bend entered last (AccSimulator.f90:1491-1494). */
int impz_bend_exit(impz_bunch_t b);
/* conv1st_BeamBunch (Flagbc=1) + update_CompDom (BeamBunch.f90:1252-1663,
 * CompDom.f90:509-823): z->t range and loss count on the device, current
 * rescale.  Outputs (each may be NULL): *nptot, ptrange[6] (the particle
 * range), range[6] (grid xmin..zmax) and msize[3] (hx,hy,hz). */
int impz_sc_prepare(impz_bunch_t b, double piperad, double piperad2, long long* nptot,
                    double ptrange[6], double range[6], double msize[3]);
/* charge_BeamBunch/deposit_BeamBunch (BeamBunch.f90:3535-3768): CIC into
 * int64 fixed point.  chgdens (nx*ny*nz, may be NULL) receives the FP64 grid
 * in Coulomb like the reference; counts (may be NULL) the per-cell counts. */
int impz_deposit(impz_bunch_t b, double* chgdens, int* counts);
/* update3O_FieldQuant/openBC3D (Field.f90:108-331) on the deposited charge;
 * phi (nx*ny*nz, may be NULL) receives the potential as the reference's FieldQ. */
int impz_poisson_open(impz_bunch_t b, double* phi);
/* cvbkforth1st + kick1 + scatter1 (BeamBunch.f90:1667-2181) with the
 * potential of the last impz_poisson_open; drops the particles conv1st lost
 * and re-sorts the bunch by deposit cell.  egrid (3*nx*ny*nz, may be NULL)
 * receives Ex, Ey, Ez as kick1's egx/egy/egz. */
int impz_kick(impz_bunch_t b, double tau, double* egrid);
/* The Lorentz integrator's per-step calls (Flagmap=2, AccSimulator.f90:
 * 1109-1116, 1446-1469).  impz_drift2 is map1_BeamBunch(Bpts,z,tau2) =
 * drift2_BeamBunch (BeamBunch.f90:467-509): a drift by tau/2,
 * refptcl(5) += tau/(2 Scxl beta0), *z += tau/2.  impz_kick2 is
 * map2_BeamBunch = kick2_BeamBunch (BeamBunch.f90:2187-2508) in element e
 * (zedge = Param(1)) at position z: after impz_sc_prepare, impz_deposit and
 * impz_poisson_open, scatter2 with the space-charge field (as impz_kick it
 * drops the particles conv1st lost and re-sorts; egrid likewise); for a
 * bunch created with current below 1e-10 A, with no solve, scatter20 with
 * the element's field alone.  refptcl(6) then moves by tau qmcc Ez0.
 * IMPZ_ERR_UNSUPPORTED for an element outside impz_set_integrator's list,
 * IMPZ_ERR_STATE for a bunch with current and no solve. */
int impz_drift2(impz_bunch_t b, double* z, double tau);
int impz_kick2(impz_bunch_t b, const impz_elem_t* e, double zedge, double z, double tau,
               double* egrid);
/* diagnostic1_Output sums (Output.f90:133-245) of the current state:
 * rec[IMPZ_MOMREC] = 37 sums, 6 |max|, max r^2, Npt, Nptlocal, Current, 0. */
int impz_moments(impz_bunch_t b, double rec[IMPZ_MOMREC]);
/* diagnostic1_Output's formulas and write columns (Output.f90:247-352):
 * row[0]=z, [1..5] fort.18, [6..11] fort.24, [12..17] fort.25,
 * [18..23] fort.26, [24..29] fort.27, [30..32] fort.28, [33..38] fort.29,
 * [39..44] fort.30.  Host-only arithmetic. */
int impz_diag_row(double z, const double rec[IMPZ_MOMREC], const double refptcl[6],
                  double mass, double freq, double row[IMPZ_DIAG_LEN]);

/* ---- whole-lattice runner ---------------------------------------------- */
/* run_AccSimulator's element/segment loop (AccSimulator.f90:742-1504) for
 * Flagmap=1, Flagbc=1, Flagerr=0, one rank, over elements [0,nelem).
 * Every step is one fused particle pass plus deposit and field solve,
 * replayed from a CUDA graph; with a read-in wake on (impz_wake_set) or in
 * and after CSR bends the step adds the wake's line density and field
 * kernels.  The CSR bookkeeping (AccSimulator.f90:1035-1051, 1131-1138,
 * 1498-1499: lengths passed, distance from the last CSR bend) carries from
 * one run to the next, as one element loop of the reference would; upload
 * resets it.  recs (capacity maxrec records of
 * IMPZ_MOMREC doubles, may be NULL) receives the initial record and one per
 * step; zs (may be NULL) the z of each record; *nrec their number. */
int impz_run(impz_bunch_t b, const impz_elem_t* elems, int nelem, double* recs, double* zs,
             int maxrec, int* nrec);
/* The same, but returns after enqueuing (records land in device memory and
 * are fetched by impz_run_fetch); lets one host thread drive many bunches. */
int impz_run_async(impz_bunch_t b, const impz_elem_t* elems, int nelem);
int impz_run_fetch(impz_bunch_t b, double* recs, double* zs, int maxrec, int* nrec);
/* impz_run_async in parts, for callers that interleave many bunches:
 * begin compiles the lattice and enqueues the prologue; each advance enqueues
 * up to `budget` further steps (at least one) and reports how many remain;
 * once none remain the records can be fetched with impz_run_fetch. */
int impz_run_begin(impz_bunch_t b, const impz_elem_t* elems, int nelem);
int impz_run_advance(impz_bunch_t b, int budget, int* remaining);
/* Advances several bunches, each in its own run (impz_run_begin done; any
 * step counts, grid sizes and lattices; one device and form; no wakes), by
 * up to `steps` steps each, with packed launches: per step one launch of
 * the particle pass, the deposit and the count scan for all of them over a
 * (bunch, block) work list, and one launch per field-solve kernel for each
 * group of equal grid size.  A bunch's arithmetic is that of its own run.
 * remaining[i] (may be NULL) receives each bunch's steps left; a finished
 * run is ready for impz_run_fetch.  The launches go to the first bunch's
 * stream; the other bunches' streams are ordered after them.  The serving
 * loop's multi-job counterpart of impz_run_advance (AccSimulator.f90's
 * step loop for many independent runs at once: no reference counterpart). */
int impz_run_advance_packed(impz_bunch_t* bunches, int nb, int steps, int* remaining);
/* Runs nb bunches, each over its own lattice, with their steps interleaved
 * two at a time on the bunches' own streams so that their kernels overlap on
 * the device (batched scans).  Returns once everything is enqueued; fetch
 * each bunch's records with impz_run_fetch. */
int impz_run_batch(impz_bunch_t* bunches, const impz_elem_t* const* lattices,
                   const int* nelem, int nb);
/* Number of steps (records - 1) impz_run would take for this lattice. */
/* refptcl(1..6) at each record of the last run (6 doubles per record, as
 * BeamBunch%refptcl when diagnostic1_Output wrote that record), for
 * impz_diag_row; *nrec receives the record count (refrec may be NULL). */
int impz_run_reference(impz_bunch_t b, double* refrec, int maxrec, int* nrec);
/* The species of the bunch: (q/m, weight) = Pts1 rows 7 and 8 of each, in
 * order of first appearance in the uploaded rows; returns their number
 * (1 for a bunch without IMPZ_FLAG_SPECIES) and fills up to cap of them. */
int impz_bunch_species(impz_bunch_t b, double* qm, double* weight, int cap);
/* chgupdate_BeamBunch (BeamBunch.f90:688-728): idchg[j] = particles whose
 * q/m is within relative 1e-4 of qmcclist[j], counting those the latest
 * conv1st kept (between impz_sc_prepare and the kick, its loss test
 * decides; otherwise every stored particle).  The rescale of Pts1(8) the
 * reference keeps commented out is not done. */
int impz_chgupdate(impz_bunch_t b, int nchge, const double* qmcclist, int* idchg);
/* For a bunch with IMPZ_FLAG_SPECIES, chgupdate's count of each species at
 * every record of the last whole-lattice run: counts[r * nspecies + k]
 * (nspecies from impz_bunch_species), the particles each step's pass kept
 * after that step's conv1st (a step without space charge loses none).
 * diagnostic1 writes them per charge state to fort.32 (Output.f90:352).
 * IMPZ_ERR_STATE without the flag. */
int impz_run_species(impz_bunch_t b, int* counts, int maxrec, int* nrec);
int impz_count_steps(const impz_elem_t* elems, int nelem);

/* ---- instrumentation --------------------------------------------------- */
/* Kernel groups timed by impz_profile_*: */
#define IMPZ_PROF_DEPOSIT 0  /* charge deposit */
#define IMPZ_PROF_SCAN 1     /* per-cell count scan (sort cursors) */
#define IMPZ_PROF_GREEN 2    /* integrated Green function + its DCT-I */
#define IMPZ_PROF_CONV 3     /* doubled-grid FFT convolution (3 kernels) */
#define IMPZ_PROF_EFIELD 4   /* finite-difference field */
#define IMPZ_PROF_PUSH 5     /* fused gather/kick/map/moments/range/sort pass */
#define IMPZ_PROF_WAKE 6     /* read-in wake: line density + wake field (2 kernels) */
#define IMPZ_PROF_NCAT 7
/* When on, CUDA events bracket every kernel group on the bunch's stream;
 * runs launch directly (no graph replay) and the Green build runs on the
 * bunch's stream, so the groups' intervals are disjoint. */
int impz_profile_enable(impz_bunch_t b, int on);
/* Synchronizes; accumulated milliseconds and launches per group since enable. */
int impz_profile_fetch(impz_bunch_t b, double ms[IMPZ_PROF_NCAT],
                       long long launches[IMPZ_PROF_NCAT]);
/* Process-wide number of kernels this library has launched. */
long long impz_kernel_launches(void);
/* Replace the particles of an existing bunch (same grid and form); n may
 * not exceed the capacity the bunch was created with.  Resets Current to
 * `current` and the bunch's reference particle to refptcl. */
int impz_bunch_upload(impz_bunch_t b, const double* pts, long long n, double current,
                      const double refptcl[6]);

/* ---- serving loop ------------------------------------------------------- */
/* Jobs (a bunch plus its lattice) submitted over time share the GPU: a worker
 * thread admits them in arrival order as soon as their footprint fits the
 * HBM budget and one of max_active slots is free, keeps each job's state
 * resident in HBM, and advances all running jobs a few steps at a time round
 * robin so that their kernels overlap (continuous batching). */
typedef struct impz_server_s* impz_server_t;
int impz_server_create(double hbm_budget_bytes, int max_active, impz_server_t* out);
/* Copies the inputs and queues the job; *job receives its id. */
int impz_server_submit(impz_server_t s, const double* pts, long long n, double current,
                       double mass, double charge, double freq, const double refptcl[6],
                       int nx, int ny, int nz, int form, const impz_elem_t* elems, int nelem,
                       long long* job);
/* Waits up to timeout_s (< 0: forever; returns 1 if still running) for the
 * job; copies its records (as impz_run) and times[3] = latency from submit
 * to completion [s], time queued [s], measured device bytes. */
int impz_server_wait(impz_server_t s, long long job, double timeout_s, double* recs, int maxrec,
                     int* nrec, double times[3]);
/* completed, failed, particle-steps done, seconds from first submit to last
 * completion, bytes admitted now, peak admitted, peak measured per job, queued. */
int impz_server_stats(impz_server_t s, double out[8]);
/* Finishes the queued and running jobs, then stops the worker. */
int impz_server_destroy(impz_server_t s);

/* Host-side maps (for checking and for callers that keep their own loop):
 * maplinear_Quadrupole (Quadrupole.f90:120-252) and the RF gaps'
 * maplinear_DTL / CCDTL / CCL / SC (DTL.f90:136-418, CCDTL.f90, CCL.f90,
 * SC.f90:122-328) by the same RK6; refpt is updated like the reference. */
int impz_maplinear(const impz_elem_t* e, double zedge, double t, double tau,
                   double refpt[6], double charge, double mass, double freq, double xm[36]);

/* ---- charge deposit without device allocation ---------------------------
 * No counterpart in the reference (its deposit works on arrays its own code
 * allocated).  For callers that may not allocate device memory while they
 * run: a host code whose GPU memory all comes from its own pool or arena,
 * or a timed loop that cannot take the device-wide synchronization that
 * cudaMalloc and cudaFree imply.  The caller passes the particles and the
 * output in device memory it owns; the only scratch, the int64 accumulator,
 * is a fixed array of IMPZ_STATIC_MAX_CELLS nodes (4 MiB) in the library's
 * device image, which every GPU that loads the library holds until exit.
 *
 * Deposits the charge density of deposit_BeamBunch (BeamBunch.f90:3678-3768)
 * after conv1st's z->t conversion and loss test, in int64 fixed point with
 * 2^-f of the weight per particle, f = min(40, 62 - ceil(log2(n + 1))) from
 * this call's n.  A bunch fixes its f from its particle count at creation,
 * so chgdens equals impz_deposit's bit for bit when that bunch was created
 * with this n (tested in the plain FP64 form).  Particles outside the box
 * are skipped without a count, as deposit_BeamBunch skips them: a stale box
 * loses their charge silently.  x..pt: device columns of
 * Pts1 rows 1..6 (n particles); gam = -refptcl(6); piperad, piperad2 as for
 * impz_sc_prepare; freq = Scfreq; weight = Pts1 row 8; range[6] (host) =
 * the mesh box (impz_sc_prepare's range); chgdens: device, nx*ny*nz doubles,
 * x fastest.  Launches on `stream` (a cudaStream_t, 0 = default) and returns
 * without synchronizing; IMPZ_ERR_LIMIT if nx*ny*nz > IMPZ_STATIC_MAX_CELLS.
 * The first call on each device (the current one) looks up the array's
 * device address and keeps it; make that first call before any stream
 * capture, and do not use the library across a cudaDeviceReset.  All
 * calls share the array: calls whose kernels can overlap on the GPU (other
 * streams, other host threads) race and give wrong sums. */
#define IMPZ_STATIC_MAX_CELLS (1 << 19)
int impz_deposit_static(const double* x, const double* px, const double* y, const double* py,
                        const double* ph, const double* pt, long long n, double gam,
                        double piperad, double piperad2, double freq, double weight,
                        const double range[6], int nx, int ny, int nz, double* chgdens,
                        void* stream);

#ifdef __cplusplus
}
#endif
#endif
