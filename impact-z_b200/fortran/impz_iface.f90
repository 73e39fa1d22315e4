!----------------------------------------------------------------
! impz_iface.f90 -- iso_c_binding interfaces to libimpz_b200.so
! (include/impz_b200.h) for IMPACT-Z's Fortran driver.
!
! The driver keeps its deck parsing, its element objects and its output
! writers; at each call site of the space-charge step it passes scalars and
! c_loc() of contiguous arrays (never the derived types, which hold pointer
! components and are not interoperable).  Pts1(9,N) is passed as is: its
! column-major layout is the library's particle layout.
!
! Compile with the driver, e.g.  gfortran -c impz_iface.f90, and link
! libimpz_b200.so.  Source only: no Fortran compiler was available where the
! library was built, so this module has been checked against the C header by
! reading, not by compiling.
!----------------------------------------------------------------
      module impz_iface
        use iso_c_binding
        implicit none

        integer(c_int), parameter :: IMPZ_OK = 0
        integer(c_int), parameter :: IMPZ_FORM_FP64 = 0
        integer(c_int), parameter :: IMPZ_FORM_FP32CONV = 1
        integer(c_int), parameter :: IMPZ_FLAG_TRACK_IDS = 1
        integer(c_int), parameter :: IMPZ_FLAG_SPECIES = 2
        integer(c_int), parameter :: IMPZ_MAX_SPECIES = 128
        integer(c_int), parameter :: IMPZ_MOMREC = 48
        integer(c_int), parameter :: IMPZ_DIAG_LEN = 45

        ! one ImpactZ.in lattice line (impz_elem_t)
        type, bind(C) :: impz_elem_t
          integer(c_int) :: type
          integer(c_int) :: nseg
          integer(c_int) :: mapstp
          integer(c_int) :: ndata
          real(c_double) :: length
          real(c_double) :: val(24)
          type(c_ptr) :: zdat = c_null_ptr
          type(c_ptr) :: edat = c_null_ptr
          type(c_ptr) :: epdat = c_null_ptr
          type(c_ptr) :: eppdat = c_null_ptr
        end type impz_elem_t

        interface
          integer(c_int) function impz_set_device(dev) bind(C, name="impz_set_device")
            import :: c_int
            integer(c_int), value :: dev
          end function

          integer(c_int) function impz_bunch_create(pts, n, current, mass, charge, freq, &
              refptcl, nx, ny, nz, form, flags, bunch) bind(C, name="impz_bunch_create")
            import :: c_int, c_long_long, c_double, c_ptr
            real(c_double), intent(in) :: pts(9, *)
            integer(c_long_long), value :: n
            real(c_double), value :: current, mass, charge, freq
            real(c_double), intent(in) :: refptcl(6)
            integer(c_int), value :: nx, ny, nz, form, flags
            type(c_ptr), intent(out) :: bunch
          end function

          integer(c_int) function impz_bunch_download(bunch, pts, cap, n) &
              bind(C, name="impz_bunch_download")
            import :: c_int, c_long_long, c_double, c_ptr
            type(c_ptr), value :: bunch
            real(c_double), intent(out) :: pts(9, *)
            integer(c_long_long), value :: cap
            integer(c_long_long), intent(out) :: n
          end function

          integer(c_int) function impz_bunch_destroy(bunch) bind(C, name="impz_bunch_destroy")
            import :: c_int, c_ptr
            type(c_ptr), value :: bunch
          end function

          integer(c_int) function impz_map_half(bunch, elem, zedge, z, tau, nst, ihlf) &
              bind(C, name="impz_map_half")
            import :: c_int, c_double, c_ptr, impz_elem_t
            type(c_ptr), value :: bunch
            type(impz_elem_t), intent(in) :: elem
            real(c_double), value :: zedge, tau
            real(c_double), intent(inout) :: z
            integer(c_int), value :: nst
            integer(c_int), intent(inout) :: ihlf
          end function

          integer(c_int) function impz_bend_entry(bunch, elem) bind(C, name="impz_bend_entry")
            import :: c_int, c_ptr, impz_elem_t
            type(c_ptr), value :: bunch
            type(impz_elem_t), intent(in) :: elem
          end function

          integer(c_int) function impz_bend_sector(bunch, z, tau) &
              bind(C, name="impz_bend_sector")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: bunch
            real(c_double), intent(inout) :: z
            real(c_double), value :: tau
          end function

          integer(c_int) function impz_bend_exit(bunch) bind(C, name="impz_bend_exit")
            import :: c_int, c_ptr
            type(c_ptr), value :: bunch
          end function

          integer(c_int) function impz_sc_prepare(bunch, piperad, piperad2, nptot, ptrange, &
              range, msize) bind(C, name="impz_sc_prepare")
            import :: c_int, c_long_long, c_double, c_ptr
            type(c_ptr), value :: bunch
            real(c_double), value :: piperad, piperad2
            integer(c_long_long), intent(out) :: nptot
            real(c_double), intent(out) :: ptrange(6), range(6), msize(3)
          end function

          integer(c_int) function impz_deposit(bunch, chgdens, counts) &
              bind(C, name="impz_deposit")
            import :: c_int, c_ptr
            type(c_ptr), value :: bunch
            type(c_ptr), value :: chgdens   ! c_loc(chgdens) or c_null_ptr
            type(c_ptr), value :: counts    ! c_loc(counts) or c_null_ptr
          end function

          integer(c_int) function impz_poisson_open(bunch, phi) &
              bind(C, name="impz_poisson_open")
            import :: c_int, c_ptr
            type(c_ptr), value :: bunch
            type(c_ptr), value :: phi       ! c_loc(Potential%FieldQ) or c_null_ptr
          end function

          integer(c_int) function impz_kick(bunch, tau, egrid) bind(C, name="impz_kick")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: bunch
            real(c_double), value :: tau
            type(c_ptr), value :: egrid
          end function

          ! the Lorentz integrator's half step (drift2_BeamBunch) and kick
          ! (kick2_BeamBunch) for Flagmap=2 call sites
          integer(c_int) function impz_drift2(bunch, z, tau) bind(C, name="impz_drift2")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: bunch
            real(c_double), intent(inout) :: z
            real(c_double), value :: tau
          end function

          integer(c_int) function impz_kick2(bunch, elem, zedge, z, tau, egrid) &
              bind(C, name="impz_kick2")
            import :: c_int, c_double, c_ptr, impz_elem_t
            type(c_ptr), value :: bunch
            type(impz_elem_t), intent(in) :: elem
            real(c_double), value :: zedge, z, tau
            type(c_ptr), value :: egrid
          end function

          integer(c_int) function impz_moments(bunch, rec) bind(C, name="impz_moments")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: bunch
            real(c_double), intent(out) :: rec(48)
          end function

          integer(c_int) function impz_diag_row(z, rec, refptcl, mass, freq, row) &
              bind(C, name="impz_diag_row")
            import :: c_int, c_double
            real(c_double), value :: z, mass, freq
            real(c_double), intent(in) :: rec(48), refptcl(6)
            real(c_double), intent(out) :: row(45)
          end function

          integer(c_int) function impz_run(bunch, elems, nelem, recs, zs, maxrec, nrec) &
              bind(C, name="impz_run")
            import :: c_int, c_double, c_ptr, impz_elem_t
            type(c_ptr), value :: bunch
            type(impz_elem_t), intent(in) :: elems(*)
            integer(c_int), value :: nelem, maxrec
            real(c_double), intent(out) :: recs(48, *), zs(*)
            integer(c_int), intent(out) :: nrec
          end function

          ! read-in wakefield of a type -41 element: table(4, ntab) holds
          ! the rows (z, Ez, Ex, Ey wake) that read1wk_Data read
          integer(c_int) function impz_wake_set(bunch, table, ntab, scale, transverse) &
              bind(C, name="impz_wake_set")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: bunch
            real(c_double), intent(in) :: table(4, *)
            integer(c_int), value :: ntab, transverse
            real(c_double), value :: scale
          end function

          integer(c_int) function impz_wake_off(bunch) bind(C, name="impz_wake_off")
            import :: c_int, c_ptr
            type(c_ptr), value :: bunch
          end function

          ! ---- library: the strings are NUL-terminated C strings
          ! (c_f_pointer onto a character(kind=c_char) array to print them)
          type(c_ptr) function impz_version() bind(C, name="impz_version")
            import :: c_ptr
          end function

          type(c_ptr) function impz_error_string(code) bind(C, name="impz_error_string")
            import :: c_int, c_ptr
            integer(c_int), value :: code
          end function

          type(c_ptr) function impz_last_cuda_error() bind(C, name="impz_last_cuda_error")
            import :: c_ptr
          end function

          ! ---- deck-level switches and bunch state between runs
          ! Flagmap of the deck or of a -25 element (1 map, 2 Lorentz)
          integer(c_int) function impz_set_integrator(bunch, flagmap) &
              bind(C, name="impz_set_integrator")
            import :: c_int, c_ptr
            type(c_ptr), value :: bunch
            integer(c_int), value :: flagmap
          end function

          ! laser heater of a -52 element: Param(2), Param(3), Param(4)
          integer(c_int) function impz_laser_heater(bunch, rsig, wavelength, ez) &
              bind(C, name="impz_laser_heater")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: bunch
            real(c_double), value :: rsig, wavelength, ez
          end function

          ! Current, Npt, Nptlocal, refptcl(1..6), z, device bytes
          integer(c_int) function impz_bunch_info(bunch, info) bind(C, name="impz_bunch_info")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: bunch
            real(c_double), intent(out) :: info(11)
          end function

          ! range and msize of the last space-charge step, as outpoint_Output writes
          integer(c_int) function impz_bunch_geom(bunch, range, msize) &
              bind(C, name="impz_bunch_geom")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: bunch
            real(c_double), intent(out) :: range(6), msize(3)
          end function

          ! z of a restart from a checkpoint (inpoint_Output)
          integer(c_int) function impz_bunch_set_z(bunch, z) bind(C, name="impz_bunch_set_z")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: bunch
            real(c_double), value :: z
          end function

          integer(c_int) function impz_bunch_upload(bunch, pts, n, current, refptcl) &
              bind(C, name="impz_bunch_upload")
            import :: c_int, c_long_long, c_double, c_ptr
            type(c_ptr), value :: bunch
            real(c_double), intent(in) :: pts(9, *)
            integer(c_long_long), value :: n
            real(c_double), value :: current
            real(c_double), intent(in) :: refptcl(6)
          end function

          integer(c_long_long) function impz_bunch_footprint(n, nx, ny, nz, form, flags, &
              nsteps) bind(C, name="impz_bunch_footprint")
            import :: c_int, c_long_long
            integer(c_long_long), value :: n
            integer(c_int), value :: nx, ny, nz, form, flags, nsteps
          end function

          ! the bunch's cudaStream_t
          type(c_ptr) function impz_bunch_stream(bunch) bind(C, name="impz_bunch_stream")
            import :: c_ptr
            type(c_ptr), value :: bunch
          end function

          integer(c_int) function impz_bunching(bunch, wavenumber, out) &
              bind(C, name="impz_bunching")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: bunch
            real(c_double), value :: wavenumber
            real(c_double), intent(out) :: out(2)
          end function

          ! ---- whole-lattice runner: records and refptcl per record
          integer(c_int) function impz_run_reference(bunch, refrec, maxrec, nrec) &
              bind(C, name="impz_run_reference")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: bunch
            real(c_double), intent(out) :: refrec(6, *)
            integer(c_int), value :: maxrec
            integer(c_int), intent(out) :: nrec
          end function

          ! the bunch's species (Pts1 rows 7 and 8 of each), their number returned
          integer(c_int) function impz_bunch_species(bunch, qm, weight, cap) &
              bind(C, name="impz_bunch_species")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: bunch
            real(c_double), intent(out) :: qm(*), weight(*)
            integer(c_int), value :: cap
          end function

          ! chgupdate_BeamBunch (BeamBunch.f90:688-728)
          integer(c_int) function impz_chgupdate(bunch, nchge, qmcclist, idchg) &
              bind(C, name="impz_chgupdate")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: bunch
            integer(c_int), value :: nchge
            real(c_double), intent(in) :: qmcclist(*)
            integer(c_int), intent(out) :: idchg(*)
          end function

          ! per-record counts of each species of the last impz_run
          integer(c_int) function impz_run_species(bunch, counts, maxrec, nrec) &
              bind(C, name="impz_run_species")
            import :: c_int, c_ptr
            type(c_ptr), value :: bunch
            integer(c_int), intent(out) :: counts(*)
            integer(c_int), value :: maxrec
            integer(c_int), intent(out) :: nrec
          end function

          integer(c_int) function impz_count_steps(elems, nelem) &
              bind(C, name="impz_count_steps")
            import :: c_int, impz_elem_t
            type(impz_elem_t), intent(in) :: elems(*)
            integer(c_int), value :: nelem
          end function

          integer(c_int) function impz_run_async(bunch, elems, nelem) &
              bind(C, name="impz_run_async")
            import :: c_int, c_ptr, impz_elem_t
            type(c_ptr), value :: bunch
            type(impz_elem_t), intent(in) :: elems(*)
            integer(c_int), value :: nelem
          end function

          integer(c_int) function impz_run_fetch(bunch, recs, zs, maxrec, nrec) &
              bind(C, name="impz_run_fetch")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: bunch
            real(c_double), intent(out) :: recs(48, *), zs(*)
            integer(c_int), value :: maxrec
            integer(c_int), intent(out) :: nrec
          end function

          integer(c_int) function impz_run_begin(bunch, elems, nelem) &
              bind(C, name="impz_run_begin")
            import :: c_int, c_ptr, impz_elem_t
            type(c_ptr), value :: bunch
            type(impz_elem_t), intent(in) :: elems(*)
            integer(c_int), value :: nelem
          end function

          integer(c_int) function impz_run_advance(bunch, budget, remaining) &
              bind(C, name="impz_run_advance")
            import :: c_int, c_ptr
            type(c_ptr), value :: bunch
            integer(c_int), value :: budget
            integer(c_int), intent(out) :: remaining
          end function

          ! launch shapes for this bunch: out = deposit blocks, push blocks,
          ! z lines per block, ms per step
          integer(c_int) function impz_autotune(bunch, nsteps, out) &
              bind(C, name="impz_autotune")
            import :: c_int, c_double, c_ptr
            type(c_ptr), value :: bunch
            integer(c_int), value :: nsteps
            real(c_double), intent(out) :: out(4)
          end function

          ! host RK6 linear map of one element (maplinear_*)
          integer(c_int) function impz_maplinear(elem, zedge, t, tau, refpt, charge, mass, &
              freq, xm) bind(C, name="impz_maplinear")
            import :: c_int, c_double, impz_elem_t
            type(impz_elem_t), intent(in) :: elem
            real(c_double), value :: zedge, t, tau, charge, mass, freq
            real(c_double), intent(inout) :: refpt(6)
            real(c_double), intent(out) :: xm(6, 6)
          end function

          ! bytes per step of the step table a run uploads
          integer(c_int) function impz_step_params_size() &
              bind(C, name="impz_step_params_size")
            import :: c_int
          end function

          ! ---- instrumentation
          integer(c_int) function impz_profile_enable(bunch, on) &
              bind(C, name="impz_profile_enable")
            import :: c_int, c_ptr
            type(c_ptr), value :: bunch
            integer(c_int), value :: on
          end function

          integer(c_int) function impz_profile_fetch(bunch, ms, launches) &
              bind(C, name="impz_profile_fetch")
            import :: c_int, c_long_long, c_double, c_ptr
            type(c_ptr), value :: bunch
            real(c_double), intent(out) :: ms(7)
            integer(c_long_long), intent(out) :: launches(7)
          end function

          integer(c_long_long) function impz_kernel_launches() &
              bind(C, name="impz_kernel_launches")
            import :: c_long_long
          end function

          ! ---- deposit into caller-owned device memory (no allocation):
          ! x..pt and chgdens are device addresses, stream a cudaStream_t
          integer(c_int) function impz_deposit_static(x, px, y, py, ph, pt, n, gam, piperad, &
              piperad2, freq, weight, range, nx, ny, nz, chgdens, stream) &
              bind(C, name="impz_deposit_static")
            import :: c_int, c_long_long, c_double, c_ptr
            type(c_ptr), value :: x, px, y, py, ph, pt
            integer(c_long_long), value :: n
            real(c_double), value :: gam, piperad, piperad2, freq, weight
            real(c_double), intent(in) :: range(6)
            integer(c_int), value :: nx, ny, nz
            type(c_ptr), value :: chgdens, stream
          end function
        end interface
      end module impz_iface
