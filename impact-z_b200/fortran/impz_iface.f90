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
        end interface
      end module impz_iface
