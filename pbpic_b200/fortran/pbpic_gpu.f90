!******************************************************************************
! pbpic_gpu: Fortran 2003 ISO_C_BINDING interface to the C ABI of the B200
! step (include/pbpic.h). It lets the reference's time loop
! (src/programs/pic2d.f90:171-188) call the GPU step in place of its own
! subroutines:
!
!     call pusher        ->  ierr = pbpic_push(h)          (pic2d.f90:177)
!     call fieldsolver   ->  ierr = pbpic_fieldsolve(h)    (pic2d.f90:178)
!     call countingsort  ->  ierr = pbpic_sort(h)          (pic2d.f90:161, 181)
!
! The reference's `type particle` (pic2d.f90:47-50) has no bind(c) or sequence
! attribute, so its layout is compiler-defined; c_particle below is the
! interoperable record (5 x real(c_float), 3 x integer(c_int32_t), 32 bytes)
! that pbpic_load_particles_f32 / pbpic_store_particles_f32 exchange. Copy
! ptl(1:nptlact) into an array of c_particle before loading.
!
! Not compiled in the build environment of this repository (it has no Fortran
! compiler). It declares every single-handle function of include/pbpic.h that
! a Fortran time loop uses, with the header's argument order and types; the
! batched, differentiable and slab-band entry points (C and Python callers)
! are left out.
!******************************************************************************
module pbpic_gpu
    use iso_c_binding
    implicit none

    integer(c_int), parameter :: PBPIC_OK = 0
    integer(c_int32_t), parameter :: PBPIC_BC_PERIODIC = 0, PBPIC_BC_CONDUCTING = 1
    integer(c_int32_t), parameter :: PBPIC_FP64_PLAIN = 0, PBPIC_FP32_MIXED = 1
    integer(c_int32_t), parameter :: PBPIC_COMPAT_BORIS = 1, PBPIC_COMPAT_FOLD = 2, PBPIC_COMPAT_RHO = 4
    integer(c_int32_t), parameter :: PBPIC_OPT_NO_AUTOSORT = 1, PBPIC_OPT_EXACT_FP64 = 2
    integer(c_int32_t), parameter :: PBPIC_FILTER_MARDER = 1, PBPIC_FILTER_CERENKOV = 2
    integer(c_int32_t), parameter :: PBPIC_LOAD_UNIFORM = 0, PBPIC_LOAD_HARRIS = 1, PBPIC_LOAD_TWO_STREAM = 2, &
                                     PBPIC_LOAD_WEIBEL = 3, PBPIC_LOAD_DOUBLE_HARRIS = 4

    type, bind(c) :: pbpic_config
        integer(c_int32_t) :: mx, my
        real(c_double) :: dx, dy, dt, cva, mime, in0
        integer(c_int32_t) :: ybc, precision, compat, track_pid
        integer(c_int64_t) :: capacity
        integer(c_int32_t) :: tile_rows, options
    end type

    type, bind(c) :: c_particle
        real(c_float) :: dx, dy, ux, uy, uz
        integer(c_int32_t) :: grid, q, pid
    end type

    ! pbpic_particle_f64: the double-precision twin (56 bytes)
    type, bind(c) :: c_particle_f64
        real(c_double) :: dx, dy, ux, uy, uz
        integer(c_int32_t) :: grid, q, pid, pad
    end type

    ! pbpic_loader: the seeded plasma loaders (kind PBPIC_LOAD_DOUBLE_HARRIS is the
    ! reference's initparticles / initfields, pic2d.f90:357-648); seed is unsigned in C
    type, bind(c) :: pbpic_loader
        integer(c_int32_t) :: kind, ppc
        real(c_double) :: vthe, vthi, vdrift_e, vdrift_i, lambda, nb, psi0, bguide, b0z, anisotropy
        integer(c_int64_t) :: seed
        integer(c_int32_t) :: immobile_ions, reserved
        real(c_double) :: vthe_bg, vthi_bg
    end type

    interface
        function pbpic_create(cfg, h) bind(c, name="pbpic_create") result(ierr)
            import :: c_int, c_ptr, pbpic_config
            type(pbpic_config), intent(in) :: cfg
            type(c_ptr), intent(out) :: h
            integer(c_int) :: ierr
        end function
        function pbpic_destroy(h) bind(c, name="pbpic_destroy") result(ierr)
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int) :: ierr
        end function
        function pbpic_load_particles_f32(h, p, n) bind(c, name="pbpic_load_particles_f32") result(ierr)
            import :: c_int, c_ptr, c_int64_t, c_particle
            type(c_ptr), value :: h
            type(c_particle), intent(in) :: p(*)
            integer(c_int64_t), value :: n
            integer(c_int) :: ierr
        end function
        function pbpic_store_particles_f32(h, p, cap, n) bind(c, name="pbpic_store_particles_f32") result(ierr)
            import :: c_int, c_ptr, c_int64_t, c_particle
            type(c_ptr), value :: h
            type(c_particle), intent(out) :: p(*)
            integer(c_int64_t), value :: cap
            integer(c_int64_t), intent(out) :: n
            integer(c_int) :: ierr
        end function
        function pbpic_load_fields_f64(h, yee6) bind(c, name="pbpic_load_fields_f64") result(ierr)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: yee6(*)
            integer(c_int) :: ierr
        end function
        function pbpic_store_fields_f64(h, yee6) bind(c, name="pbpic_store_fields_f64") result(ierr)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: yee6(*)
            integer(c_int) :: ierr
        end function
        function pbpic_push(h) bind(c, name="pbpic_push") result(ierr)
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int) :: ierr
        end function
        function pbpic_fieldsolve(h) bind(c, name="pbpic_fieldsolve") result(ierr)
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int) :: ierr
        end function
        function pbpic_sort(h) bind(c, name="pbpic_sort") result(ierr)
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int) :: ierr
        end function
        function pbpic_step(h, nsteps, sort_every) bind(c, name="pbpic_step") result(ierr)
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value :: h
            integer(c_int32_t), value :: nsteps, sort_every
            integer(c_int) :: ierr
        end function
        function pbpic_energies(h, e) bind(c, name="pbpic_energies") result(ierr)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: e(4)
            integer(c_int) :: ierr
        end function
        function pbpic_cell_counts(h, counts) bind(c, name="pbpic_cell_counts") result(ierr)
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value :: h
            integer(c_int32_t), intent(out) :: counts(*)
            integer(c_int) :: ierr
        end function
        function pbpic_status(h, bits) bind(c, name="pbpic_status") result(ierr)
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value :: h
            integer(c_int32_t), intent(out) :: bits
            integer(c_int) :: ierr
        end function
        function pbpic_gauss_residual(h, r) bind(c, name="pbpic_gauss_residual") result(ierr)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: r
            integer(c_int) :: ierr
        end function
        function pbpic_energy_history(h, out, max_rows, n_rows) bind(c, name="pbpic_energy_history") result(ierr)
            import :: c_int, c_ptr, c_double, c_int32_t
            type(c_ptr), value :: h
            real(c_double), intent(out) :: out(*)
            integer(c_int32_t), value :: max_rows
            integer(c_int32_t), intent(out) :: n_rows
            integer(c_int) :: ierr
        end function
        ! fieldsinfo / particlesinfo: dir is a NUL-terminated character array
        function pbpic_dump(h, dir) bind(c, name="pbpic_dump") result(ierr)
            import :: c_int, c_ptr, c_char
            type(c_ptr), value :: h
            character(kind=c_char), intent(in) :: dir(*)
            integer(c_int) :: ierr
        end function
        ! the reference's own HDF5 files: particles.h5, fields%05d.h5, spectra.h5, energy_tot.h5
        function pbpic_dump_h5(h, dir, de_electron, de_ion, nbins) bind(c, name="pbpic_dump_h5") result(ierr)
            import :: c_int, c_ptr, c_char, c_double, c_int32_t
            type(c_ptr), value :: h
            character(kind=c_char), intent(in) :: dir(*)
            real(c_double), value :: de_electron, de_ion
            integer(c_int32_t), value :: nbins
            integer(c_int) :: ierr
        end function
        function pbpic_restart(h, dir) bind(c, name="pbpic_restart") result(ierr)
            import :: c_int, c_ptr, c_char
            type(c_ptr), value :: h
            character(kind=c_char), intent(in) :: dir(*)
            integer(c_int) :: ierr
        end function
        ! divergenceclean / suppresscerenkov (pic2d.f90:867-907)
        function pbpic_set_field_filters(h, flags, marder_d, cerenkov_tau) &
                bind(c, name="pbpic_set_field_filters") result(ierr)
            import :: c_int, c_ptr, c_int32_t, c_double
            type(c_ptr), value :: h
            integer(c_int32_t), value :: flags
            real(c_double), value :: marder_d, cerenkov_tau
            integer(c_int) :: ierr
        end function
        ! energyspectra (pic2d.f90:1957-1990): counts(nbins, 2) in Fortran order
        function pbpic_energy_spectra(h, de_electron, de_ion, nbins, counts) &
                bind(c, name="pbpic_energy_spectra") result(ierr)
            import :: c_int, c_ptr, c_int32_t, c_int64_t, c_double
            type(c_ptr), value :: h
            real(c_double), value :: de_electron, de_ion
            integer(c_int32_t), value :: nbins
            integer(c_int64_t), intent(out) :: counts(*)
            integer(c_int) :: ierr
        end function
        function pbpic_set_stream(h, stream) bind(c, name="pbpic_set_stream") result(ierr)
            import :: c_int, c_ptr
            type(c_ptr), value :: h, stream
            integer(c_int) :: ierr
        end function
        function pbpic_synchronize(h) bind(c, name="pbpic_synchronize") result(ierr)
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int) :: ierr
        end function
        function pbpic_init_plasma(h, ld) bind(c, name="pbpic_init_plasma") result(ierr)
            import :: c_int, c_ptr, pbpic_loader
            type(c_ptr), value :: h
            type(pbpic_loader), intent(in) :: ld
            integer(c_int) :: ierr
        end function
        function pbpic_loader_count(h, ld, n) bind(c, name="pbpic_loader_count") result(ierr)
            import :: c_int, c_ptr, c_int64_t, pbpic_loader
            type(c_ptr), value :: h
            type(pbpic_loader), intent(in) :: ld
            integer(c_int64_t), intent(out) :: n
            integer(c_int) :: ierr
        end function
        function pbpic_num_particles(h, n) bind(c, name="pbpic_num_particles") result(ierr)
            import :: c_int, c_ptr, c_int64_t
            type(c_ptr), value :: h
            integer(c_int64_t), intent(out) :: n
            integer(c_int) :: ierr
        end function
        function pbpic_load_particles_f64(h, p, n) bind(c, name="pbpic_load_particles_f64") result(ierr)
            import :: c_int, c_ptr, c_int64_t, c_particle_f64
            type(c_ptr), value :: h
            type(c_particle_f64), intent(in) :: p(*)
            integer(c_int64_t), value :: n
            integer(c_int) :: ierr
        end function
        function pbpic_store_particles_f64(h, p, cap, n) bind(c, name="pbpic_store_particles_f64") result(ierr)
            import :: c_int, c_ptr, c_int64_t, c_particle_f64
            type(c_ptr), value :: h
            type(c_particle_f64), intent(out) :: p(*)
            integer(c_int64_t), value :: cap
            integer(c_int64_t), intent(out) :: n
            integer(c_int) :: ierr
        end function
        ! emfgrid (pic2d.f90:72): (mx+1) x (my+1) nodes of 8 values; the record varies
        ! fastest, then y, then x
        function pbpic_store_emfgrid_f64(h, grid8) bind(c, name="pbpic_store_emfgrid_f64") result(ierr)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: grid8(*)
            integer(c_int) :: ierr
        end function
        ! denjr (pic2d.f90:73): jx, jy, jz, rho as 4 planes of mx x (my+1)
        function pbpic_store_denjr_f64(h, j4) bind(c, name="pbpic_store_denjr_f64") result(ierr)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: j4(*)
            integer(c_int) :: ierr
        end function
        function pbpic_reconnected_flux(h, flux) bind(c, name="pbpic_reconnected_flux") result(ierr)
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: flux
            integer(c_int) :: ierr
        end function
        ! energies and Gauss residual of the rows [y_lo, y_hi) of one y slab
        function pbpic_energies_rows(h, y_lo, y_hi, wall_lo, wall_hi, e) &
                bind(c, name="pbpic_energies_rows") result(ierr)
            import :: c_int, c_ptr, c_int32_t, c_double
            type(c_ptr), value :: h
            integer(c_int32_t), value :: y_lo, y_hi, wall_lo, wall_hi
            real(c_double), intent(out) :: e(4)
            integer(c_int) :: ierr
        end function
        function pbpic_gauss_residual_rows(h, y_lo, y_hi, r) bind(c, name="pbpic_gauss_residual_rows") result(ierr)
            import :: c_int, c_ptr, c_int32_t, c_double
            type(c_ptr), value :: h
            integer(c_int32_t), value :: y_lo, y_hi
            real(c_double), intent(out) :: r
            integer(c_int) :: ierr
        end function
        function pbpic_get_config(h, cfg) bind(c, name="pbpic_get_config") result(ierr)
            import :: c_int, c_ptr, pbpic_config
            type(c_ptr), value :: h
            type(pbpic_config), intent(out) :: cfg
            integer(c_int) :: ierr
        end function
        ! dispersioninfo (pic2d.f90:2124-2142): node values along node rows rows(1:nrows)
        ! and node columns cols(1:ncols), 0-based indices; out holds nrows*mx*6 then
        ! ncols*my*6 values, the 6 components varying fastest
        function pbpic_field_cuts(h, rows, nrows, cols, ncols, out) bind(c, name="pbpic_field_cuts") result(ierr)
            import :: c_int, c_ptr, c_int32_t, c_double
            type(c_ptr), value :: h
            integer(c_int32_t), intent(in) :: rows(*), cols(*)
            integer(c_int32_t), value :: nrows, ncols
            real(c_double), intent(out) :: out(*)
            integer(c_int) :: ierr
        end function
        function pbpic_last_error() bind(c, name="pbpic_last_error") result(msg)
            import :: c_ptr
            type(c_ptr) :: msg
        end function
    end interface
end module pbpic_gpu
