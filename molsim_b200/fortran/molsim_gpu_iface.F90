! molsim_gpu_iface.F90 -- Fortran 2003 ISO_C_BINDING interface to libmolsim_gpu.so
!
! Binds the C-ABI of include/molsim_gpu.h for MOLSIM's Fortran host, the same
! way MOLSIM binds FFTW (use, intrinsic :: iso_c_binding; Src/energy.F90:100-110).
! Fortran (3,N) real(8) arrays are passed as they are (column-major (3,N) is
! C [N][3]); type, table and neighbour indices keep MOLSIM's 1-based values.
!
! Build: gfortran -c molsim_gpu_iface.F90, link molsim_ser with
!        -L<dir> -lmolsim_gpu -Wl,-rpath,<dir>
! This file was not compiled in this repository's build (no Fortran compiler
! in the build image); the C side it binds is tested through the same
! entry points from Python.

module MolsimGpu

   use, intrinsic :: iso_c_binding
   implicit none

   integer(c_int32_t), parameter :: MSG_OK = 0, MSG_ERR_TABLE_MIN = 1, MSG_ERR_TABLE_RANGE = 2, &
                                    MSG_ERR_CAPACITY = 3, MSG_ERR_CUDA = 4, MSG_ERR_TIMEOUT = 5, &
                                    MSG_ERR_ARG = 6, MSG_ERR_NONFINITE = 7, MSG_ERR_HARDCORE = 8
   integer(c_int32_t), parameter :: MSG_PREC_FP64 = 0, MSG_PREC_MIXED = 1

   ! struct msg_params (field order and types as in molsim_gpu.h)
   type, bind(c) :: msg_params
      integer(c_int32_t) :: np, npt
      real(c_double)     :: boxlen(3)
      real(c_double)     :: rcut, drnlist
      type(c_ptr)        :: iptpn, az, masspt, ubuf
      integer(c_int32_t) :: nbuf
      type(c_ptr)        :: iubuflow, r2umin, r2atat
      integer(c_int32_t) :: lewald, order, nmesh, lsurf
      real(c_double)     :: ualpha, epsi_four_pi
      integer(c_int32_t) :: nbond
      type(c_ptr)        :: bond_ij, bond_k, bond_eq, bond_p
      real(c_double)     :: tstep
      type(c_ptr)        :: bd_fac1, bd_fac2
      integer(c_int32_t) :: maxnneigh
      integer(c_int32_t) :: ncut, ncutregion
      integer(c_int32_t) :: lewald2dlc
      integer(c_int32_t) :: inlist
      integer(c_int32_t) :: lvlistllist
   end type msg_params

   ! struct msg_energy
   type, bind(c) :: msg_energy
      real(c_double) :: utot, utwob0, utwob(10), urec, ubond, virial, ekin
   end type msg_energy

   ! struct msg_mc_params
   type, bind(c) :: msg_mc_params
      real(c_double)     :: beta                 ! MOLSIM's beta
      type(c_ptr)        :: dtran                ! c_loc(dtran(1:npt))
      integer(c_int32_t) :: isamp, pad
   end type msg_mc_params

   ! struct msg_mcall_params
   ! struct msg_tab_params (msg_pot_tab)
   type, bind(c) :: msg_tab_params
      integer(c_int32_t) :: npt
      type(c_ptr)        :: zat, sigat, epsat   ! [npt]
      real(c_double)     :: rcut, ualpha, epsi_four_pi
      integer(c_int32_t) :: lewald, lljcut
      real(c_double)     :: ljrcut, ljushift
      real(c_double)     :: r2uminin, utoltab, ftoltab, umaxtab, fmaxtab, rumaxfac
   end type msg_tab_params

   type, bind(c) :: msg_mcall_params
      real(c_double)     :: beta
      type(c_ptr)        :: dtranall              ! c_loc(dtranall(1:npt))
   end type msg_mcall_params

   ! struct msg_site_ewald
   type, bind(c) :: msg_site_ewald
      integer(c_int32_t) :: lewald               ! 1: 'spm', 2: 'std'
      integer(c_int32_t) :: order, nmesh         ! SPME
      integer(c_int32_t) :: ncut, ncutregion     ! standard Ewald (0 sphere, 1 cube)
      integer(c_int32_t) :: lsurf
      real(c_double)     :: ualpha, epsi_four_pi
      type(c_ptr)        :: az                   ! c_loc(az(1:na))
   end type msg_site_ewald

   interface
      integer(c_int) function msg_create(p, precision, h) bind(c, name='msg_create')
         import :: c_int, c_int32_t, c_ptr, msg_params
         type(msg_params), intent(in)         :: p
         integer(c_int32_t), value            :: precision
         type(c_ptr), intent(out)             :: h
      end function msg_create

      subroutine msg_destroy(h) bind(c, name='msg_destroy')
         import :: c_ptr
         type(c_ptr), value :: h
      end subroutine msg_destroy

      type(c_ptr) function msg_last_error(h) bind(c, name='msg_last_error')
         import :: c_ptr
         type(c_ptr), value :: h
      end function msg_last_error

      integer(c_int) function msg_nlist_before_macrostep(h) bind(c, name='msg_nlist_before_macrostep')
         import :: c_int, c_ptr
         type(c_ptr), value        :: h
      end function msg_nlist_before_macrostep

      integer(c_int) function msg_set_state(h, isys, ro, rod, rodd) bind(c, name='msg_set_state')
         import :: c_int, c_int32_t, c_ptr
         type(c_ptr), value        :: h
         integer(c_int32_t), value :: isys
         type(c_ptr), value        :: ro, rod, rodd
      end function msg_set_state

      integer(c_int) function msg_get_state(h, isys, ro, rod, rodd) bind(c, name='msg_get_state')
         import :: c_int, c_int32_t, c_ptr
         type(c_ptr), value        :: h
         integer(c_int32_t), value :: isys
         type(c_ptr), value        :: ro, rod, rodd
      end function msg_get_state

      integer(c_int) function msg_build_nlist(h, isys, nneighpn, jpnlist, maxnneigh, npair) &
            bind(c, name='msg_build_nlist')
         import :: c_int, c_int32_t, c_int64_t, c_ptr
         type(c_ptr), value        :: h
         integer(c_int32_t), value :: isys
         type(c_ptr), value        :: nneighpn, jpnlist
         integer(c_int32_t), value :: maxnneigh
         integer(c_int64_t), intent(out) :: npair
      end function msg_build_nlist

      integer(c_int) function msg_utotal(h, isys, force, forceo, e) bind(c, name='msg_utotal')
         import :: c_int, c_int32_t, c_ptr, msg_energy
         type(c_ptr), value        :: h
         integer(c_int32_t), value :: isys
         type(c_ptr), value        :: force, forceo
         type(msg_energy), intent(out) :: e
      end function msg_utotal

      integer(c_int) function msg_get_linacc(h) bind(c, name='msg_get_linacc')
         import :: c_int, c_ptr
         type(c_ptr), value :: h
      end function msg_get_linacc

      integer(c_int) function msg_velver(h, nsteps, isys, e) bind(c, name='msg_velver')
         import :: c_int, c_int32_t, c_ptr
         type(c_ptr), value        :: h
         integer(c_int32_t), value :: nsteps, isys
         type(c_ptr), value        :: e          ! msg_energy(nsteps) or c_null_ptr
      end function msg_velver

      integer(c_int) function msg_velver_host(h, isys, nsteps, ro, rod, rodd, e) bind(c, name='msg_velver_host')
         import :: c_int, c_int32_t, c_ptr
         type(c_ptr), value        :: h
         integer(c_int32_t), value :: isys, nsteps
         type(c_ptr), value        :: ro, rod, rodd, e   ! (3,np) real(8) each; e: msg_energy(nsteps) or c_null_ptr
      end function msg_velver_host

      integer(c_int) function msg_utwobody_p(np, na, npt, nat, boxlen, rcut, ro, r, iptpn, ianpn, napt, iatan, &
            nneighpn, jpnlist, maxnneigh, ubuf, nbuf, iubuflow, r2umin, force, utwob, virial, kernel_ms) &
            bind(c, name='msg_utwobody_p')
         import :: c_int, c_int32_t, c_double, c_ptr
         integer(c_int32_t), value :: np, na, npt, nat
         real(c_double), intent(in) :: boxlen(3)
         real(c_double), value     :: rcut
         type(c_ptr), value        :: ro, r, iptpn, ianpn, napt, iatan, nneighpn, jpnlist
         integer(c_int32_t), value :: maxnneigh
         type(c_ptr), value        :: ubuf
         integer(c_int32_t), value :: nbuf
         type(c_ptr), value        :: iubuflow, r2umin, force, utwob, virial, kernel_ms
      end function msg_utwobody_p

      integer(c_int) function msg_velver_p(nsteps, np, na, npt, nat, boxlen, rcut, tstep, nvvite, tvvite, ro, rod, &
            rodd, qua, quad, quadd, r, iptpn, ianpn, napt, iatan, ra, maxsite, masspt, momp, nneighpn, jpnlist, &
            maxnneigh, ubuf, nbuf, iubuflow, r2umin, utwob, virial, kernel_ms) bind(c, name='msg_velver_p')
         import :: c_int, c_int32_t, c_double, c_ptr
         integer(c_int32_t), value :: nsteps, np, na, npt, nat
         real(c_double), intent(in) :: boxlen(3)
         real(c_double), value     :: rcut, tstep
         integer(c_int32_t), value :: nvvite
         real(c_double), value     :: tvvite
         type(c_ptr), value        :: ro, rod, rodd, qua, quad, quadd, r, iptpn, ianpn, napt, iatan, ra
         integer(c_int32_t), value :: maxsite
         type(c_ptr), value        :: masspt, momp, nneighpn, jpnlist
         integer(c_int32_t), value :: maxnneigh
         type(c_ptr), value        :: ubuf
         integer(c_int32_t), value :: nbuf
         type(c_ptr), value        :: iubuflow, r2umin, utwob, virial, kernel_ms
      end function msg_velver_p

      integer(c_int) function msg_velver_p_ewald(nsteps, np, na, npt, nat, boxlen, rcut, tstep, nvvite, tvvite, &
            ro, rod, rodd, qua, quad, quadd, r, iptpn, ianpn, napt, iatan, ra, maxsite, masspt, momp, nneighpn, &
            jpnlist, maxnneigh, ubuf, nbuf, iubuflow, r2umin, ew, utwob, urec, virial, kernel_ms) &
            bind(c, name='msg_velver_p_ewald')
         import :: c_int, c_int32_t, c_double, c_ptr, msg_site_ewald
         integer(c_int32_t), value :: nsteps, np, na, npt, nat
         real(c_double), intent(in) :: boxlen(3)
         real(c_double), value     :: rcut, tstep
         integer(c_int32_t), value :: nvvite
         real(c_double), value     :: tvvite
         type(c_ptr), value        :: ro, rod, rodd, qua, quad, quadd, r, iptpn, ianpn, napt, iatan, ra
         integer(c_int32_t), value :: maxsite
         type(c_ptr), value        :: masspt, momp, nneighpn, jpnlist
         integer(c_int32_t), value :: maxnneigh
         type(c_ptr), value        :: ubuf
         integer(c_int32_t), value :: nbuf
         type(c_ptr), value        :: iubuflow, r2umin
         type(msg_site_ewald), intent(in) :: ew
         type(c_ptr), value        :: utwob
         real(c_double), intent(out) :: urec, virial
         type(c_ptr), value        :: kernel_ms
      end function msg_velver_p_ewald

      integer(c_int) function msg_uewald_sites(na, boxlen, ualpha, ncut, ncutregion, lsurf, epsfp, r, az, np, &
            iptpn, ianpn, napt, npt, force, urec, virrec, kernel_ms) bind(c, name='msg_uewald_sites')
         import :: c_int, c_int32_t, c_double, c_ptr
         integer(c_int32_t), value :: na
         real(c_double), intent(in) :: boxlen(3)
         real(c_double), value     :: ualpha
         integer(c_int32_t), value :: ncut, ncutregion, lsurf
         real(c_double), value     :: epsfp
         type(c_ptr), value        :: r, az
         integer(c_int32_t), value :: np
         type(c_ptr), value        :: iptpn, ianpn, napt
         integer(c_int32_t), value :: npt
         type(c_ptr), value        :: force
         real(c_double), intent(out) :: urec, virrec
         type(c_ptr), value        :: kernel_ms
      end function msg_uewald_sites

      integer(c_int) function msg_uewald_sites_spm(na, boxlen, ualpha, order, nmesh, lsurf, epsfp, r, az, np, &
            iptpn, ianpn, napt, npt, force, urec, virrec, kernel_ms) bind(c, name='msg_uewald_sites_spm')
         import :: c_int, c_int32_t, c_double, c_ptr
         integer(c_int32_t), value :: na
         real(c_double), intent(in) :: boxlen(3)
         real(c_double), value     :: ualpha
         integer(c_int32_t), value :: order, nmesh, lsurf
         real(c_double), value     :: epsfp
         type(c_ptr), value        :: r, az
         integer(c_int32_t), value :: np
         type(c_ptr), value        :: iptpn, ianpn, napt
         integer(c_int32_t), value :: npt
         type(c_ptr), value        :: force
         real(c_double), intent(out) :: urec, virrec
         type(c_ptr), value        :: kernel_ms
      end function msg_uewald_sites_spm

      integer(c_int) function msg_mcall_pass(h, npass, p, accepted, isys, e) bind(c, name='msg_mcall_pass')
         import :: c_int, c_int32_t, c_ptr, msg_mcall_params
         type(c_ptr), value        :: h
         integer(c_int32_t), value :: npass
         type(msg_mcall_params), intent(in) :: p(*)
         type(c_ptr), value        :: accepted, e
         integer(c_int32_t), value :: isys
      end function msg_mcall_pass

      integer(c_int) function msg_random_jump(ix, iy, k, out) bind(c, name='msg_random_jump')
         import :: c_int, c_int32_t
         integer(c_int32_t), value :: ix, iy, k
         integer(c_int32_t), intent(out) :: out(2)
      end function msg_random_jump

      integer(c_int) function msg_mc_seed(h, isys, iseed) bind(c, name='msg_mc_seed')
         import :: c_int, c_int32_t, c_ptr
         type(c_ptr), value        :: h
         integer(c_int32_t), value :: isys, iseed
      end function msg_mc_seed

      integer(c_int) function msg_mc_pass(h, npass, p, accepted, hsreject, isys, e) bind(c, name='msg_mc_pass')
         import :: c_int, c_int32_t, c_ptr, msg_mc_params
         type(c_ptr), value        :: h
         integer(c_int32_t), value :: npass
         type(msg_mc_params), intent(in) :: p(*)
         type(c_ptr), value        :: accepted, hsreject, e   ! int64(nsys), int64(nsys), msg_energy, or c_null_ptr
         integer(c_int32_t), value :: isys
      end function msg_mc_pass

      integer(c_int) function msg_bd_step(h, nsteps, seed, isys, xi, xi_out, e) bind(c, name='msg_bd_step')
         import :: c_int, c_int32_t, c_int64_t, c_ptr
         type(c_ptr), value        :: h
         integer(c_int32_t), value :: nsteps
         integer(c_int64_t), value :: seed
         integer(c_int32_t), value :: isys
         type(c_ptr), value        :: xi, xi_out, e
      end function msg_bd_step

      integer(c_int) function msg_put_state(h, isys, ro, rod, rodd, keep_list) bind(c, name='msg_put_state')
         import :: c_int, c_int32_t, c_ptr
         type(c_ptr), value        :: h
         integer(c_int32_t), value :: isys
         type(c_ptr), value        :: ro, rod, rodd
         integer(c_int32_t), value :: keep_list
      end function msg_put_state

      integer(c_int64_t) function msg_nrebuild(h, isys) bind(c, name='msg_nrebuild')
         import :: c_int32_t, c_int64_t, c_ptr
         type(c_ptr), value        :: h
         integer(c_int32_t), value :: isys
      end function msg_nrebuild

      real(c_double) function msg_rcut_to_alpha(uewaldtol, q2sum, epsi_four_pi, boxlenshort, rcut, status) &
            bind(c, name='msg_rcut_to_alpha')
         import :: c_double, c_int32_t
         real(c_double), value :: uewaldtol, q2sum, epsi_four_pi, boxlenshort, rcut
         integer(c_int32_t), intent(out) :: status
      end function msg_rcut_to_alpha

      integer(c_int32_t) function msg_alpha_to_ncut(uewaldtol, q2sum, epsi_four_pi, boxlenshort, ualpha, status) &
            bind(c, name='msg_alpha_to_ncut')
         import :: c_double, c_int32_t
         real(c_double), value :: uewaldtol, q2sum, epsi_four_pi, boxlenshort, ualpha
         integer(c_int32_t), intent(out) :: status
      end function msg_alpha_to_ncut
      ! batches, serving, tuning, timing and set-up helpers

      integer(c_int) function msg_create_batch(p, nsys, precision, h) bind(c, name='msg_create_batch')
         import :: c_int, c_int32_t, c_ptr, msg_params
         type(msg_params), intent(in)         :: p(*)
         integer(c_int32_t), value            :: nsys, precision
         type(c_ptr), intent(out)             :: h
      end function msg_create_batch

      integer(c_int32_t) function msg_nsys(h) bind(c, name='msg_nsys')
         import :: c_int32_t, c_ptr
         type(c_ptr), value :: h
      end function msg_nsys

      integer(c_int) function msg_set_state_all(h, ro, rod, rodd) bind(c, name='msg_set_state_all')
         import :: c_int, c_ptr
         type(c_ptr), value :: h, ro, rod, rodd
      end function msg_set_state_all

      integer(c_int) function msg_get_forces(h, isys, force, forceo) bind(c, name='msg_get_forces')
         import :: c_int, c_int32_t, c_ptr
         type(c_ptr), value        :: h
         integer(c_int32_t), value :: isys
         type(c_ptr), value        :: force, forceo
      end function msg_get_forces

      integer(c_int) function msg_get_energy(h, isys, e) bind(c, name='msg_get_energy')
         import :: c_int, c_int32_t, c_ptr, msg_energy
         type(c_ptr), value        :: h
         integer(c_int32_t), value :: isys
         type(msg_energy), intent(out) :: e
      end function msg_get_energy

      integer(c_int) function msg_velver_async(h, nsteps) bind(c, name='msg_velver_async')
         import :: c_int, c_int32_t, c_ptr
         type(c_ptr), value        :: h
         integer(c_int32_t), value :: nsteps
      end function msg_velver_async

      integer(c_int) function msg_pending(h) bind(c, name='msg_pending')
         import :: c_int, c_ptr
         type(c_ptr), value :: h
      end function msg_pending

      integer(c_int) function msg_estimate_bytes(p, nsys, precision, bytes) bind(c, name='msg_estimate_bytes')
         import :: c_int, c_int32_t, c_int64_t, msg_params
         type(msg_params), intent(in)    :: p(*)
         integer(c_int32_t), value       :: nsys, precision
         integer(c_int64_t), intent(out) :: bytes
      end function msg_estimate_bytes

      integer(c_int64_t) function msg_device_bytes(h) bind(c, name='msg_device_bytes')
         import :: c_int64_t, c_ptr
         type(c_ptr), value :: h
      end function msg_device_bytes

      integer(c_int) function msg_trim_caches() bind(c, name='msg_trim_caches')
         import :: c_int
      end function msg_trim_caches

      type(c_ptr) function msg_stream(h) bind(c, name='msg_stream')
         import :: c_ptr
         type(c_ptr), value :: h
      end function msg_stream

      integer(c_int) function msg_tune(h, key, val) bind(c, name='msg_tune')
         import :: c_int, c_int32_t, c_ptr
         type(c_ptr), value        :: h
         integer(c_int32_t), value :: key, val
      end function msg_tune

      integer(c_int64_t) function msg_launch_count(h) bind(c, name='msg_launch_count')
         import :: c_int64_t, c_ptr
         type(c_ptr), value :: h
      end function msg_launch_count

      integer(c_int) function msg_set_timing(h, on) bind(c, name='msg_set_timing')
         import :: c_int, c_int32_t, c_ptr
         type(c_ptr), value        :: h
         integer(c_int32_t), value :: on
      end function msg_set_timing

      integer(c_int32_t) function msg_ntimers() bind(c, name='msg_ntimers')
         import :: c_int32_t
      end function msg_ntimers

      integer(c_int) function msg_kernel_time(h, k, kname, total_ms, launches) bind(c, name='msg_kernel_time')
         import :: c_int, c_int32_t, c_int64_t, c_double, c_ptr
         type(c_ptr), value              :: h
         integer(c_int32_t), value       :: k
         type(c_ptr), intent(out)        :: kname       ! const char *
         real(c_double), intent(out)     :: total_ms
         integer(c_int64_t), intent(out) :: launches
      end function msg_kernel_time

      integer(c_int) function msg_pot_tab(p, ubuf, nbuf, iubuflow, nugrid, r2umin, nused) bind(c, name='msg_pot_tab')
         import :: c_int, c_int32_t, c_ptr, msg_tab_params
         type(msg_tab_params), intent(in) :: p
         type(c_ptr), value               :: ubuf
         integer(c_int32_t), value        :: nbuf
         type(c_ptr), value               :: iubuflow, nugrid, r2umin
         integer(c_int32_t), intent(out)  :: nused
      end function msg_pot_tab

      integer(c_int) function msg_utwobody_noalloc(np, npt, boxlen, rcut, ro, iptpn, nneighpn, jpnlist, maxnneigh, &
            lmc, ubuf, nbuf, iubuflow, r2umin, r2atat, force, utwob, virial, stop_ipjp, stream) &
            bind(c, name='msg_utwobody_noalloc')
         import :: c_int, c_int32_t, c_double, c_ptr
         integer(c_int32_t), value  :: np, npt
         real(c_double), intent(in) :: boxlen(3)
         real(c_double), value      :: rcut
         type(c_ptr), value         :: ro, iptpn, nneighpn, jpnlist   ! device pointers
         integer(c_int32_t), value  :: maxnneigh, lmc
         type(c_ptr), value         :: ubuf
         integer(c_int32_t), value  :: nbuf
         type(c_ptr), value         :: iubuflow, r2umin, r2atat, force, utwob, virial
         integer(c_int32_t)         :: stop_ipjp(2)                 ! ip, jp of a nonzero status
         type(c_ptr), value         :: stream
      end function msg_utwobody_noalloc
   end interface

contains

   ! The message of the last error of handle h as a Fortran string.
   function MsgError(h) result(txt)
      type(c_ptr), intent(in) :: h
      character(len=256) :: txt
      character(kind=c_char), pointer :: s(:)
      integer :: i
      txt = ''
      call c_f_pointer(msg_last_error(h), s, [256])
      do i = 1, 256
         if (s(i) == c_null_char) exit
         txt(i:i) = s(i)
      end do
   end function MsgError

end module MolsimGpu
