!+
! Module bmadgpu_mod
!
! Fortran binding of the B200 tracker (include/bmadgpu.h) for Bmad programs. It installs a
! track1_bunch hook (bmad/custom/track1_bunch_hook.f90:25-43, pointer at
! bmad/modules/bmad_routine_interface.f90:4034, called by track1_bunch at
! bmad/multiparticle/beam_mod.f90:263-266) and offers a ring-level routine for the turn loop of
! long_term_tracking (bsim/modules/lt_tracking_mod.f90:1631-1713).
!
! Marshalling follows cpp_bmad_interface's coord_to_c / coord_to_f2 idiom
! (cpp_bmad_interface/code/bmad_cpp_convert_mod.f90:1767-1844): component by component into
! structure-of-arrays buffers, since coord_struct is not C interoperable (real(qp) time,
! allocatables).
!
! This file is compiled with the caller's Bmad build (gfortran/ifort with bmad modules on the
! include path) and linked with libbmadgpu.so; it has not been compiled in this repository
! (no Fortran compiler in the build image).
!-

module bmadgpu_mod

use bmad
use, intrinsic :: iso_c_binding

implicit none

integer, parameter :: bmadgpu_n_pole = 22

type, bind(c) :: bmadgpu_element_t
  integer(c_int32_t) :: key, is_on, fringe_type, fringe_at, aperture_at, aperture_type
  integer(c_int32_t) :: num_steps, scale_multipoles, field_master, exact_multipoles, orientation, reserved
  real(c_double) :: l, k1, k2, k3, g, dg, e1, e2, fint, fintx, hgap, hgapx
  real(c_double) :: tilt, ref_tilt, roll, x_offset, y_offset, z_offset, x_pitch, y_pitch
  real(c_double) :: hkick, vkick
  real(c_double) :: x1_limit, x2_limit, y1_limit, y2_limit
  real(c_double) :: voltage, rf_frequency, phi0, phi0_multipass
  real(c_double) :: ds_step, r0_mag, r0_elec
  real(c_double) :: delta_ref_time
  real(c_double) :: a_pole(0:bmadgpu_n_pole-1), b_pole(0:bmadgpu_n_pole-1)
  real(c_double) :: a_pole_elec(0:bmadgpu_n_pole-1), b_pole_elec(0:bmadgpu_n_pole-1)
  real(c_double) :: fq1, fq2
  real(c_double) :: px_aperture_width2, px_aperture_center, py_aperture_width2, py_aperture_center
  real(c_double) :: z_aperture_width2, z_aperture_center, pz_aperture_width2, pz_aperture_center
  real(c_double) :: kick
end type

type, bind(c) :: bmadgpu_param_t
  real(c_double) :: p0c, e_tot, mass, charge, max_aperture_limit, default_ds_step
  integer(c_int32_t) :: aperture_limit_on, absolute_time_tracking, radiation_on, reserved
end type

type, bind(c) :: bmadgpu_bunch_t
  integer(c_int64_t) :: n
  type(c_ptr) :: vec, beta, t, state, ix_ele, ix_turn, location
end type

! bmadgpu_twiss of include/bmadgpu.h (what twiss_from_mat6 fills in ele%a, ele%b, ele%x, ele%y).
type, bind(c) :: bmadgpu_twiss_t
  real(c_double) :: beta_a, alpha_a, gamma_a, phi_a, beta_b, alpha_b, gamma_b, phi_b
  real(c_double) :: eta_a, etap_a, deta_ds_a, eta_b, etap_b, deta_ds_b
  real(c_double) :: eta_x, etap_x, deta_ds_x, eta_y, etap_y, deta_ds_y
  real(c_double) :: c_mat(4), gamma_c, growth_rate, symp_error
  integer(c_int32_t) :: status, reserved
end type

! bmadgpu_ltt_params of include/bmadgpu.h: the ltt_params_struct settings that ltt_run_beam_mode
! (bsim/modules/lt_tracking_mod.f90:46-110) reads. File names are NUL-terminated C strings
! (c_loc of a character(kind=c_char) array), c_null_ptr for none.
type, bind(c) :: bmadgpu_ltt_params_t
  integer(c_int32_t) :: n_turns, averages_every_n_turns, particle_every_n_turns, output_only_last_turns
  integer(c_int32_t) :: only_live_particles_out, ix_turn_start, beam_every_n_turns, beam_exact
  real(c_double) :: dead_cutoff
  type(c_ptr) :: averages_file, phase_space_file, beam_file
  real(c_double) :: core_emit_cutoff(8)
  integer(c_int32_t) :: core_emit_per_mode
  type(c_ptr) :: action_angle_file, per_particle_file, action_angle_n_inv
end type

interface
  integer(c_int) function bmadgpu_ctx_create(device, ctx) bind(c, name='bmadgpu_ctx_create')
    import
    integer(c_int32_t), value :: device
    type(c_ptr) :: ctx
  end function
  integer(c_int) function bmadgpu_lattice_create(ctx, eles, n_ele, param, lat) bind(c, name='bmadgpu_lattice_create')
    import
    type(c_ptr), value :: ctx
    type(bmadgpu_element_t) :: eles(*)
    integer(c_int32_t), value :: n_ele
    type(bmadgpu_param_t) :: param
    type(c_ptr) :: lat
  end function
  integer(c_int) function bmadgpu_track_bunch(ctx, lat, bunch, ix_start, ix_end, turn0, n_turns, moments) &
                                                                              bind(c, name='bmadgpu_track_bunch')
    import
    type(c_ptr), value :: ctx, lat
    type(bmadgpu_bunch_t) :: bunch
    integer(c_int32_t), value :: ix_start, ix_end, turn0, n_turns
    type(c_ptr), value :: moments
  end function
  integer(c_int) function bmadgpu_track1_bunch(ctx, lat, bunch, ix_ele, turn) bind(c, name='bmadgpu_track1_bunch')
    import
    type(c_ptr), value :: ctx, lat
    type(bmadgpu_bunch_t) :: bunch
    integer(c_int32_t), value :: ix_ele, turn
  end function
  type(c_ptr) function bmadgpu_last_error() bind(c, name='bmadgpu_last_error')
    import
  end function
  integer(c_int) function bmadgpu_closed_orbit(ctx, lat, dim, orbit, mat, rel_tol, abs_tol, max_iter, iterations) &
                                                                             bind(c, name='bmadgpu_closed_orbit')
    import
    type(c_ptr), value :: ctx, lat
    integer(c_int32_t), value :: dim, max_iter
    real(c_double) :: orbit(6), mat(36)
    real(c_double), value :: rel_tol, abs_tol
    integer(c_int32_t) :: iterations
  end function
  integer(c_int) function bmadgpu_one_turn_matrix(ctx, lat, orbit, rf_on, orbit_end, mat) &
                                                                             bind(c, name='bmadgpu_one_turn_matrix')
    import
    type(c_ptr), value :: ctx, lat
    real(c_double) :: orbit(6), orbit_end(6), mat(36)
    integer(c_int32_t), value :: rf_on
  end function
  integer(c_int) function bmadgpu_twiss_from_mat6(mat, orb0, tw) bind(c, name='bmadgpu_twiss_from_mat6')
    import
    real(c_double) :: mat(36), orb0(6)
    type(bmadgpu_twiss_t) :: tw
  end function
  integer(c_int) function bmadgpu_ltt_run(ctx, lat, bunch, params, turns_done) bind(c, name='bmadgpu_ltt_run')
    import
    type(c_ptr), value :: ctx, lat
    type(bmadgpu_bunch_t) :: bunch
    type(bmadgpu_ltt_params_t) :: params
    integer(c_int32_t) :: turns_done
  end function
end interface

type(c_ptr), save :: gpu_ctx = c_null_ptr, gpu_lat = c_null_ptr
integer, save :: gpu_branch = 0
! Turn index passed to the tracker (coord%ix_turn of particles lost in a call): advanced by
! bmadgpu_track_turns and, when the hook tracks the branch's last element, by the hook; a caller
! whose turn loop starts elsewhere sets it with bmadgpu_set_turn.
integer, save :: gpu_turn = 0
type (lat_struct), pointer, save :: gpu_lat_f => null()

contains

!+
! Subroutine bmadgpu_install (lat, ix_branch, err)
!
! Packs branch%ele(1:n_ele_track) into the device element table and points
! track1_bunch_hook_ptr at bmadgpu_track1_bunch_hook. Elements outside the device path make
! bmadgpu_lattice_create return an error and nothing is installed.
!-

subroutine bmadgpu_install (lat, ix_branch, err)

type (lat_struct), target :: lat
integer ix_branch
logical err
type (branch_struct), pointer :: branch
type (bmadgpu_element_t), allocatable :: eles(:)
type (bmadgpu_param_t) param
integer i, n

err = .true.
branch => lat%branch(ix_branch)
n = branch%n_ele_track
allocate (eles(n))
do i = 1, n
  call pack_element(branch%ele(i), eles(i))
enddo

param%p0c = branch%ele(0)%value(p0c$)
param%e_tot = branch%ele(0)%value(e_tot$)
param%mass = mass_of(branch%param%particle)
param%charge = charge_of(branch%param%particle)
param%max_aperture_limit = bmad_com%max_aperture_limit
param%default_ds_step = bmad_com%default_ds_step
param%aperture_limit_on = merge(1, 0, bmad_com%aperture_limit_on)
param%absolute_time_tracking = merge(1, 0, bmad_com%absolute_time_tracking)
param%radiation_on = merge(1, 0, bmad_com%radiation_damping_on .or. bmad_com%radiation_fluctuations_on .or. &
                                 bmad_com%spin_tracking_on)
param%reserved = 0

if (.not. c_associated(gpu_ctx)) then
  if (bmadgpu_ctx_create(0_c_int32_t, gpu_ctx) /= 0) return
endif
if (bmadgpu_lattice_create(gpu_ctx, eles, int(n, c_int32_t), param, gpu_lat) /= 0) return
gpu_branch = ix_branch
gpu_lat_f => lat
gpu_turn = 0
track1_bunch_hook_ptr => bmadgpu_track1_bunch_hook
err = .false.

end subroutine bmadgpu_install

!+
! Subroutine pack_element (ele, e)
! One bmadgpu_element from ele%value(...) and the multipole arrays.
!-

subroutine pack_element (ele, e)

type (ele_struct) ele
type (bmadgpu_element_t) e

e%key = ele%key;  e%is_on = merge(1, 0, ele%is_on)
e%fringe_type = nint(ele%value(fringe_type$));  e%fringe_at = nint(ele%value(fringe_at$))
e%aperture_at = ele%aperture_at;  e%aperture_type = ele%aperture_type
e%num_steps = nint(ele%value(num_steps$));  e%scale_multipoles = merge(1, 0, ele%scale_multipoles)
e%field_master = merge(1, 0, ele%field_master);  e%exact_multipoles = nint(ele%value(exact_multipoles$))
e%orientation = ele%orientation;  e%reserved = 0
e%l = ele%value(l$);  e%k1 = ele%value(k1$);  e%k2 = ele%value(k2$);  e%k3 = ele%value(k3$)
e%g = ele%value(g$);  e%dg = ele%value(dg$);  e%e1 = ele%value(e1$);  e%e2 = ele%value(e2$)
e%fint = ele%value(fint$);  e%fintx = ele%value(fintx$);  e%hgap = ele%value(hgap$);  e%hgapx = ele%value(hgapx$)
e%tilt = ele%value(tilt_tot$);  e%ref_tilt = ele%value(ref_tilt_tot$);  e%roll = ele%value(roll_tot$)
e%x_offset = ele%value(x_offset_tot$);  e%y_offset = ele%value(y_offset_tot$);  e%z_offset = ele%value(z_offset_tot$)
e%x_pitch = ele%value(x_pitch_tot$);  e%y_pitch = ele%value(y_pitch_tot$)
e%hkick = ele%value(hkick$);  e%vkick = ele%value(vkick$)
e%x1_limit = ele%value(x1_limit$);  e%x2_limit = ele%value(x2_limit$)
e%y1_limit = ele%value(y1_limit$);  e%y2_limit = ele%value(y2_limit$)
e%voltage = ele%value(voltage$);  e%rf_frequency = ele%value(rf_frequency$)
e%phi0 = ele%value(phi0$);  e%phi0_multipass = ele%value(phi0_multipass$)
e%ds_step = ele%value(ds_step$);  e%r0_mag = ele%value(r0_mag$);  e%r0_elec = ele%value(r0_elec$)
e%delta_ref_time = ele%value(delta_ref_time$)
e%fq1 = 0;  e%fq2 = 0
if (ele%key == quadrupole$) then
  e%fq1 = ele%value(fq1$);  e%fq2 = ele%value(fq2$)
endif
e%px_aperture_width2 = 0;  e%px_aperture_center = 0;  e%py_aperture_width2 = 0;  e%py_aperture_center = 0
e%z_aperture_width2 = 0;  e%z_aperture_center = 0;  e%pz_aperture_width2 = 0;  e%pz_aperture_center = 0
e%kick = 0
if (ele%key == hkicker$ .or. ele%key == vkicker$) e%kick = ele%value(kick$)
if (ele%key == ecollimator$ .or. ele%key == rcollimator$) then
  e%px_aperture_width2 = ele%value(px_aperture_width2$);  e%px_aperture_center = ele%value(px_aperture_center$)
  e%py_aperture_width2 = ele%value(py_aperture_width2$);  e%py_aperture_center = ele%value(py_aperture_center$)
  e%z_aperture_width2 = ele%value(z_aperture_width2$);  e%z_aperture_center = ele%value(z_aperture_center$)
  e%pz_aperture_width2 = ele%value(pz_aperture_width2$);  e%pz_aperture_center = ele%value(pz_aperture_center$)
endif
e%a_pole = 0;  e%b_pole = 0;  e%a_pole_elec = 0;  e%b_pole_elec = 0
if (associated(ele%a_pole)) then
  e%a_pole = ele%a_pole(0:bmadgpu_n_pole-1);  e%b_pole = ele%b_pole(0:bmadgpu_n_pole-1)
endif
if (associated(ele%a_pole_elec)) then
  e%a_pole_elec = ele%a_pole_elec(0:bmadgpu_n_pole-1);  e%b_pole_elec = ele%b_pole_elec(0:bmadgpu_n_pole-1)
endif

end subroutine pack_element

!+
! Subroutine bmadgpu_track1_bunch_hook (bunch, ele, err, centroid, direction, finished, bunch_track)
! The track1_bunch_hook_def procedure: tracks the bunch through ele on the GPU.
!-

subroutine bmadgpu_track1_bunch_hook (bunch, ele, err, centroid, direction, finished, bunch_track)

type (bunch_struct), target :: bunch
type (ele_struct), target :: ele
logical err, finished
type (coord_struct), optional :: centroid(0:)
integer, optional :: direction
type (bunch_track_struct), optional :: bunch_track

finished = .false.
err = .false.
if (integer_option(1, direction) /= 1 .or. present(bunch_track)) return   ! Bmad's own code path
if (ele%ix_branch /= gpu_branch .or. ele%ix_ele < 1) return
call track_on_gpu (bunch, ele%ix_ele - 1, ele%ix_ele, 1, err)
finished = .not. err
if (finished .and. ele%ix_ele == gpu_lat_f%branch(gpu_branch)%n_ele_track) gpu_turn = gpu_turn + 1

end subroutine bmadgpu_track1_bunch_hook

!+
! Subroutine bmadgpu_set_turn (ix_turn)
! Sets the turn index the next tracking call starts at (recorded in coord%ix_turn of the
! particles it loses).
!-

subroutine bmadgpu_set_turn (ix_turn)
integer ix_turn
gpu_turn = ix_turn
end subroutine bmadgpu_set_turn

!+
! Subroutine bmadgpu_track_turns (bunch, n_turns, err)
! All elements of the installed branch, n_turns times (the element and turn loops of
! track_bunch / ltt_run_beam_mode in one call).
!-

subroutine bmadgpu_track_turns (bunch, n_turns, n_ele_track, err)

type (bunch_struct), target :: bunch
integer n_turns, n_ele_track
logical err

call track_on_gpu (bunch, 0, n_ele_track, n_turns, err)
if (.not. err) gpu_turn = gpu_turn + n_turns

end subroutine bmadgpu_track_turns

subroutine track_on_gpu (bunch, ix_start, ix_end, n_turns, err)

type (bunch_struct), target :: bunch
integer ix_start, ix_end, n_turns
logical err
real(c_double), allocatable, target :: vec(:,:), beta(:), t(:)
integer(c_int32_t), allocatable, target :: state(:), ix_ele(:), ix_turn(:), location(:)
type (bmadgpu_bunch_t) b
type (branch_struct), pointer :: branch
type (ele_struct), pointer :: ele
integer j, n, i

branch => gpu_lat_f%branch(gpu_branch)

n = size(bunch%particle)
allocate (vec(n, 6), beta(n), t(n), state(n), ix_ele(n), ix_turn(n), location(n))
do j = 1, n
  do i = 1, 6
    vec(j, i) = bunch%particle(j)%vec(i)
  enddo
  beta(j) = bunch%particle(j)%beta
  t(j) = real(bunch%particle(j)%t, c_double)
  state(j) = bunch%particle(j)%state
enddo
ix_ele = -1;  ix_turn = -1;  location = 0
b%n = n
b%vec = c_loc(vec);  b%beta = c_loc(beta);  b%t = c_loc(t);  b%state = c_loc(state)
b%ix_ele = c_loc(ix_ele);  b%ix_turn = c_loc(ix_turn);  b%location = c_loc(location)
err = (bmadgpu_track_bunch(gpu_ctx, gpu_lat, b, int(ix_start, c_int32_t), int(ix_end, c_int32_t), &
                           int(gpu_turn, c_int32_t), int(n_turns, c_int32_t), c_null_ptr) /= 0)
if (err) return
do j = 1, n
  do i = 1, 6
    bunch%particle(j)%vec(i) = vec(j, i)
  enddo
  bunch%particle(j)%beta = beta(j)
  bunch%particle(j)%t = t(j)
  bunch%particle(j)%state = state(j)
  if (ix_ele(j) >= 0) then        ! lost in this call
    ! as track1 leaves a particle lost at element ix: ix_ele (track1.f90:92), the location, and s
    ! at the element's end unless the loss was at its entrance (track1_bmad.f90:277-281)
    ele => branch%ele(ix_ele(j) + 1)
    bunch%particle(j)%ix_ele = ix_ele(j) + 1
    bunch%particle(j)%ix_turn = ix_turn(j)
    bunch%particle(j)%location = location(j)
    bunch%particle(j)%s = merge(ele%s_start, ele%s, location(j) == upstream_end$)
  elseif (state(j) == alive$) then
    ! survivors as track1 leaves them after the last element tracked (track1.f90:92, 296-304;
    ! track1_bmad.f90:277-281)
    bunch%particle(j)%ix_ele = ix_end
    bunch%particle(j)%location = downstream_end$
    bunch%particle(j)%s = branch%ele(ix_end)%s
  endif
enddo
bunch%n_live = count(bunch%particle%state == alive$)
bunch%charge_live = sum(bunch%particle%charge, mask = (bunch%particle%state == alive$))

end subroutine track_on_gpu

!+
! Subroutine bmadgpu_closed_orbit_calc (closed_orb, i_dim, err)
!
! closed_orbit_calc (bmad/code/closed_orbit_calc.f90:192) for the installed branch, forward: the
! closed orbit at the branch start, found by Newton's method on the GPU's one-turn map. The guess
! is closed_orb(0)%vec (its vec(6) the energy for i_dim = 4); the result goes to closed_orb(0)%vec
! only -- the orbit at the other elements is not filled. i_dim = 0 takes 6 when a cavity is on,
! else 4. Tolerances are bmad_com%rel_tol_tracking / %abs_tol_tracking.
!-

subroutine bmadgpu_closed_orbit_calc (closed_orb, i_dim, err)

type (coord_struct) :: closed_orb(0:)
integer i_dim
logical err
real(c_double) orbit(6), mat(36)
integer(c_int32_t) its

orbit = closed_orb(0)%vec
err = (bmadgpu_closed_orbit(gpu_ctx, gpu_lat, int(i_dim, c_int32_t), orbit, mat, bmad_com%rel_tol_tracking, &
                            bmad_com%abs_tol_tracking, 0_c_int32_t, its) /= 0)
if (err) return
closed_orb(0)%vec = orbit

end subroutine bmadgpu_closed_orbit_calc

!+
! Subroutine bmadgpu_twiss_at_start (lat, orbit, status)
!
! The periodic Twiss of twiss_at_start (bmad/code/twiss_at_start.f90:29) for the installed
! branch: the RF-off one-turn matrix about orbit(1:6) from GPU tracking, decoupled as
! twiss_from_mat6 does, written to branch%ele(0) (a, b, x, y, c_mat, gamma_c) and the tunes to
! lat%a%tune, lat%b%tune. status is Bmad's matrix status (ok$ = 1).
!-

subroutine bmadgpu_twiss_at_start (lat, orbit, status)

type (lat_struct), target :: lat
real(rp) orbit(6)
integer status
type (ele_struct), pointer :: ele0
type (bmadgpu_twiss_t) tw
real(c_double) orb(6), orb_end(6), mat(36)

status = unstable$
orb = orbit
if (bmadgpu_one_turn_matrix(gpu_ctx, gpu_lat, orb, 0_c_int32_t, orb_end, mat) /= 0) return
if (bmadgpu_twiss_from_mat6(mat, orb, tw) /= 0) return
status = tw%status
if (status /= ok$) return
ele0 => lat%branch(gpu_branch)%ele(0)
ele0%a%beta = tw%beta_a;  ele0%a%alpha = tw%alpha_a;  ele0%a%gamma = tw%gamma_a
ele0%a%eta = tw%eta_a;  ele0%a%etap = tw%etap_a;  ele0%a%deta_ds = tw%deta_ds_a
ele0%b%beta = tw%beta_b;  ele0%b%alpha = tw%alpha_b;  ele0%b%gamma = tw%gamma_b
ele0%b%eta = tw%eta_b;  ele0%b%etap = tw%etap_b;  ele0%b%deta_ds = tw%deta_ds_b
ele0%x%eta = tw%eta_x;  ele0%x%etap = tw%etap_x;  ele0%x%deta_ds = tw%deta_ds_x
ele0%y%eta = tw%eta_y;  ele0%y%etap = tw%etap_y;  ele0%y%deta_ds = tw%deta_ds_y
ele0%c_mat = reshape(tw%c_mat, [2, 2], order = [2, 1])   ! C row-major -> c_mat(i,j)
ele0%gamma_c = tw%gamma_c
ele0%a%phi = 0;  ele0%b%phi = 0
lat%a%tune = tw%phi_a;  lat%b%tune = tw%phi_b

end subroutine bmadgpu_twiss_at_start

!+
! Subroutine bmadgpu_ltt_beam (bunch, n_turns, averages_file, phase_space_file, beam_file,
!     averages_every, particle_every, beam_every, dead_cutoff, core_emit_cutoff,
!     core_emit_combined_calc, action_angle_file, per_particle_file, only_live_out,
!     output_only_last_turns, ix_turn_start, turns_done, err)
!
! ltt_run_beam_mode (bsim/modules/lt_tracking_mod.f90:1571-1715) for one bunch on the installed
! branch, outputs included. The arguments are the ltt%... settings of the same meaning
! (ltt%averages_output_file, ltt%phase_space_output_file, ltt%beam_output_file,
! ltt%averages_output_every_n_turns, ltt%particle_output_every_n_turns,
! ltt%beam_output_every_n_turns, ltt%dead_cutoff, ltt%core_emit_cutoff,
! ltt%core_emit_combined_calc, ltt%action_angle_output_file, ltt%per_particle_output_file,
! ltt%only_live_particles_out, ltt%output_only_last_turns, ltt%ix_turn_start); '' means no
! file. The bunch is updated in place as bmadgpu_track_turns updates it; turns_done is the turn
! reached (n_turns, or the turn the stop conditions ended the run).
!-

subroutine bmadgpu_ltt_beam (bunch, n_turns, averages_file, phase_space_file, beam_file, averages_every, &
                             particle_every, beam_every, dead_cutoff, core_emit_cutoff, core_emit_combined_calc, &
                             action_angle_file, per_particle_file, only_live_out, output_only_last_turns, &
                             ix_turn_start, turns_done, err)

type (bunch_struct), target :: bunch
integer n_turns, averages_every, particle_every, beam_every, output_only_last_turns, ix_turn_start, turns_done
character(*) averages_file, phase_space_file, beam_file, action_angle_file, per_particle_file
real(rp) dead_cutoff, core_emit_cutoff(:)
logical core_emit_combined_calc, only_live_out, err
character(kind=c_char), allocatable, target :: f_ave(:), f_ps(:), f_beam(:), f_aa(:), f_pp(:)
real(c_double), allocatable, target :: vec(:,:), beta(:), t(:)
integer(c_int32_t), allocatable, target :: state(:), ix_ele(:), ix_turn(:), location(:)
type (bmadgpu_bunch_t) b
type (bmadgpu_ltt_params_t) p
integer(c_int32_t) done
integer i, j, n

n = size(bunch%particle)
allocate (vec(n, 6), beta(n), t(n), state(n), ix_ele(n), ix_turn(n), location(n))
do j = 1, n
  do i = 1, 6
    vec(j, i) = bunch%particle(j)%vec(i)
  enddo
  beta(j) = bunch%particle(j)%beta
  t(j) = real(bunch%particle(j)%t, c_double)
  state(j) = bunch%particle(j)%state
enddo
ix_ele = -1;  ix_turn = -1;  location = 0
b%n = n
b%vec = c_loc(vec);  b%beta = c_loc(beta);  b%t = c_loc(t);  b%state = c_loc(state)
b%ix_ele = c_loc(ix_ele);  b%ix_turn = c_loc(ix_turn);  b%location = c_loc(location)

p%n_turns = n_turns
p%averages_every_n_turns = averages_every
p%particle_every_n_turns = particle_every
p%output_only_last_turns = output_only_last_turns
p%only_live_particles_out = merge(1, 0, only_live_out)
p%ix_turn_start = ix_turn_start
p%beam_every_n_turns = beam_every
p%beam_exact = 0
p%dead_cutoff = dead_cutoff
p%core_emit_cutoff = -1
do i = 1, min(8, size(core_emit_cutoff))
  p%core_emit_cutoff(i) = core_emit_cutoff(i)
enddo
p%core_emit_per_mode = merge(0, 1, core_emit_combined_calc)
call c_string (averages_file, f_ave, p%averages_file)
call c_string (phase_space_file, f_ps, p%phase_space_file)
call c_string (beam_file, f_beam, p%beam_file)
call c_string (action_angle_file, f_aa, p%action_angle_file)
call c_string (per_particle_file, f_pp, p%per_particle_file)
p%action_angle_n_inv = c_null_ptr

err = (bmadgpu_ltt_run(gpu_ctx, gpu_lat, b, p, done) /= 0)
if (err) return
turns_done = done
do j = 1, n
  do i = 1, 6
    bunch%particle(j)%vec(i) = vec(j, i)
  enddo
  bunch%particle(j)%beta = beta(j)
  bunch%particle(j)%t = t(j)
  bunch%particle(j)%state = state(j)
  if (ix_ele(j) >= 0) then        ! lost in this run
    bunch%particle(j)%ix_ele = ix_ele(j) + 1
    bunch%particle(j)%location = location(j)
  else
    bunch%particle(j)%location = downstream_end$
  endif
enddo
bunch%n_live = count(bunch%particle%state == alive$)
bunch%charge_live = sum(bunch%particle%charge, mask = (bunch%particle%state == alive$))

contains

! A NUL-terminated copy of trim(str) in buf and its address, or c_null_ptr for an empty name.
subroutine c_string (str, buf, ptr)
character(*) str
character(kind=c_char), allocatable, target :: buf(:)
type(c_ptr) ptr
integer k, m
m = len_trim(str)
if (m == 0) then
  ptr = c_null_ptr
  return
endif
allocate (buf(m + 1))
do k = 1, m
  buf(k) = str(k:k)
enddo
buf(m + 1) = c_null_char
ptr = c_loc(buf)
end subroutine c_string

end subroutine bmadgpu_ltt_beam

end module bmadgpu_mod
