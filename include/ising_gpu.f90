! ising_gpu.f90 -- Fortran 2008 bindings (ISO_C_BINDING) of libisinggpu, the C-ABI declared in
! ising_gpu.h.  The reference's drivers (src/PT.f90, src/ISING.f90) use this module in place of
! the mesh, energy, sweep and exchange routines of chainMesh.f90, energyMin.f90 and PT.f90;
! every function returns the library's status and ising_check turns a nonzero status into
! error stop, the reference's behaviour on a failed call.  Link with -lisinggpu.
module ising_gpu
  use iso_c_binding
  implicit none
  integer(c_int), parameter :: ISING_OK = 0
  integer(c_int), parameter :: ISING_MOVE_UNIFORM = 0, ISING_MOVE_BALL = 1
  integer(c_int), parameter :: ISING_DMI_INTERFACIAL = 0, ISING_DMI_BULK = 1

  type, bind(C) :: ising_params
    real(c_double) :: J, J_prime, Dz, Dz_prime, B, K
    real(c_double) :: K_axis(3)
    real(c_double) :: zeeman_factor
    integer(c_int) :: include_Jp, dmi_mode
    real(c_double) :: dmi_axis(3)
    integer(c_int) :: legacy_neighbours, demag
  end type

  type, bind(C) :: ising_pt_options
    integer(c_int64_t) :: seed
    integer(c_int32_t) :: ensemble
    integer(c_int) :: move
    real(c_double) :: r
    integer(c_int) :: scheme, resync_every, record, record_capacity, l2_group, sweep_kernel
  end type

  type, bind(C) :: ising_ensemble_desc         ! one parameter slot of src/PT.f90:147-176
    type(c_ptr) :: mesh                          ! its own mesh
    integer(c_int) :: n_temps
    type(c_ptr) :: betas                         ! c_loc of n_temps inverse temperatures
    type(ising_params) :: params
    integer(c_int32_t) :: ensemble               ! Philox key component (< 2**24)
  end type

  type, bind(C) :: ising_ensembles_options
    integer(c_int64_t) :: seed
    integer(c_int) :: move
    real(c_double) :: r
    integer(c_int) :: scheme, resync_every, wait_timeout_ms
  end type

  ! schedule of the batched engine (ising_ensembles_schedule_t); loader selects how a sweep
  ! reads its neighbours: per thread, TMA-staged rows, or both colour passes fused into one
  ! pass over two spin buffers (even sweeps_per_swap)
  integer(c_int), parameter :: ISING_ENS_ORDER_PHASE = 0, ISING_ENS_ORDER_GROUPS = 1, ISING_ENS_ORDER_WAVE = 2
  integer(c_int), parameter :: ISING_ENS_LOADER_REGISTERS = 0, ISING_ENS_LOADER_STAGED = 1, &
      ISING_ENS_LOADER_FUSED = 2
  type, bind(C) :: ising_ensembles_schedule
    integer(c_int) :: block_threads, chunk_pairs, order
    integer(c_int64_t) :: group_bytes
    real(c_double) :: ms_per_round
    integer(c_int) :: loader
  end type

  interface
    integer(c_int) function ising_mesh_create(frac, n_atoms_cell, nx, ny, nz, a, b, c, ab, bc, ca, &
        shell_tol, n_shells, n_replicas, device, mesh) bind(C, name="ising_mesh_create")
      import :: c_int, c_float, c_double, c_ptr
      real(c_float), intent(in) :: frac(*)
      integer(c_int), value :: n_atoms_cell, nx, ny, nz, n_shells, n_replicas, device
      real(c_double), value :: a, b, c, ab, bc, ca, shell_tol
      type(c_ptr), intent(out) :: mesh
    end function
    integer(c_int) function ising_mesh_destroy(mesh) bind(C, name="ising_mesh_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: mesh
    end function
    integer(c_int) function ising_spins_set(mesh, replica, spins) bind(C, name="ising_spins_set")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: mesh
      integer(c_int), value :: replica
      real(c_double), intent(in) :: spins(*)          ! atomSpins(numAtoms,3), column-major
    end function
    integer(c_int) function ising_spins_get(mesh, replica, spins) bind(C, name="ising_spins_get")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: mesh
      integer(c_int), value :: replica
      real(c_double), intent(out) :: spins(*)
    end function
    ! queued forms: the array must stay allocated and untouched until ising_spins_wait
    ! (declare it with the asynchronous attribute, or pass c_loc of a pinned buffer)
    integer(c_int) function ising_spins_get_async(mesh, replica, spins) bind(C, name="ising_spins_get_async")
      import :: c_int, c_ptr
      type(c_ptr), value :: mesh, spins
      integer(c_int), value :: replica
    end function
    integer(c_int) function ising_spins_set_async(mesh, replica, spins) bind(C, name="ising_spins_set_async")
      import :: c_int, c_ptr
      type(c_ptr), value :: mesh, spins
      integer(c_int), value :: replica
    end function
    integer(c_int) function ising_spins_wait(mesh) bind(C, name="ising_spins_wait")
      import :: c_int, c_ptr
      type(c_ptr), value :: mesh
    end function
    integer(c_int) function ising_params_reference(which, J, Jp, Dz, Dzp, B, p) &
        bind(C, name="ising_params_reference")
      import :: c_int, c_double, ising_params
      integer(c_int), value :: which                  ! 0 local routines, 1 TotalHeisenbergEnergy
      real(c_double), value :: J, Jp, Dz, Dzp, B
      type(ising_params), intent(out) :: p
    end function
    integer(c_int) function ising_metropolis_mcs(mesh, replica, beta, n_sweeps, p, r, seed) &
        bind(C, name="ising_metropolis_mcs")
      import :: c_int, c_double, c_int64_t, c_ptr, ising_params
      type(c_ptr), value :: mesh
      integer(c_int), value :: replica, n_sweeps
      real(c_double), value :: beta, r
      type(ising_params), intent(in) :: p
      integer(c_int64_t), value :: seed
    end function
    integer(c_int) function ising_local_energy(mesh, replica, atom, p, s_prop, old_e, new_e) &
        bind(C, name="ising_local_energy")
      import :: c_int, c_double, c_ptr, ising_params
      type(c_ptr), value :: mesh
      integer(c_int), value :: replica, atom        ! atom is 1-based like atomIndex
      type(ising_params), intent(in) :: p
      real(c_double), intent(in) :: s_prop(3)
      real(c_double), intent(out) :: old_e, new_e
    end function
    integer(c_int) function ising_total_energy(mesh, replica, p, e) bind(C, name="ising_total_energy")
      import :: c_int, c_double, c_ptr, ising_params
      type(c_ptr), value :: mesh
      integer(c_int), value :: replica
      type(ising_params), intent(in) :: p
      real(c_double), intent(out) :: e
    end function
    integer(c_int) function ising_demag_field(mesh, replica, h) bind(C, name="ising_demag_field")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: mesh
      integer(c_int), value :: replica
      real(c_double), intent(out) :: h(*)           ! outputArray(numAtoms, 3), column-major
    end function
    integer(c_int) function ising_write_demag_csv(mesh, replica, path) bind(C, name="ising_write_demag_csv")
      import :: c_int, c_char, c_ptr
      type(c_ptr), value :: mesh
      integer(c_int), value :: replica
      character(kind=c_char), intent(in) :: path(*)  ! NUL-terminated
    end function
    integer(c_int) function ising_winding_number(mesh, replica, z_index, q) bind(C, name="ising_winding_number")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: mesh
      integer(c_int), value :: replica, z_index     ! 1-based like Z_index
      real(c_double), intent(out) :: q
    end function
    integer(c_int) function ising_statistics(mesh, replica, wnd_mid, wnd_spread, m) bind(C, name="ising_statistics")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: mesh
      integer(c_int), value :: replica
      real(c_double), intent(out) :: wnd_mid, wnd_spread, m(3)
    end function
    integer(c_int) function ising_pt_create(mesh, n_temps, betas, p, opt, pt) bind(C, name="ising_pt_create")
      import :: c_int, c_double, c_ptr, ising_params, ising_pt_options
      type(c_ptr), value :: mesh
      integer(c_int), value :: n_temps
      real(c_double), intent(in) :: betas(*)
      type(ising_params), intent(in) :: p
      type(ising_pt_options), intent(in) :: opt
      type(c_ptr), intent(out) :: pt
    end function
    integer(c_int) function ising_pt_run(pt, sweeps_per_swap, rounds) bind(C, name="ising_pt_run")
      import :: c_int, c_ptr
      type(c_ptr), value :: pt
      integer(c_int), value :: sweeps_per_swap, rounds
    end function
    integer(c_int) function ising_pt_relax(pt, n_sweeps) bind(C, name="ising_pt_relax")
      import :: c_int, c_ptr
      type(c_ptr), value :: pt
      integer(c_int), value :: n_sweeps
    end function
    integer(c_int) function ising_pt_permutation(pt, temp_to_replica) bind(C, name="ising_pt_permutation")
      import :: c_int, c_ptr
      type(c_ptr), value :: pt
      integer(c_int), intent(out) :: temp_to_replica(*)   ! 0-based replica per temperature slot
    end function
    integer(c_int) function ising_write_spins_csv(mesh, replica, path, append, header, frame) &
        bind(C, name="ising_write_spins_csv")
      import :: c_int, c_char, c_ptr
      type(c_ptr), value :: mesh
      integer(c_int), value :: replica, append, header, frame
      character(kind=c_char), intent(in) :: path(*)       ! NUL-terminated
    end function
    integer(c_int) function ising_write_pt_data_csv(path, J, D, B, T, wnd_mid, sk_mid, wnd_spread, m) &
        bind(C, name="ising_write_pt_data_csv")
      import :: c_int, c_char, c_double
      character(kind=c_char), intent(in) :: path(*)
      real(c_double), value :: J, D, B, T, wnd_mid, wnd_spread
      integer(c_int), value :: sk_mid
      real(c_double), intent(in) :: m(3)
    end function
    integer(c_int) function ising_chain_mesh_statistics(mesh, replica, sk_mid, wnd_mid, wnd_spread, m) &
        bind(C, name="ising_chain_mesh_statistics")             ! chainMesh_statistics, PT-Utils.f90:33-66
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: mesh
      integer(c_int), value :: replica
      integer(c_int), intent(out) :: sk_mid
      real(c_double), intent(out) :: wnd_mid, wnd_spread, m(3)
    end function
    integer(c_int) function ising_mesh_set_interpolation_scale(mesh, sclx, scly) &
        bind(C, name="ising_mesh_set_interpolation_scale")      ! makeChainMesh's sclx, scly
      import :: c_int, c_ptr
      type(c_ptr), value :: mesh
      integer(c_int), value :: sclx, scly
    end function
    integer(c_int) function ising_skyrmion_number(mesh, replica, z, q_threshold, particle_number, sigma, n) &
        bind(C, name="ising_skyrmion_number")                   ! calculate_skyrmion_number, rsp:627-812
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: mesh
      integer(c_int), value :: replica, z, particle_number
      real(c_double), value :: q_threshold, sigma
      integer(c_int), intent(out) :: n
    end function
    integer(c_int) function ising_skyrmion_distribution(mesh, replica, N, min_t, max_t, num_t, z, winding) &
        bind(C, name="ising_skyrmion_distribution")             ! compute_skyrmion_distribution, rsp:930-983
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: mesh
      integer(c_int), value :: replica, N, num_t, z
      real(c_double), value :: min_t, max_t
      integer(c_int), intent(out) :: winding(*)
    end function
    integer(c_int) function ising_winding_density_all(mesh, replica, density) &
        bind(C, name="ising_winding_density_all")               ! every slice's density_matrix
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: mesh
      integer(c_int), value :: replica
      real(c_double), intent(out) :: density(*)             ! (numCellsX, numCellsY, numCellsZ)
    end function
    type(c_ptr) function ising_last_error() bind(C, name="ising_last_error")
      import :: c_ptr
    end function
    integer(c_int) function ising_ensembles_create(n, desc, opt, eng) bind(C, name="ising_ensembles_create")
      import :: c_int, c_ptr, ising_ensemble_desc, ising_ensembles_options
      integer(c_int), value :: n
      type(ising_ensemble_desc), intent(in) :: desc(*)
      type(ising_ensembles_options), intent(in) :: opt
      type(c_ptr), intent(out) :: eng
    end function
    integer(c_int) function ising_ensembles_destroy(eng) bind(C, name="ising_ensembles_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: eng
    end function
    integer(c_int) function ising_ensembles_run(eng, sweeps_per_swap, rounds) bind(C, name="ising_ensembles_run")
      import :: c_int, c_ptr
      type(c_ptr), value :: eng
      integer(c_int), value :: sweeps_per_swap, rounds
    end function
    integer(c_int) function ising_ensembles_autotune(eng, sweeps_per_swap, rounds_per_trial, trials, &
        max_trials, n_trials) bind(C, name="ising_ensembles_autotune")
      import :: c_int, c_ptr
      type(c_ptr), value :: eng, trials, n_trials      ! c_null_ptr when the trials are not wanted
      integer(c_int), value :: sweeps_per_swap, rounds_per_trial, max_trials
    end function
    integer(c_int) function ising_ensembles_set_schedule(eng, sched) bind(C, name="ising_ensembles_set_schedule")
      import :: c_int, c_ptr, ising_ensembles_schedule
      type(c_ptr), value :: eng
      type(ising_ensembles_schedule), intent(in) :: sched
    end function
    integer(c_int) function ising_ensembles_get_schedule(eng, sched, grid_blocks, tasks_per_pass) &
        bind(C, name="ising_ensembles_get_schedule")
      import :: c_int, c_int64_t, c_ptr, ising_ensembles_schedule
      type(c_ptr), value :: eng
      type(ising_ensembles_schedule), intent(out) :: sched
      integer(c_int), intent(out) :: grid_blocks
      integer(c_int64_t), intent(out) :: tasks_per_pass
    end function
    integer(c_int) function ising_ensembles_set_resync(eng, every) bind(C, name="ising_ensembles_set_resync")
      import :: c_int, c_ptr
      type(c_ptr), value :: eng
      integer(c_int), value :: every
    end function
    integer(c_int) function ising_ensembles_permutation(eng, e, temp_to_replica) &
        bind(C, name="ising_ensembles_permutation")
      import :: c_int, c_ptr
      type(c_ptr), value :: eng
      integer(c_int), value :: e                        ! 0-based ensemble (slot) index
      integer(c_int), intent(out) :: temp_to_replica(*)
    end function
    integer(c_int) function ising_ensembles_energies(eng, e, e_per_replica, m_per_replica) &
        bind(C, name="ising_ensembles_energies")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: eng
      integer(c_int), value :: e
      real(c_double), intent(out) :: e_per_replica(*), m_per_replica(3, *)
    end function
  end interface
contains
  subroutine ising_check(status, where)          ! the reference's error stop behaviour
    integer(c_int), intent(in) :: status
    character(len=*), intent(in) :: where
    if (status /= ISING_OK) then
      write(*, '(A,A,I0)') where, ": libisinggpu status ", status
      error stop "libisinggpu call failed"
    end if
  end subroutine
end module ising_gpu
