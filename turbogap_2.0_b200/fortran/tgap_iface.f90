! ISO_C_BINDING interface to libtgap (include/tgap.h) for a TurboGAP build.
!
! Each interface mirrors the Fortran routine it replaces; the wrapper subroutines keep the
! reference argument lists so call sites change only the routine name:
!   tgap_build_neighbors            <- build_neighbors_list        (src/neighbors/neighbors_interface.f90:144)
!   tgap_get_soap                   <- soap_turbo get_soap         (src/gap/gap_interface.f90:301-306)
!   tgap_get_soap_energy_and_forces <- get_soap_energy_and_forces  (src/gap/gap.f90:39)
!   tgap_get_gap_soap               <- get_gap_soap                (src/gap/gap_interface.f90:41)
! Not compiled in the build image (it has no Fortran compiler).
module tgap_iface
   use iso_c_binding
   implicit none

   integer(c_int), parameter :: TGAP_OK = 0, TGAP_ERR_CAPACITY = 3
   integer(c_int), parameter :: TGAP_FP64 = 0, TGAP_MIXED = 1

   type, bind(C) :: tgap_soap_hypers
      integer(c_int) :: n_species
      type(c_ptr) :: alpha_max
      integer(c_int) :: l_max
      type(c_ptr) :: rcut_hard, rcut_soft, nf, global_scaling
      type(c_ptr) :: atom_sigma_r, atom_sigma_r_scaling, atom_sigma_t, atom_sigma_t_scaling
      type(c_ptr) :: amplitude_scaling, central_weight
      integer(c_int) :: radial_enhancement
   end type

   interface
      integer(c_int) function tgap_create(device, ctx) bind(C, name="tgap_create")
         import :: c_int, c_ptr
         integer(c_int), value :: device
         type(c_ptr) :: ctx
      end function

      integer(c_int) function tgap_destroy(ctx) bind(C, name="tgap_destroy")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function

      ! page-lock a host array reused across calls (c_loc of a target array), so the host-buffer
      ! entries copy to and from it directly
      integer(c_int) function tgap_host_register(ctx, ptr, bytes) bind(C, name="tgap_host_register")
         import :: c_int, c_ptr, c_size_t
         type(c_ptr), value :: ctx, ptr
         integer(c_size_t), value :: bytes
      end function

      integer(c_int) function tgap_host_unregister(ctx, ptr) bind(C, name="tgap_host_unregister")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx, ptr
      end function

      type(c_ptr) function tgap_last_error(ctx) bind(C, name="tgap_last_error")
         import :: c_ptr
         type(c_ptr), value :: ctx
      end function

      integer(c_int) function tgap_number_of_unit_cells(a, b, c, rcut, indices) &
         bind(C, name="tgap_number_of_unit_cells")
         import :: c_int, c_double
         real(c_double), intent(in) :: a(3), b(3), c(3)
         real(c_double), value :: rcut
         integer(c_int) :: indices(3)
      end function

      integer(c_int) function tgap_build_neighbors(ctx, n_sites, n_sites_supercell, positions, a_box, &
                                                   b_box, c_box, box_small, rcut_max, species_supercell, &
                                                   rebuild, n_neigh, neighbors_list, rjs, xyz, thetas, phis, &
                                                   neighbor_species, capacity, n_atom_pairs) &
         bind(C, name="tgap_build_neighbors")
         import :: c_int, c_ptr, c_double, c_int64_t
         type(c_ptr), value :: ctx
         integer(c_int), value :: n_sites, n_sites_supercell, box_small, rebuild
         real(c_double), intent(in) :: positions(3, *), a_box(3), b_box(3), c_box(3)
         real(c_double), value :: rcut_max
         integer(c_int), intent(in) :: species_supercell(*)
         integer(c_int) :: n_neigh(*), neighbors_list(*), neighbor_species(*)
         real(c_double) :: rjs(*), xyz(3, *), thetas(*), phis(*)
         integer(c_int64_t), value :: capacity
         integer(c_int64_t) :: n_atom_pairs
      end function

      integer(c_int) function tgap_get_soap(ctx, n_sites, n_neigh, n_species, species, species_multiplicity, &
                                            n_atom_pairs, mask, rjs, thetas, phis, alpha_max, l_max, rcut_hard, &
                                            rcut_soft, nf, global_scaling, atom_sigma_r, atom_sigma_r_scaling, &
                                            atom_sigma_t, atom_sigma_t_scaling, amplitude_scaling, &
                                            radial_enhancement, central_weight, basis, scaling_mode, &
                                            do_derivatives, compress_soap, compress_P_nonzero, compress_P_i, &
                                            compress_P_j, compress_P_el, soap, soap_cart_der) &
         bind(C, name="tgap_get_soap")
         import :: c_int, c_ptr, c_double, c_char, c_signed_char
         type(c_ptr), value :: ctx
         integer(c_int), value :: n_sites, n_species, n_atom_pairs, l_max, radial_enhancement
         integer(c_int), value :: do_derivatives, compress_soap, compress_P_nonzero
         integer(c_int), intent(in) :: n_neigh(*), species(*), species_multiplicity(*), alpha_max(*)
         integer(c_signed_char), intent(in) :: mask(n_atom_pairs, *)
         real(c_double), intent(in) :: rjs(*), thetas(*), phis(*), rcut_hard(*), rcut_soft(*), nf(*)
         real(c_double), intent(in) :: global_scaling(*), atom_sigma_r(*), atom_sigma_r_scaling(*)
         real(c_double), intent(in) :: atom_sigma_t(*), atom_sigma_t_scaling(*), amplitude_scaling(*)
         real(c_double), intent(in) :: central_weight(*), compress_P_el(*)
         integer(c_int), intent(in) :: compress_P_i(*), compress_P_j(*)
         character(kind=c_char), intent(in) :: basis(*), scaling_mode(*)
         real(c_double) :: soap(*), soap_cart_der(*)
      end function

      integer(c_int) function tgap_get_soap_energy_and_forces(ctx, n_soap, n_sites, n_sparse, soap, soap_der, &
                                                              alphas, delta, zeta0, e0, Qs, n_neigh, &
                                                              neighbors_list, xyz, n_atom_pairs, do_forces, &
                                                              n_sites0, energies, forces, virial) &
         bind(C, name="tgap_get_soap_energy_and_forces")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         integer(c_int), value :: n_soap, n_sites, n_sparse, n_atom_pairs, do_forces, n_sites0
         real(c_double), intent(in) :: soap(n_soap, *), soap_der(3, n_soap, *), alphas(*), Qs(n_soap, *)
         real(c_double), value :: delta, zeta0, e0
         integer(c_int), intent(in) :: n_neigh(*), neighbors_list(*)
         real(c_double), intent(in) :: xyz(3, *)
         real(c_double) :: energies(*), forces(3, *), virial(3, 3)
      end function

      integer(c_int) function tgap_get_gap_soap(ctx, hypers, n_total_sites, n_sites0, n_neigh0, neighbors_list0, &
                                                rjs0, xyz0, species_supercell, central_species, n_sparse, alphas, &
                                                Qs, delta, zeta, do_forces, precision, energies0, forces0, virial, &
                                                soap_out) bind(C, name="tgap_get_gap_soap")
         import :: c_int, c_ptr, c_double, tgap_soap_hypers
         type(c_ptr), value :: ctx
         type(tgap_soap_hypers), intent(in) :: hypers
         integer(c_int), value :: n_total_sites, n_sites0, central_species, n_sparse, do_forces, precision
         integer(c_int), intent(in) :: n_neigh0(*), neighbors_list0(*), species_supercell(*)
         real(c_double), intent(in) :: rjs0(*), xyz0(3, *), alphas(*), Qs(*)
         real(c_double), value :: delta, zeta
         real(c_double) :: energies0(*), forces0(3, *), virial(3, 3)
         type(c_ptr), value :: soap_out
      end function

      integer(c_int) function tgap_local_property_predict(ctx, n_soap, n_sites, n_sparse, soap, Qs, alphas, &
                                                          V0, delta, zeta, do_derivatives, soap_cart_der, &
                                                          n_neigh, n_atom_pairs, V, V_der) &
         bind(C, name="tgap_local_property_predict")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         integer(c_int), value :: n_soap, n_sites, n_sparse, do_derivatives, n_atom_pairs
         real(c_double), intent(in) :: soap(n_soap, *), Qs(n_soap, *), alphas(*), soap_cart_der(3, n_soap, *)
         real(c_double), value :: V0, delta, zeta
         integer(c_int), intent(in) :: n_neigh(*)
         real(c_double) :: V(*), V_der(3, *)
      end function

      ! resident models and structures (calculate_gap_soap.f90:171 on device-resident state)
      integer(c_int) function tgap_model_create(ctx, hypers, central_species, n_sparse, alphas, Qs, delta, &
                                                zeta, model) bind(C, name="tgap_model_create")
         import :: c_int, c_ptr, c_double, tgap_soap_hypers
         type(c_ptr), value :: ctx
         type(tgap_soap_hypers), intent(in) :: hypers
         integer(c_int), value :: central_species, n_sparse
         real(c_double), intent(in) :: alphas(*), Qs(*)
         real(c_double), value :: delta, zeta
         type(c_ptr), intent(out) :: model
      end function

      ! a model read with compress_soap (read_gap.f90:489-559): compress_P_* as read_gap_hypers fills them
      integer(c_int) function tgap_model_create_compressed(ctx, hypers, central_species, n_sparse, alphas, &
                                                           Qs, delta, zeta, dim_out, P_nonzero, P_i, P_j, &
                                                           P_el, model) &
         bind(C, name="tgap_model_create_compressed")
         import :: c_int, c_ptr, c_double, tgap_soap_hypers
         type(c_ptr), value :: ctx
         type(tgap_soap_hypers), intent(in) :: hypers
         integer(c_int), value :: central_species, n_sparse, dim_out, P_nonzero
         real(c_double), intent(in) :: alphas(*), Qs(*), P_el(*)
         integer(c_int), intent(in) :: P_i(*), P_j(*)
         real(c_double), value :: delta, zeta
         type(c_ptr), intent(out) :: model
      end function

      integer(c_int) function tgap_model_destroy(model) bind(C, name="tgap_model_destroy")
         import :: c_int, c_ptr
         type(c_ptr), value :: model
      end function

      integer(c_int) function tgap_system_create(ctx, n_structures, offsets, positions, boxes, species, &
                                                 rcut_max, system) bind(C, name="tgap_system_create")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         integer(c_int), value :: n_structures
         integer(c_int), intent(in) :: offsets(*), species(*)
         real(c_double), intent(in) :: positions(3, *), boxes(9, *)
         real(c_double), value :: rcut_max
         type(c_ptr), intent(out) :: system
      end function

      integer(c_int) function tgap_system_destroy(system) bind(C, name="tgap_system_destroy")
         import :: c_int, c_ptr
         type(c_ptr), value :: system
      end function

      ! one host-buffer evaluation of a host MD step: positions (c_loc, or c_null_ptr to keep the
      ! resident ones) in, energies, forces and virial out; rebuild = 1 on list-rebuild steps
      integer(c_int) function tgap_calculate_gap_soap(ctx, system, n_models, models, precision, positions, &
                                                      rebuild, energies, forces, virial) &
         bind(C, name="tgap_calculate_gap_soap")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx, system, positions
         integer(c_int), value :: n_models, precision, rebuild
         type(c_ptr), intent(in) :: models(*)
         real(c_double), intent(out) :: energies(*), forces(3, *), virial(9, *)
      end function

      ! calculate_e0 (calculate_gap_soap.f90:135-169) on a resident system: species_info%e0(1:n_species)
      integer(c_int) function tgap_system_set_e0(system, n_species, e0) bind(C, name="tgap_system_set_e0")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: system
         integer(c_int), value :: n_species
         real(c_double), intent(in) :: e0(*)
      end function

      ! split_tasks (misc.f90:88-111): this rank's sites are split%i_beg .. split%i_end, passed as
      ! the 0-based half-open range (i_beg - 1, i_end)
      integer(c_int) function tgap_system_set_site_range(system, beg, end) bind(C, name="tgap_system_set_site_range")
         import :: c_int, c_ptr
         type(c_ptr), value :: system
         integer(c_int), value :: beg, end
      end function

      ! velocity_verlet (md_utils.f90:486-532) on device arrays (CUDA Fortran device memory or
      ! OpenACC host_data use_device), after the ranks' forces have been summed
      integer(c_int) function tgap_velocity_verlet(ctx, n_sites, positions, positions_prev, velocities, &
                                                   forces, forces_prev, masses, dt, dt_prev, first_step) &
         bind(C, name="tgap_velocity_verlet")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx, positions, positions_prev, velocities, forces, forces_prev, masses
         integer(c_int), value :: n_sites, first_step
         real(c_double), value :: dt, dt_prev
      end function

      ! the same update on host arrays, for a host MD loop around tgap_calculate_gap_soap
      integer(c_int) function tgap_velocity_verlet_host(n_sites, positions, positions_prev, velocities, &
                                                        forces, forces_prev, masses, dt, dt_prev, first_step) &
         bind(C, name="tgap_velocity_verlet_host")
         import :: c_int, c_double, c_ptr
         integer(c_int), value :: n_sites, first_step
         real(c_double), intent(inout) :: positions(3, *), velocities(3, *), forces_prev(3, *)
         type(c_ptr), value :: positions_prev
         real(c_double), intent(in) :: forces(3, *), masses(*)
         real(c_double), value :: dt, dt_prev
      end function
   end interface

contains

   ! Drop-in body for get_soap_energy_and_forces (gap.f90:39-41 argument list).
   subroutine tgap_soap_energy_and_forces_f(ctx, soap, soap_der, alphas, delta, zeta0, e0, Qs, &
                                            n_neigh, neighbors_list, xyz, do_forces, energies, forces, virial)
      type(c_ptr), intent(in) :: ctx
      real(c_double), intent(in) :: soap(:, :), soap_der(:, :, :), alphas(:), delta, zeta0, e0, Qs(:, :)
      integer, intent(in) :: n_neigh(:), neighbors_list(:)
      real(c_double), intent(in) :: xyz(:, :)
      logical, intent(in) :: do_forces
      real(c_double), intent(out) :: energies(:), forces(:, :), virial(3, 3)
      integer(c_int) :: st
      st = tgap_get_soap_energy_and_forces(ctx, size(soap, 1), size(soap, 2), size(alphas), soap, soap_der, &
                                           alphas, delta, zeta0, e0, Qs, n_neigh, neighbors_list, xyz, &
                                           sum(n_neigh), merge(1, 0, do_forces), size(forces, 2), energies, &
                                           forces, virial)
      if (st /= TGAP_OK) then
         write (*, *) "tgap_get_soap_energy_and_forces failed with status", st
         stop
      end if
   end subroutine

   ! Drop-in body for local_property_predict (local_properties.f90:46-50 argument list).
   subroutine tgap_local_property_predict_f(ctx, soap, Qs, alphas, V0, delta, zeta, V, do_derivatives, &
                                            soap_cart_der, n_neigh, V_der)
      type(c_ptr), intent(in) :: ctx
      real(c_double), intent(in) :: soap(:, :), Qs(:, :), alphas(:), V0, delta, zeta, soap_cart_der(:, :, :)
      integer, intent(in) :: n_neigh(:)
      logical, intent(in) :: do_derivatives
      real(c_double), intent(out) :: V(:), V_der(:, :)
      integer(c_int) :: st
      st = tgap_local_property_predict(ctx, size(soap, 1), size(soap, 2), size(alphas), soap, Qs, alphas, V0, &
                                       delta, zeta, merge(1, 0, do_derivatives), soap_cart_der, n_neigh, &
                                       sum(n_neigh), V, V_der)
      if (st /= TGAP_OK) then
         write (*, *) "tgap_local_property_predict failed with status", st
         stop
      end if
   end subroutine

end module tgap_iface
