/*
 * ORACLE — test infrastructure only.
 *
 * CPU (FP64) restatement of the TurboGAP SOAP/GAP energy-and-force path, used by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / --impl reference
 * leg as the checker. Nothing in the product links, imports or calls this code.
 *
 * Sources restated (reference paths are relative to the TurboGAP project root):
 *   neighbors  : src/neighbors/neighbors_interface.f90:144-524 (build_neighbors_list),
 *                :547-643 (get_distance), :655-708 (number_of_unit_cells_for_given_cutoff)
 *   supercell  : src/xyz/read_xyz.f90:323-373 (set_supercell)
 *   subset     : src/gap/gap_interface.f90:162-289 (get_gap_soap site/pair renumbering)
 *   GAP        : src/gap/gap.f90:39-244 (get_soap_energy_and_forces)
 *   dynamics   : src/md/md_utils.f90:486-532 (velocity_verlet),
 *                src/mc/mc_utils.f90:172-180,215-257 (monte_carlo_move, get_mc_acceptance)
 *   descriptor : soap_turbo get_soap (argument list at src/gap/gap_interface.f90:301-306);
 *                the soap_turbo submodule (libAtoms/soap_turbo, no pinned commit) is absent,
 *                so the descriptor is restated from the published method (M. A. Caro,
 *                Phys. Rev. B 100, 024112 (2019)). Parity against soap_turbo is UNPINNED.
 *
 * Conventions follow the Fortran call surface: arrays are column-major with the first
 * index fastest, neighbor ids are 1-based supercell indices, the first pair slot of
 * every site is the site itself (r = 0).
 */
#ifndef TGAP_ORACLE_H
#define TGAP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- neighbors ---------------- */

/* neighbors_interface.f90:547-643. PBC is always full here (the only mode the hot path uses). */
void orc_get_distance(const double posi[3], const double posj[3], const double a[3],
                      const double b[3], const double c[3], double dist[3], double *d,
                      int i_shift[3]);

/* neighbors_interface.f90:655-708 */
void orc_number_of_unit_cells(const double a[3], const double b[3], const double c[3],
                              double rcut, int indices[3]);

/* read_xyz.f90:323-373. pos_sc must hold 3*n_sites*prod(indices). Box vectors are scaled
 * in place by indices. species_sc receives the replicated species. */
void orc_set_supercell(int n_sites, const double *pos, const int *species,
                       const int indices[3], double a[3], double b[3], double c[3],
                       double *pos_sc, int *species_sc);

/* build_neighbors_list (neighbors_interface.f90:144-524), rebuild = .true., single rank.
 * Pass 1: returns the number of pairs (including self slots) when neighbors_list == NULL.
 * Pass 2: fills every output array (capacity >= returned count).
 * box_small: any(indices > 1) (the caller's supercell state, read_xyz.f90:133-147).
 * Returns -1 on an unsupported lattice. */
int64_t orc_build_neighbors(int n_sites, int n_sites_supercell, const double *positions,
                            double a[3], double b[3], double c[3], int box_small,
                            double rcut_max, const int *species_supercell, int *n_neigh,
                            int *neighbors_list, double *rjs, double *xyz, double *thetas,
                            double *phis, int *neighbor_species);

/* Geometry refresh only (build_neighbors_list with rebuild = .false., :445-510). */
void orc_neighbor_geometry(int n_sites, const double *positions, const double a[3],
                           const double b[3], const double c[3], const int *n_neigh,
                           const int *neighbors_list, const int *species_supercell,
                           double *rjs, double *xyz, double *thetas, double *phis,
                           int *neighbor_species);

/* ---------------- SOAP descriptor ---------------- */

typedef struct {
    int n_species;
    const int *alpha_max;               /* [n_species] */
    int l_max;
    const double *rcut_hard;            /* [n_species] */
    const double *rcut_soft;
    const double *nf;
    const double *global_scaling;
    const double *atom_sigma_r;
    const double *atom_sigma_r_scaling;
    const double *atom_sigma_t;
    const double *atom_sigma_t_scaling;
    const double *amplitude_scaling;
    const double *central_weight;
    int radial_enhancement;             /* 0, 1 or 2 */
    /* SOAP compression (read_gap.f90:489-559, the P_transformation of file_compress_soap): the
     * descriptor is P p / |P p| with p the uncompressed power spectrum and P sparse, given as
     * n_compress entries (compress_P_i, compress_P_j 1-based, compress_P_el) and dim_out rows;
     * n_compress = 0: no compression. */
    int n_compress;
    int dim_out;
    const int *compress_P_i;
    const int *compress_P_j;
    const double *compress_P_el;
} orc_soap_hypers;

/* Length of the descriptor: dim_out with compression, else n_max (n_max+1)/2 (l_max+1),
 * n_max = sum alpha_max. */
int orc_soap_dim(const orc_soap_hypers *h);

/* Quadrature tables for one species channel (exposed for the known-answer tests).
 * Returns the number of nodes; xq/tq receive node positions (in units of rcut_hard) and
 * the weighted orthonormal basis values tq[q*alpha_max + n] (filter folded in). */
int orc_radial_nodes(const orc_soap_hypers *h, int s, double *xq, double *tq, int cap);

/* Orthonormalisation matrix W = S^{-1/2} of the poly3 basis (alpha x alpha, computed in
 * binary128 and rounded). */
void orc_poly3_w(int alpha_max, double *W);

/* Radial coefficients R_n(r) and dR_n/dr of channel s for one neighbor distance r (Å).
 * central != 0 evaluates the central-atom term (r = 0, central_weight applied). */
void orc_radial(const orc_soap_hypers *h, int s, double r, int central, double *R, double *dR);

/* Angular factors f_l(r) Y_lm(u) ((l_max+1)^2 values) and their gradient (3 per value)
 * with respect to the neighbor vector r u, for channel s. */
void orc_angular(const orc_soap_hypers *h, int s, double r, const double u[3], double *A,
                 double *dA);

/* get_soap (gap_interface.f90:301-306 argument order; compression as the hypers give it).
 * mask is n_atom_pairs x n_species (column-major, nonzero = neighbor belongs to channel).
 * soap: D x n_sites (normalised). soap_cart_der: 3 x D x n_atom_pairs, or NULL. */
int orc_get_soap(const orc_soap_hypers *h, int n_sites, const int *n_neigh,
                 int n_atom_pairs, const unsigned char *mask, const double *rjs,
                 const double *thetas, const double *phis, double *soap,
                 double *soap_cart_der);

/* ---------------- GAP ---------------- */

/* get_soap_energy_and_forces (gap.f90:39-244). forces has n_sites0 columns (fold modulus). */
void orc_get_soap_energy_and_forces(int n_soap, int n_sites, int n_sparse, const double *soap,
                                    const double *soap_der, const double *alphas, double delta,
                                    double zeta0, double e0, const double *Qs,
                                    const int *n_neigh, const int *neighbors_list,
                                    const double *xyz, int do_forces, int n_sites0,
                                    double *energies, double *forces, double *virial);

/* local_property_predict (local_properties.f90:46-147): V (n_sites) = delta^2 K^zeta alphas + V0
 * clipped at zero; with do_derivatives, V_der (3 x n_pairs) = Qss(i,:) . soap_cart_der(:,:,j). */
void orc_local_property_predict(int n_soap, int n_sites, int n_sparse, const double *soap, const double *Qs,
                                 const double *alphas, double V0, double delta, double zeta, int do_derivatives,
                                 const double *soap_cart_der, const int *n_neigh, double *V, double *V_der);

/* get_2b_energy_and_forces (gap.f90:329-460): species given as channel indices (sp1, sp2 the
 * pair's); energies = e0 + the pair terms of each site, forces on the sites, half pair virial. */
void orc_get_2b_energy_and_forces(int n_sites, const double *rjs, const double *xyz, int n_sparse,
                                  const double *alphas, const double *cutoff, double rcut, double buffer,
                                  double delta, double sigma, double e0, const double *Qs, const int *n_neigh,
                                  int do_forces, const int *species, const int *neighbor_species, int sp1, int sp2,
                                  int n_sites0, double *energies, double *forces, double *virial);
/* get_core_pot_energy_and_forces (gap.f90:552-686) with the cubic spline of splines.f90:33-156. */
void orc_get_core_pot_energy_and_forces(int n_sparse, int n_sites, int n_sites0, const double *rjs,
                                        const double *xyz, const double *x, const double *V, double yp1,
                                        double ypn, const double *dVdx2, const int *n_neigh, int do_forces,
                                        const int *species, const int *neighbor_species, int sp1, int sp2,
                                        double *energies, double *forces, double *virial);

/* get_3b_energy_and_forces (gap.f90:756-1015): angle_3b GAP on triplets (i; j < k) of each
 * species_center site; kernel_pol 0: "exp", 1: "pol" (cov_pp, d = 3, q = 1); Qs (n_sparse x 3,
 * column-major), sigma[3]; forces (3 x n_sites0) on the folded triplet atoms. */
void orc_get_3b_energy_and_forces(int n_sites0, int n_sites, const double *rjs, const double *xyz, int n_sparse,
                                  const double *alphas, const double *cutoff, double rcut, double buffer,
                                  double delta, const double *sigma, double e0, const double *Qs,
                                  const int *n_neigh, const int *neighbors_list, int do_forces, int kernel_pol,
                                  const int *species, const int *neighbor_species, int sp0, int sp1, int sp2,
                                  double *energies, double *forces, double *virial);

/* get_gap_soap (gap_interface.f90:41-433) for one SOAP model on the global neighbor list:
 * subset by rcut/species, central-species filter, get_soap, energies/forces, scatter back.
 * species_supercell: species channel (1..n_species) per supercell atom, 0 = blind.
 * energies0 (n_total_sites) / forces0 (3 x n_total_sites) are overwritten for touched sites. */
int orc_get_gap_soap(const orc_soap_hypers *h, int n_total_sites, int n_sites0,
                     const int *n_neigh0, const int *neighbors_list0, const double *rjs0,
                     const double *thetas0, const double *phis0, const double *xyz0,
                     const int *species_supercell, int central_species, int n_sparse,
                     const double *alphas, const double *Qs, double delta, double zeta,
                     int do_forces, double *energies0, double *forces0, double *virial);

/* ---------------- dynamics ---------------- */

/* velocity_verlet (md_utils.f90:486-532), no fixed atoms. */
void orc_velocity_verlet(int n_sites, double *positions, double *positions_prev,
                         double *velocities, const double *forces, double *forces_prev,
                         const double *masses, double dt, double *dt_prev, int first_step);

/* monte_carlo_move (mc_utils.f90:172-180) with min(1, p) of get_mc_acceptance (:255).
 * kB is the reference's default-real literal 8.617333262e-5 (rounded to binary32). */
double orc_mc_move_acceptance(double e_new, double e_prev, double temp);

/* calculate_e0 (calculate_gap_soap.f90:135-169): per-site e0 by species channel. */
void orc_calculate_e0(int n_sites, const int *species, int n_species, const double *e0, double *energies_e0);

/* Thread count used by the OpenMP regions (for the CPU baseline). */
int orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
