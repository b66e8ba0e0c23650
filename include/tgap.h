/*
 * tgap.h — C ABI of the B200 (sm_100a) SOAP/GAP energy-and-force path.
 *
 * Drop-in boundary for the TurboGAP `predict` / `md` / `mc` hot path. The first group of
 * entry points mirrors, argument for argument, the Fortran routines a TurboGAP build calls
 * (the Fortran side binds them with ISO_C_BINDING; see fortran/tgap_iface.f90 in the package):
 *
 *   tgap_build_neighbors            build_neighbors_list   src/neighbors/neighbors_interface.f90:144
 *   tgap_number_of_unit_cells       number_of_unit_cells_for_given_cutoff  neighbors_interface.f90:655
 *   tgap_get_soap                   soap_turbo get_soap    (call site src/gap/gap_interface.f90:301-306)
 *   tgap_get_soap_energy_and_forces get_soap_energy_and_forces  src/gap/gap.f90:39
 *   tgap_get_gap_soap               get_gap_soap           src/gap/gap_interface.f90:41
 *
 * These take HOST arrays in Fortran layout (column-major, first index fastest, neighbor ids
 * 1-based supercell indices, self first in every site's neighbor block) and copy to and
 * from the device inside the call.
 *
 * The second group keeps models, structures and MD state resident in HBM (device-pointer
 * interface, no host copies) for the MD/MC drivers and batched evaluation.
 *
 * Conventions: every entry point returns a tgap_status (0 = success) and never aborts.
 * Output capacities are passed in; a too-small capacity returns TGAP_ERR_CAPACITY and
 * writes the required size (mirrors the grow-on-demand of check_extend_neighbor_list,
 * neighbors_interface.f90:526-540). A context owns its device buffers and one CUDA stream;
 * calls on one context are not thread-safe.
 */
#ifndef TGAP_H
#define TGAP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    TGAP_OK = 0,
    TGAP_ERR_ARGUMENT = 1,     /* bad size, null pointer, inconsistent dimensions */
    TGAP_ERR_CUDA = 2,         /* a CUDA runtime call failed (message: tgap_last_error) */
    TGAP_ERR_CAPACITY = 3,     /* output capacity too small; required size written back */
    TGAP_ERR_HYPERS = 4,       /* unsupported descriptor hyperparameters */
    TGAP_ERR_TIMEOUT = 5,      /* a bounded device wait gave up */
    TGAP_ERR_UNSUPPORTED = 6,  /* valid in the reference, not implemented on this path */
    TGAP_ERR_NOMEM = 7,        /* device allocation failed */
    TGAP_ERR_NUMERIC = 8       /* non-finite input or result detected */
} tgap_status;

typedef enum { TGAP_FP64 = 0, TGAP_MIXED = 1 } tgap_precision;

typedef struct tgap_context tgap_context;

/* ------------------------------------------------------------------ context */

int tgap_create(int device, tgap_context **ctx);
int tgap_destroy(tgap_context *ctx);
/* Page-locks and maps the caller's host memory [ptr, ptr + bytes) (cudaHostRegister, mapped) for this
 * context: the host-buffer entries (tgap_calculate_gap_soap) then read positions from and write
 * results to such arrays directly, by a copy kernel over their device addresses, instead of through
 * the context's staging buffers. For arrays reused across calls; unregister before freeing them
 * (unregistering synchronizes the context stream). */
int tgap_host_register(tgap_context *ctx, void *ptr, size_t bytes);
int tgap_host_unregister(tgap_context *ctx, void *ptr);
/* Use an external stream (cudaStream_t) for all later work; NULL restores the own stream. */
int tgap_set_stream(tgap_context *ctx, void *stream);
int tgap_synchronize(tgap_context *ctx);
/* Message of the last failed call on ctx; with ctx == NULL, of the last failed context-free call
 * (tgap_soap_energies_noalloc) made by the calling host thread. */
const char *tgap_last_error(const tgap_context *ctx);
const char *tgap_version(void);
/* Number of kernels this library launched on ctx since creation (instrumentation). */
int64_t tgap_kernel_launches(const tgap_context *ctx);
/* Stage timing (the tracing counterpart of the reference's time_start/time_end,
 * src/utils/timing.f90:117-131): when enabled, CUDA events bracket every kernel stage on the
 * context stream (outside graph capture). tgap_timing_report synchronizes and returns up to
 * `cap` stages: names (32 chars each, NUL padded), total milliseconds and launch counts. */
int tgap_timing_enable(tgap_context *ctx, int enable);
int tgap_timing_reset(tgap_context *ctx);
int tgap_timing_report(tgap_context *ctx, int cap, char *names, double *total_ms,
                       int64_t *counts, int *n_stages);

/* ------------------------------------------------------------------ reference call surface */

/* neighbors_interface.f90:655-708: replicas per lattice vector so that the cell's planes are
 * at least 2*rcut apart. Pure host arithmetic. */
int tgap_number_of_unit_cells(const double a_box[3], const double b_box[3],
                              const double c_box[3], double rcut, int indices[3]);

/* build_neighbors_list (neighbors_interface.f90:144-524), single rank, all sites owned.
 *  positions           3 x n_sites_supercell (supercell already replicated, read_xyz.f90:323)
 *  box_small           any(indices > 1): the brute-force path is used, as in the reference
 *  rebuild             1: build the list; 0: keep n_neigh/neighbors_list (inputs) and only
 *                      refresh rjs/xyz/thetas/phis/neighbor_species (:445-510)
 *  capacity            length of neighbors_list and of the per-pair outputs
 *  n_atom_pairs        in/out: pairs written (or required, with TGAP_ERR_CAPACITY)
 * Pair lists are bit-identical to the reference ordering (cell traversal z->y->x with LIFO
 * cells, or ascending supercell index on the brute-force path). */
int tgap_build_neighbors(tgap_context *ctx, int n_sites, int n_sites_supercell,
                         const double *positions, const double a_box[3], const double b_box[3],
                         const double c_box[3], int box_small, double rcut_max,
                         const int *species_supercell, int rebuild, int *n_neigh,
                         int *neighbors_list, double *rjs, double *xyz, double *thetas,
                         double *phis, int *neighbor_species, int64_t capacity,
                         int64_t *n_atom_pairs);

/* soap_turbo get_soap, argument order of gap_interface.f90:301-306 (do_timing dropped).
 *  species              max_species_multiplicity x n_sites (only multiplicity 1 supported)
 *  mask                 n_atom_pairs x n_species, nonzero = neighbor belongs to the channel
 *  basis                "poly3" (poly3gauss: TGAP_ERR_UNSUPPORTED)
 *  scaling_mode         "polynomial"
 *  compress_soap        with compress_P_* (1-based entries): the descriptor is P p / |P p|
 *                       (read_gap.f90:489-559), n_soap = the largest P_i
 *  soap                 out, n_soap x n_sites (normalised q; n_soap the descriptor length,
 *                       the compressed one with compress_soap)
 *  soap_cart_der        out, 3 x n_soap x n_atom_pairs (dq_i/dr_j; self slot = -sum), or NULL
 *                       when do_derivatives == 0 */
int tgap_get_soap(tgap_context *ctx, int n_sites, const int *n_neigh, int n_species,
                  const int *species, const int *species_multiplicity, int n_atom_pairs,
                  const unsigned char *mask, const double *rjs, const double *thetas,
                  const double *phis, const int *alpha_max, int l_max,
                  const double *rcut_hard, const double *rcut_soft, const double *nf,
                  const double *global_scaling, const double *atom_sigma_r,
                  const double *atom_sigma_r_scaling, const double *atom_sigma_t,
                  const double *atom_sigma_t_scaling, const double *amplitude_scaling,
                  int radial_enhancement, const double *central_weight, const char *basis,
                  const char *scaling_mode, int do_derivatives, int compress_soap,
                  int compress_P_nonzero, const int *compress_P_i, const int *compress_P_j,
                  const double *compress_P_el, double *soap, double *soap_cart_der);

/* get_soap_energy_and_forces (gap.f90:39-244).
 *  soap (n_soap x n_sites), soap_der (3 x n_soap x n_atom_pairs), Qs (n_soap x n_sparse)
 *  forces (3 x n_sites0): n_sites0 is the fold modulus of neighbors_list (gap.f90:118,196)
 *  virial (3 x 3) */
int tgap_get_soap_energy_and_forces(tgap_context *ctx, int n_soap, int n_sites, int n_sparse,
                                    const double *soap, const double *soap_der,
                                    const double *alphas, double delta, double zeta0,
                                    double e0, const double *Qs, const int *n_neigh,
                                    const int *neighbors_list, const double *xyz,
                                    int n_atom_pairs, int do_forces, int n_sites0,
                                    double *energies, double *forces, double *virial);

/* local_property_predict (src/gap/local_properties.f90:46-147): a per-site property model (e.g.
 * Hirshfeld volumes), V(i) = delta^2 sum_s alphas(s) K(i,s)^zeta + V0 clipped at 0, zeta taken as
 * an integer when nint(zeta) is within 1e-10 (:76-77). With do_derivatives, V_der (3 x
 * n_atom_pairs) = Qss(i,:) . soap_cart_der(:,:,j) for every pair j of site i, zero for a site whose
 * V was clipped. soap (n_soap x n_sites), Qs (n_soap x n_sparse), soap_cart_der (3 x n_soap x
 * n_atom_pairs) as get_soap gives them. FP64. */
int tgap_local_property_predict(tgap_context *ctx, int n_soap, int n_sites, int n_sparse,
                                const double *soap, const double *Qs, const double *alphas,
                                double V0, double delta, double zeta, int do_derivatives,
                                const double *soap_cart_der, const int *n_neigh, int n_atom_pairs,
                                double *V, double *V_der);

/* No counterpart in the reference. Per-site GAP energies delta^2 sum_s alpha_s (q_i.Q_s)^zeta
 * + e0 (the energy half of get_soap_energy_and_forces) for inputs that are already on the
 * device, without allocating any device memory.
 *
 * Who needs it: host programs that only hold device memory handed to them by someone else, for
 * example a Fortran MD/MC driver whose arrays live in an OpenACC or CUDA Fortran data region, or
 * a code that sizes one memory pool at start-up and may not create allocations of its own in
 * its inner loop (cudaMalloc/cudaFree there can synchronize the whole device or fail when the
 * pool has taken the memory). The MC driver, which asks for energies only, is the typical caller.
 *
 * How: the only scratch the computation needs (per-tile energy partials) is a fixed array of
 * 2^20 doubles (8 MiB) compiled into the library, so every GPU that loads libtgap reserves it
 * until the process exits. Limit: n_sites * ceil(n_sparse / 64) <= 1048576, otherwise
 * TGAP_ERR_CAPACITY is returned and nothing runs. The array is shared by all calls: every entry
 * that is read is first written by the same call, so nothing has to start at zero, but calls
 * whose work overlaps on the GPU (other streams, other host threads) race on it and must be
 * serialized by the caller. The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current and keeps it for later calls; make that first
 * call before any stream capture. The kept address belongs to the device's primary context: after
 * a cudaDeviceReset of that device, do not call this entry again in the same process.
 * `stream` (a cudaStream_t, NULL = default stream) must belong to the current device, otherwise
 * TGAP_ERR_ARGUMENT; the scratch address used is the current device's. Pointers are device
 * pointers in the layout of tgap_get_soap_energy_and_forces (d_soap: n_soap x n_sites, d_Qs:
 * n_soap x n_sparse, d_alphas: n_sparse, d_energies: n_sites, overwritten). The call does not
 * synchronize; its status covers its own launches (an error left pending by earlier work on the
 * device is neither reported nor cleared), and a failure leaves a message for
 * tgap_last_error(NULL). */
int tgap_soap_energies_noalloc(void *stream, int n_soap, int n_sites, int n_sparse,
                               const double *d_soap, const double *d_alphas, double delta,
                               double zeta0, double e0, const double *d_Qs, double *d_energies);

/* Descriptor hyperparameters of one soap_turbo model (read_gap.f90:156-432), per species. */
typedef struct {
    int n_species;
    const int *alpha_max;
    int l_max;
    const double *rcut_hard, *rcut_soft, *nf, *global_scaling;
    const double *atom_sigma_r, *atom_sigma_r_scaling, *atom_sigma_t, *atom_sigma_t_scaling;
    const double *amplitude_scaling, *central_weight;
    int radial_enhancement;
} tgap_soap_hypers;

/* get_gap_soap (gap_interface.f90:41-433) for one model on the global neighbor list:
 * subset (rjs < max rcut_hard, species known), central-species filter, descriptor,
 * energies/forces/virial, scatter back to global indices.
 *  species_supercell    species channel 1..n_species per supercell atom (0 = not seen by the
 *                       model); tgap_assign_species maps character*8 names to it
 *  energies0 (n_total_sites), forces0 (3 x n_total_sites): overwritten for touched sites
 *  soap_out             optional (NULL), n_soap x n_sites0 (write_soap, :391-401)
 *  precision            TGAP_FP64 or TGAP_MIXED
 * Forces are computed without materialising dq/dr (adjoint back-scatter). */
int tgap_get_gap_soap(tgap_context *ctx, const tgap_soap_hypers *hypers, int n_total_sites,
                      int n_sites0, const int *n_neigh0, const int *neighbors_list0,
                      const double *rjs0, const double *xyz0, const int *species_supercell,
                      int central_species, int n_sparse, const double *alphas,
                      const double *Qs, double delta, double zeta, int do_forces,
                      int precision, double *energies0, double *forces0, double *virial,
                      double *soap_out);

/* assign_species_multiplicity (soap_turbo; call site gap_interface.f90:175): map Fortran
 * character*8 species names to channel ids. species_types: n_species x 8 chars, names:
 * n x 8 chars (blank padded). out: channel 1..n_species, 0 if absent. Duplicated
 * species_types (multiplicity > 1) returns TGAP_ERR_UNSUPPORTED. */
int tgap_assign_species(int n_species, const char *species_types, int n, const char *names,
                        int *out);

/* ------------------------------------------------------------------ resident (device) API */

typedef struct tgap_model tgap_model;
typedef struct tgap_system tgap_system;

/* One soap_turbo GAP model resident on the device. Qs: n_soap x n_sparse (Fortran layout,
 * read_gap.f90:810-827). central_species: 0 = all sites. */
int tgap_model_create(tgap_context *ctx, const tgap_soap_hypers *hypers, int central_species,
                      int n_sparse, const double *alphas, const double *Qs, double delta,
                      double zeta, tgap_model **model);
/* The same with SOAP compression (read_gap.f90:489-559, the P_transformation of a
 * file_compress_soap): the descriptor is P p / |P p|, p the uncompressed power spectrum in the
 * component order of tgap_get_soap (n <= n', then l) and P a sparse dim_out x dim matrix given as
 * P_nonzero entries (P_i in 1..dim_out, P_j in 1..dim, 1-based; entries of one row or column are
 * summed in the order given). Qs: dim_out x n_sparse. The old index-list format is P_i = i,
 * P_el = 1. A compress_mode recipe (soap_turbo's get_compress_indices, not in the reference
 * sources) is not available. */
int tgap_model_create_compressed(tgap_context *ctx, const tgap_soap_hypers *hypers, int central_species,
                                 int n_sparse, const double *alphas, const double *Qs, double delta,
                                 double zeta, int dim_out, int P_nonzero, const int *P_i, const int *P_j,
                                 const double *P_el, tgap_model **model);
int tgap_model_destroy(tgap_model *model);
int tgap_model_dim(const tgap_model *model);

/* A batch of periodic structures resident on the device. Structure b holds atoms
 * [offsets[b], offsets[b+1]); boxes: 9 doubles per structure (rows a, b, c); species:
 * channel ids. Small cells are replicated internally (read_xyz.f90:323-373). */
int tgap_system_create(tgap_context *ctx, int n_structures, const int *offsets,
                       const double *positions, const double *boxes, const int *species,
                       double rcut_max, tgap_system **system);
int tgap_system_destroy(tgap_system *system);
int tgap_system_n_atoms(const tgap_system *system);
/* Device pointer to the 3 x n_atoms positions (read/write, layout as on input). */
int tgap_system_positions(tgap_system *system, double **d_positions);
/* Copy the resident positions (3 x n_atoms) to the host (synchronizes the context stream). */
int tgap_system_get_positions(tgap_system *system, double *positions);
/* Copy host positions (3 x n_atoms) into the resident structure. */
int tgap_system_set_positions(tgap_system *system, const double *positions);
/* Rebuild the neighbor lists (or only refresh geometry when rebuild == 0). */
int tgap_system_update(tgap_system *system, int rebuild);
/* Pairs in the current lists (self entries included). After an MD run has rebuilt the lists on the
   device this reads the count back (synchronizes the context stream); -1 on a CUDA error. */
int64_t tgap_system_n_pairs(const tgap_system *system);

/* calculate_e0 (src/gap/calculate_gap_soap.f90:135-169): isolated-atom energies per species
 * channel, e0[c - 1] for channel c = 1..n_species (the input file's `e0` keyword,
 * src/read/read_files.f90:380-385). Every later energy output of the system (tgap_compute,
 * tgap_calculate_gap_soap, the MD potential energy, the MC state) adds each atom's e0, as
 * turbogap_main.f90:993-994 adds energies_e0 to the total; atoms of a channel outside 1..n_species
 * get 0. Set it before creating MD objects on the system, or call it again with the same
 * n_species to change the values. Forces, virials and MC energy differences are unaffected. */
int tgap_system_set_e0(tgap_system *system, int n_species, const double *e0);

/* split_tasks (src/utils/misc.f90:88-111) for one rank of an atom decomposition: only atoms
 * [beg, end) (0-based; end < 0 = n_atoms) are descriptor centres of later evaluations of the
 * system. Energies of the other atoms come out 0; forces and virials hold the range's
 * contributions on every atom its sites see (the pair lists still cover all atoms), so summing the
 * outputs of ranks whose ranges partition the atoms gives the full result, as collect_calculation
 * (src/mpi/mpi_utils.f90:515-545) sums the MPI ranks. e0 (tgap_system_set_e0) is added for the range
 * only. Monte Carlo objects need every site. */
int tgap_system_set_site_range(tgap_system *system, int beg, int end);

/* velocity_verlet (src/md/md_utils.f90:486-532) on device arrays (3 x n_sites each, masses in
 * eV fs^2 / A^2 as md_interface.f90 keeps them): v += 0.5 (F + F_prev) / m dt_prev unless
 * first_step, x_prev = x, x += v dt + 0.5 F / m dt^2, F_prev = F. For drivers that assemble the
 * forces themselves, e.g. summed over the ranks of an atom decomposition. */
int tgap_velocity_verlet(tgap_context *ctx, int n_sites, double *d_positions, double *d_positions_prev,
                         double *d_velocities, const double *d_forces, double *d_forces_prev,
                         const double *d_masses, double dt, double dt_prev, int first_step);
/* The same update on host arrays (one pass over the atoms with one reciprocal mass per atom, so it
 * agrees with the divided form to an ulp), for host-side MD loops around tgap_calculate_gap_soap,
 * where the reference integrates on the host.
 * positions_prev may be NULL. Non-finite forces return TGAP_ERR_NUMERIC before any array changes. */
int tgap_velocity_verlet_host(int n_sites, double *positions, double *positions_prev, double *velocities,
                              const double *forces, double *forces_prev, const double *masses, double dt,
                              double dt_prev, int first_step);

/* Energies (n_atoms), forces (3 x n_atoms) and virial (9 per structure), device pointers,
 * summed over models, plus each atom's e0 (tgap_system_set_e0; 0 when never set). Overwrites the
 * outputs. */
int tgap_compute(tgap_context *ctx, tgap_system *system, int n_models,
                 tgap_model *const *models, int precision, int do_forces, double *d_energies,
                 double *d_forces, double *d_virial);

/* get_2b_energy_and_forces (src/gap/gap.f90:329-460): the distance_2b GAP between species1 and
 * species2 (channel indices, as tgap_assign_species maps the reference's character*8 names) on a
 * full neighbor list (self first in each site's block, as build_neighbors_list writes it). Per
 * site energies = e0 + sum over its pairs of delta^2 alphas(s) cutoff(s) fcut(r) exp(-(r - Qs(s))^2
 * / 2 sigma^2), fcut the cosine taper over [rcut - buffer, rcut]; forces (3 x n_sites0, overwritten)
 * on the sites only; virial (3 x 3) half the pair virial. FP64. */
int tgap_get_2b_energy_and_forces(tgap_context *ctx, int n_sites, int n_atom_pairs, const double *rjs,
                                  const double *xyz, int n_sparse, const double *alphas,
                                  const double *cutoff, double rcut, double buffer, double delta,
                                  double sigma, double e0, const double *Qs, const int *n_neigh,
                                  int do_forces, const int *species, const int *neighbor_species,
                                  int species1, int species2, int n_sites0, double *energies,
                                  double *forces, double *virial);
/* get_core_pot_energy_and_forces (src/gap/gap.f90:552-686): tabulated pair potential V(x) on an
 * increasing grid x (n_sparse points) with precomputed spline second derivatives dVdx2 and end
 * slopes yp1 / ypn, evaluated as the cubic spline of src/utils/splines.f90:33-156 for pairs with
 * r < max(x); energies = 1/2 V per pair of each site, forces on the sites, half pair virial. FP64. */
int tgap_get_core_pot_energy_and_forces(tgap_context *ctx, int n_sparse, int n_sites, int n_atom_pairs,
                                        int n_sites0, const double *rjs, const double *xyz,
                                        const double *x, const double *V, double yp1, double ypn,
                                        const double *dVdx2, const int *n_neigh, int do_forces,
                                        const int *species, const int *neighbor_species, int species1,
                                        int species2, double *energies, double *forces, double *virial);

/* get_3b_energy_and_forces (src/gap/gap.f90:756-1015): the angle_3b GAP on the triplets (i; j < k)
 * of each species_center site with neighbors of species1 and species2 inside rcut, descriptor
 * q = (r_ij + r_ik, (r_ij - r_ik)^2, r_jk), kernel_type 0 "exp" or 1 "pol" (cov_pp, d = 3, q = 1,
 * :1022-1081); Qs is n_sparse x 3 (column-major), sigma[3]. Energies = e0 + the triplet terms of
 * each site; forces (3 x n_sites0, overwritten) on the three atoms of each triplet, folded with
 * mod(neighbors_list - 1, n_sites0); virial from the arms ij and ik. At most 512 eligible pairs per
 * site. FP64. */
int tgap_get_3b_energy_and_forces(tgap_context *ctx, int n_sites0, int n_sites, int n_atom_pairs,
                                  const double *rjs, const double *xyz, int n_sparse,
                                  const double *alphas, const double *cutoff, double rcut, double buffer,
                                  double delta, const double *sigma, double e0, const double *Qs,
                                  const int *n_neigh, const int *neighbors_list, int do_forces,
                                  int kernel_type, const int *species, const int *neighbor_species,
                                  int species_center, int species1, int species2, double *energies,
                                  double *forces, double *virial);

/* Resident form of local_property_predict (local_properties.f90:46-147, as get_gap_soap calls it,
 * gap_interface.f90:314-364) for a property model held as a tgap_model (its delta, zeta, alphas
 * and sparse set; the integer-zeta test of local_properties.f90): device pointers d_V (n_atoms;
 * sites outside the model's centre species get 0) and, with do_derivatives, d_V_der (3 x the
 * system's list pairs, list order): dV_i/dr_j for each pair, the self slot holding dV_i/dr_i,
 * zero outside the model cutoff and for clipped sites. The descriptor derivatives are never
 * materialised (the adjoint writes each pair's vector). Overwrites the outputs. */
int tgap_local_property(tgap_context *ctx, tgap_system *system, tgap_model *model, double V0,
                        int precision, int do_derivatives, double *d_V, double *d_V_der);

/* Resident pair and triplet terms (the 2b / core_pot / 3b routines above, as calculate_gap_2b,
 * calculate_gap_core_pot and calculate_gap_3b apply them, gap.f90:246-754): a set of terms held on
 * the device, evaluated on a system's resident neighbor list (its cutoff must reach every term's)
 * and ADDED to energies, forces and per-structure virial. With tgap_md_set_terms the MD step adds
 * them after its SOAP models (full production GAPs: soap_turbo + 2b + 3b + core_pot). Species are
 * channel indices. Qs of a 3b term is n_sparse x 3 column-major; kernel_type 0 "exp", 1 "pol". */
typedef struct tgap_terms tgap_terms;
int tgap_terms_create(tgap_context *ctx, tgap_terms **terms);
int tgap_terms_destroy(tgap_terms *terms);
int tgap_terms_add_2b(tgap_terms *terms, int species1, int species2, int n_sparse, const double *alphas,
                      const double *cutoff, const double *Qs, double rcut, double buffer, double delta,
                      double sigma, double e0);
int tgap_terms_add_core_pot(tgap_terms *terms, int species1, int species2, int n, const double *x,
                            const double *V, double yp1, double ypn, const double *dVdx2);
int tgap_terms_add_3b(tgap_terms *terms, int species_center, int species1, int species2, int n_sparse,
                      const double *alphas, const double *cutoff, const double *Qs, double rcut,
                      double buffer, double delta, const double *sigma, double e0, int kernel_type);
int tgap_terms_compute(tgap_context *ctx, tgap_system *system, tgap_terms *terms, int do_forces,
                       double *d_energies, double *d_forces, double *d_virial);

/* Autotuner (no counterpart in the reference, which has no GPU launch shapes to choose). Runs
 * tgap_compute on this system and these models once to collect the tunable launches (sites per
 * CTA of the descriptor forward and adjoint kernels; sparse-tile chunks per CTA of the fused GAP
 * kernel), then times every candidate of each, one at a time, over `reps` evaluations with CUDA
 * events, and keeps the fastest in the context. Later launches with the same shape key (kernel,
 * precision, l_max, radial block, rows rounded up to a power of two; GAP: padded dimension,
 * row and sparse tile counts) use it; MD and MC objects capture their graphs with the tuned
 * shapes, so tune before creating them. The caller's stage timers are left as they were. */
int tgap_autotune(tgap_context *ctx, tgap_system *system, int n_models, tgap_model *const *models,
                  int precision, int reps);
/* The last tuning as text, one line per key: key, chosen value, its time, the default and its
 * time. `needed` gets the size with the terminating NUL; TGAP_ERR_CAPACITY when cap is short. */
int tgap_autotune_report(tgap_context *ctx, char *buf, int64_t cap, int64_t *needed);
/* Forgets every tuned choice (launches go back to the built-in heuristics). */
int tgap_autotune_clear(tgap_context *ctx);
/* Fixes one launch choice: `key` as tgap_autotune_report prints it, or '*' followed by a suffix
 * for every key that ends with that suffix. The suffix "/persist" selects the form of the
 * descriptor kernels: 1 the persistent work-queue form (the default of the mixed path where the
 * evaluation supplies site counters), 0 one site per warp (the FP64 default). An exact key wins
 * over a suffix. */
int tgap_autotune_set(tgap_context *ctx, const char *key, int value);

/* calculate_gap_soap (src/gap/calculate_gap_soap.f90:171-481) with HOST buffers: copies
 * `positions` (3 x n_atoms, NULL = keep the resident ones) to the device, rebuilds the
 * neighbor list when rebuild != 0 (else refreshes geometry), evaluates all models and copies
 * energies (n_atoms, with the system's e0 as in tgap_compute), forces (3 x n_atoms) and virial
 * (9 per structure) back. */
int tgap_calculate_gap_soap(tgap_context *ctx, tgap_system *system, int n_models,
                            tgap_model *const *models, int precision, const double *positions,
                            int rebuild, double *energies, double *forces, double *virial);

/* Normalised descriptors of every atom seen by the model (rows in site order), device
 * pointer out (n_sites x n_soap). */
int tgap_descriptors(tgap_context *ctx, tgap_system *system, const tgap_model *model,
                     int precision, double *d_soap, int *n_rows);

/* ------------------------------------------------------------------ MD driver */

typedef struct tgap_md tgap_md;

/* NVE velocity Verlet (md_utils.f90:486-532) on one resident structure. masses: amu.
 * The neighbor list uses rcut_max + skin and is rebuilt every `rebuild_every` steps;
 * geometry is refreshed every step. use_graph != 0 captures one step in a CUDA graph. */
int tgap_md_create(tgap_context *ctx, tgap_system *system, int n_models,
                   tgap_model *const *models, const double *masses_amu, double dt,
                   int rebuild_every, int precision, int use_graph, tgap_md **md);
int tgap_md_destroy(tgap_md *md);
/* Adds the terms (tgap_terms_*) to every MD force evaluation after the SOAP models; NULL removes
 * them. The terms object must outlive its use by the MD object. */
int tgap_md_set_terms(tgap_md *md, struct tgap_terms *terms);
int tgap_md_set_velocities(tgap_md *md, const double *velocities);
int tgap_md_run(tgap_md *md, int n_steps);
/* Host copies of the current state; any pointer may be NULL. energies: potential and
 * kinetic energy (eV) of the last step. */
int tgap_md_get_state(tgap_md *md, double *positions, double *velocities, double *forces,
                      double *e_pot, double *e_kin);

/* ------------------------------------------------------------------ Monte Carlo driver */

typedef struct tgap_mc tgap_mc;

/* Metropolis single-atom moves (mc_utils.f90:172-180, 215-277; mc_interface.f90:183-447) on a
 * resident system whose neighbor lists use (largest model cutoff + skin): the system's rcut_max
 * must exceed the models' cutoff, the difference is the skin. Each proposal re-evaluates only
 * the sites within the cutoff of the moved atom's old or new position (local update); the
 * lists are rebuilt when accumulated displacements could exceed the skin. */
int tgap_mc_create(tgap_context *ctx, tgap_system *system, int n_models, tgap_model *const *models,
                   double temperature, int precision, int use_graph, tgap_mc **mc);
int tgap_mc_destroy(tgap_mc *mc);
/* n proposals from the caller's generator: atom (0-based), displacement (3 per proposal, Å),
 * uniform deviate in [0, 1). A move is accepted when min(1, exp(-dE / (kB T))) > u with the
 * reference's kB. dE and the decision of every proposal go to de_log / acc_log when non-NULL. */
int tgap_mc_run(tgap_mc *mc, int64_t n, const int *atoms, const double *displacements,
                const double *uniforms, int64_t *n_accepted, double *de_log, unsigned char *acc_log);
/* Host copies (any pointer may be NULL): positions (3 x n_atoms), site energies summed over
 * models (n_atoms), their total, moves accepted since creation, neighbor-list rebuilds. */
int tgap_mc_get_state(tgap_mc *mc, double *positions, double *energies, double *e_total,
                      int64_t *accepted, int64_t *rebuilds);
/* Learned screen for delayed acceptance (Christen and Fox): per-atom surrogate energy
 * e(q) = w3 . silu(W2 silu(W1 P (q - mean) + b1) + b2) + b3 on the normalised descriptor
 * (row-major P: n_pca x dim, W1: n_hidden x n_pca, W2: n_hidden x n_hidden; weights kept in bf16,
 * FP32 accumulation). Each proposal is first tested with min(1, exp(-dE_s / kB T)) > u1; only
 * survivors get the exact GAP energies and min(1, exp(-(dE - dE_s) / kB T)) > u2. With a screen
 * set, tgap_mc_run takes two deviates per proposal (u1, u2 interleaved). Mixed precision, one
 * model over all sites. With a speculative batch (tgap_mc_set_batch, default 12 slots) the screen
 * judges every slot of a batch from the state before it, the exact GAP kernel skips the 128-row
 * tiles of slots it rejects, and the slots are settled in order with the same decisions as one at a
 * time. */
int tgap_mc_set_screen(tgap_mc *mc, int dim, int n_pca, int n_hidden, const float *mean,
                       const float *pca, const float *w1, const float *b1, const float *w2,
                       const float *b2, const float *w3, float b3);
/* Screen dE and the deciding stage (1: screen, 2: exact) of the last run's first n proposals. */
int tgap_mc_screen_log(tgap_mc *mc, int64_t n, double *de_screen, unsigned char *stage);
/* Fallback to plain GAP MC (no counterpart in the reference, whose MC has no screen). Over each
 * window of `window` screen-judged proposals, pass = fraction passed to the exact stage and
 * confirm = fraction of those the exact stage accepts; when pass < min_pass, or confirm <
 * min_confirm with at least 32 passed, or pass > max_pass (the screen settles too few proposals to
 * pay for its own evaluation: delayed acceptance saves only the exact energies of the proposals it
 * rejects), the screen is switched off for the rest of the MC object's life (or until
 * tgap_mc_set_screen installs one again). Proposals still take deviate pairs; plain moves use the
 * first. Defaults: 256, 0.1, 0.002, 0.99 (at a pass rate of 0.998, 256 proposals show at most two
 * rejections with high probability, so a screen that cannot pay for itself is off within a few
 * hundred proposals; a useful screen passes far fewer than 99 %). */
int tgap_mc_screen_fallback(tgap_mc *mc, int64_t window, double min_confirm, double min_pass, double max_pass);
/* Speculative batch of plain GAP MC (no counterpart in the reference, which judges proposals one
 * at a time): `slots` consecutive proposals (1..16; default 12 mixed, 4 FP64) are evaluated side by side from
 * the same state and then settled in order on the device. A proposal's energy change depends
 * only on atoms within twice the model cutoff of its atom, so it stays valid unless an accepted
 * earlier proposal of the batch moved an atom within 2 rc + |d_i| + |d_k| of it (minimum image;
 * in a cell replicated into a supercell, any two proposals of the structure); the batch stops
 * at the first one that is not valid, and that proposal opens the next batch. Decisions and
 * final positions are those of one-at-a-time evaluation. With a screen active the batch applies
 * delayed acceptance (tgap_mc_set_screen); one slot keeps the one-at-a-time screened step. */
int tgap_mc_set_batch(tgap_mc *mc, int slots);
/* Batches run since creation and the proposals they settled. */
int tgap_mc_batch_stats(tgap_mc *mc, int64_t *batches, int64_t *settled);
/* Screen counters since creation (any pointer may be NULL): whether the screen is in use,
 * proposals it judged, passed to the exact stage, confirmed there, and fallbacks taken. */
int tgap_mc_screen_stats(tgap_mc *mc, int *active, int64_t *judged, int64_t *passed,
                         int64_t *confirmed, int64_t *fallbacks);

/* ---- Screen network training and evaluation (no counterpart in the reference). The network
 * part of the screen, on standardised PCA coordinates z (row-major n x n_pca):
 *   out = w3 . silu(W2 silu(W1 z + b1) + b2) + b3   (W1: n_hidden x n_pca, W2: n_hidden x n_hidden)
 * and the loss (1/n) sum (out - t)^2 against targets t. FP32 throughout; n_pca <= 256,
 * n_hidden <= 512, with the pair limited to one CTA's shared memory (64 x 128 fits). */

/* Loss and its gradients over all n rows (n <= 16384), as one batch. Host arrays. */
int tgap_screen_grad(tgap_context *ctx, int64_t n, int n_pca, int n_hidden, const float *z,
                     const float *t, const float *w1, const float *b1, const float *w2,
                     const float *b2, const float *w3, float b3, float *g_w1, float *g_b1,
                     float *g_w2, float *g_b2, float *g_w3, float *g_b3, double *loss);
/* Adam (beta 0.9 / 0.999, eps 1e-8, bias-corrected) on minibatches of `batch` rows, epoch e
 * visiting rows order[e * n .. e * n + n) in that order (the last batch of an epoch may be
 * short), learning rate lr * (1 + cos(pi e / epochs)) / 2. The weights are read as the initial
 * point and overwritten with the result; loss_log (optional, `epochs` entries) gets each
 * epoch's mean squared error over its minibatches (weights before each update). */
int tgap_screen_train(tgap_context *ctx, int64_t n, int n_pca, int n_hidden, const float *z,
                      const float *t, int epochs, int batch, float lr, const int *order, float *w1,
                      float *b1, float *w2, float *b2, float *w3, float *b3, double *loss_log);
/* Screen energies e (n) of descriptor rows q (row-major n x dim, FP32) with the full screen
 * (PCA and network, weights as tgap_mc_set_screen takes them, rounded to bf16 the same way);
 * the kernel the Monte Carlo driver runs. */
int tgap_screen_eval(tgap_context *ctx, int64_t n, int dim, int n_pca, int n_hidden,
                     const float *mean, const float *pca, const float *w1, const float *b1,
                     const float *w2, const float *b2, const float *w3, float b3, const float *q,
                     double *e);

#ifdef __cplusplus
}
#endif
#endif
