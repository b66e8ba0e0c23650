// Neighbor-list data of a batch of periodic structures resident on the device.
#pragma once

#include <cstring>
#include <vector>

#include "tgap_internal.h"

namespace tgap {

// One periodic structure of a batch. Lattice vectors are those of the (replicated) supercell.
struct StructDesc {
    double a[3], b[3], c[3];
    double inv[9];      // inverse Gram matrix, row-major (triclinic minimum image)
    double rcut;        // list cutoff (model cutoff + skin)
    int ortho;
    int atom_off;       // first global site
    int n;              // sites
    int sc_off;         // first supercell position
    int n_sc;           // supercell atoms (n * replicas)
    int rep[3];         // replicas along a, b, c
    int cell_off;       // first cell of the linked-cell grid, -1 = brute-force path
    int mx, my, mz;
    double pa[3], pb[3], pc[3];  // primitive lattice vectors (before replication)
};

struct NeighborBatch {
    int n_structures = 0;
    int n_atoms = 0;        // central sites over all structures
    int n_sc_total = 0;
    int n_cells = 0;
    int64_t n_pairs = 0;
    // n_pairs is not yet read back: the lists were last rebuilt on the device alone
    // (neighbors_rebuild_lists_device; neighbors_sync_count reads it)
    bool count_on_device = false;
    bool replicated = true;  // every supercell is a pure replica of its primitive cell
    std::vector<StructDesc> host_structs;
    DevBuf d_structs;
    DevBuf positions;       // double [3 n_atoms] (primitive cells; MD state)
    DevBuf pos_sc;          // double [3 n_sc_total]
    DevBuf species_sc;      // int [n_sc_total]
    DevBuf site_struct;     // int [n_atoms]
    DevBuf atom_cell, cell_count, cell_start, cell_cursor, cell_atoms, cell_tmp;
    DevBuf counts;          // int64 [n_atoms + 1]
    DevBuf start;           // int64 [n_atoms + 1]
    DevBuf n_neigh;         // int [n_atoms]
    DevBuf list;            // int [P], 1-based supercell index within the structure
    DevBuf rjs, xyz, thetas, phis;
    DevBuf nspecies;        // int [P] species channel of the neighbor
    DevBuf jatom;           // int [P] folded global atom of the neighbor
    DevBuf scan_tmp;
    DevBuf stage, staged;   // int [n_atoms][96] list rows staged by the count pass, int [n_atoms] flags
    int ensure_pairs(int64_t P);
    int64_t pair_capacity() const { return (int64_t)(list.bytes / sizeof(int)); }
    void release_all()
    {
        DevBuf *bufs[] = {&d_structs, &positions, &pos_sc, &species_sc, &site_struct, &atom_cell,
                          &cell_count, &cell_start, &cell_cursor, &cell_atoms, &cell_tmp, &counts, &start,
                          &n_neigh, &list, &rjs, &xyz, &thetas, &phis, &nspecies, &jatom,
                          &scan_tmp, &stage, &staged};
        for (DevBuf *b : bufs) b->release();
    }
};

int make_struct_desc(const double a[3], const double b[3], const double c[3], int box_small,
                     double rcut, StructDesc *S);
// Host arrays in: offsets[n_structures + 1], positions 3 x n_atoms, boxes 9 per structure,
// species per atom. force_small (optional, per structure) selects the brute-force path.
int neighbors_setup(tgap_context *ctx, NeighborBatch *nb, int n_structures, const int *offsets,
                    const double *positions, const double *boxes, const int *species,
                    double rcut, const int *force_small);
// Supercell layout given directly (reference build_neighbors_list surface, one structure).
int neighbors_setup_supercell(tgap_context *ctx, NeighborBatch *nb, int n_sites, int n_sc,
                              const double *positions_sc, const double a[3], const double b[3],
                              const double c[3], int box_small, double rcut,
                              const int *species_sc);
// Rebuild the pair lists (one host synchronization for the pair count), then the geometry.
int neighbors_build(tgap_context *ctx, NeighborBatch *nb, int rebuild, int64_t capacity,
                    int64_t *n_pairs_out, bool with_angles);
int neighbors_rebuild_lists(tgap_context *ctx, NeighborBatch *nb, int64_t capacity, int64_t *n_pairs_out);
// The same lists rebuilt without a host synchronization (capturable in a graph), inside the pair
// arrays already reserved (pair_capacity(), a quarter above the count they were sized for): the
// offsets are clamped below that capacity, and with report a longer list is recorded in the device
// check word (kCheckPairCapacity, reported as TGAP_ERR_CAPACITY at the next check); without it the
// caller compares the count itself: the unclamped total is left in counts[n_atoms]. n_pairs (the
// pairs the lists hold) is then read back lazily by neighbors_sync_count.
int neighbors_rebuild_lists_device(tgap_context *ctx, NeighborBatch *nb, bool report);
int neighbors_sync_count(tgap_context *ctx, NeighborBatch *nb);
// from_positions: form supercell positions from the primitive ones inside the kernel
int neighbors_geometry(tgap_context *ctx, NeighborBatch *nb, bool with_angles, bool from_positions);
// Geometry of the current lists at the current (primitive) positions.
int neighbors_refresh(tgap_context *ctx, NeighborBatch *nb);
// Only the per-pair species and atom maps of the current lists (after a rebuild whose geometry the
// descriptor forward writes).
int neighbors_maps(tgap_context *ctx, NeighborBatch *nb);
int neighbors_set_counts(tgap_context *ctx, NeighborBatch *nb);
int neighbors_sync_positions(tgap_context *ctx, NeighborBatch *nb);

}  // namespace tgap
