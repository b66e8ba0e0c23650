// Metropolis Monte Carlo with local updates (mc.cu): device state and launchers.
//
// One proposal = move atom a by d. The sites whose descriptor can change are a and every atom
// within the largest model cutoff of a's old or new position; only those are re-evaluated
// (trial pair geometry -> descriptor forward -> GAP energy rows), the energy change is the sum
// of (new - cached) site energies, and the move is accepted when
// min(1, exp(-dE / (kB T))) > u (mc_utils.f90:172-180, :255; mc_interface.f90:245-300), with
// the reference's kB literal taken in default-real precision.
#pragma once

#include "neighbors.h"

namespace tgap {

constexpr int kMcMaxModels = 4;
constexpr int kMcMaxBatch = 16;  // proposals evaluated side by side by the speculative batch

// Device-resident driver state (one per MC object).
struct McDev {
    long long next;      // proposals of the current run consumed so far
    long long n_prop;    // proposals of the current run
    long long accepted;  // accepted moves since creation
    long long serial;    // proposals selected since creation (stamps of the dedupe marks)
    int status;          // kMcRunning / kMcNeedRebuild / kMcDone
    int atom;            // atom moved by the proposal in flight
    double pos_new[3];   // its trial position
    double dnorm;        // |d|
    double maxD;         // largest accumulated displacement since the last list build
    double de_screen;    // screen energy change of the proposal in flight
    int skip;            // 1: the proposal was settled by the screen (exact stage skipped)
    int count[kMcMaxModels];  // affected sites per model for the proposal in flight
    long long s_prop;    // proposals judged by the screen since creation (stage 1)
    long long s_pass;    // of those, passed on to the exact stage
    long long s_conf;    // of those, accepted by the exact stage
    // speculative batch (plain GAP MC): slot b holds proposal slot_prop[b], evaluated from the state
    // before the batch: first the deferred proposals pend[0, n_pend) (in order, all below next), then
    // next, next + 1, ... With n_pend = 0 the unsettled proposals are next, next + 1, ...
    int n_pend;
    long long pend[kMcMaxBatch];
    long long slot_prop[kMcMaxBatch];
    int slot_flag[kMcMaxBatch];  // 0 evaluated, 1 no proposal left, 2 needs a list rebuild
    int slot_atom[kMcMaxBatch];
    double slot_old[kMcMaxBatch][3], slot_new[kMcMaxBatch][3], slot_dn[kMcMaxBatch];
    int slot_count[kMcMaxBatch][kMcMaxModels];
    long long batches, batch_resolved;  // batches run and proposals they settled
    // delayed acceptance inside the batch: each slot's screen energy change and stage-1 verdict
    double slot_des[kMcMaxBatch];
    int slot_pass[kMcMaxBatch];
};

// Per-proposal logs (device arrays of the run's length, any may be null).
struct McLogs {
    double *de;            // exact dE (NaN when the screen rejected the move)
    unsigned char *acc;    // 1 accepted
    double *de_screen;     // screen dE (delayed acceptance only)
    unsigned char *stage;  // 1: settled by the screen, 2: by the exact energies
};

enum McStatus { kMcRunning = 0, kMcNeedRebuild = 1, kMcDone = 2 };

struct McModelSel {
    int n_models;
    int central_species[kMcMaxModels];  // 0: every site
};

// Selects the affected sites of proposal st->next into sites[m * cap + r] (list order,
// duplicates removed). Sets st->status = kMcNeedRebuild when the move could carry a pair of the
// skin-padded list inside the cutoff unseen (max accumulated displacement + this atom's + |d|
// >= skin), kMcDone when the run's proposals are exhausted.
int mc_select(tgap_context *ctx, McDev *d_st, const NeighborBatch &nb, const McModelSel &sel, double rc_sel,
              double skin, const int *d_prop_atom, const double *d_prop_disp, const double *d_dacc,
              long long *d_mark, int *d_sites, int cap);

// Pair geometry of the affected sites with the moved atom at its trial position, written as a
// fixed-stride list: row r of model m holds its site's list pairs at [r * pmax, (r+1) * pmax),
// unused slots and rows blind (species 0).
int mc_trial_geometry(tgap_context *ctx, const McDev *d_st, const NeighborBatch &nb, int n_models,
                      const int *d_sites, int cap, int pmax, double *d_txyz, double *d_trjs, int *d_tnsp);

// Delayed acceptance, stage 1 (Christen and Fox): the screen's energy change dE_s of the
// affected sites (model 0's rows) against u1 = prop_u[2k]; a rejection settles the proposal
// (st->skip = 1, logged, st->next advanced) and the exact stage does nothing.
int mc_screen_stage(tgap_context *ctx, McDev *d_st, const int *d_sites, const float *d_es_trial,
                    const float *d_es_cache, const double *d_prop_u, double temperature, McLogs logs);

// Energy change, acceptance and commit (positions, cached site energies, displacement
// bookkeeping); logs dE and the decision of proposal st->next and advances it. With a screen
// (screened != 0) the test is min(1, exp(-(dE - dE_s) / kB T)) > u2 = prop_u[2k + 1] and the
// screen cache of the affected sites is committed too; otherwise min(1, exp(-dE / kB T)) >
// prop_u[u_stride k] (u_stride 2 when the proposals carry deviate pairs for a screen that is
// installed but switched off).
int mc_accept(tgap_context *ctx, McDev *d_st, int n_models, const int *d_sites, int cap, const double *d_etrial,
              double *d_ecache, int n_atoms, double *d_positions, double *d_dacc, const double *d_prop_u,
              double temperature, McLogs logs, int screened, int u_stride, const float *d_es_trial,
              float *d_es_cache);

// Speculative batch of B consecutive proposals (plain GAP MC, same decisions as one at a time).
// Proposal k's energy change depends only on atoms within 2 rc of its atom's old or new
// position, so the proposals next .. next + B - 1 are evaluated side by side from the state
// before the batch, then settled in order: each is valid unless an accepted earlier one of the
// batch moved an atom within 2 rc + |d_i| + |d_k| of it (minimum image, same structure), and the
// batch stops at the first invalid one (it is proposed again in the next batch), at the first
// that needs a list rebuild, or when the run's proposals are exhausted. Layout: sites
// [(m B + b) cap + r], trial rows of model m contiguous over (b, r), etrial [m][B cap].
int mc_select_batch(tgap_context *ctx, McDev *d_st, const NeighborBatch &nb, const McModelSel &sel, double rc_sel,
                    double skin, const int *d_prop_atom, const double *d_prop_disp, const double *d_dacc,
                    long long *d_mark, int *d_sites, int cap, int B);
int mc_trial_geometry_batch(tgap_context *ctx, const McDev *d_st, const NeighborBatch &nb, int n_models,
                            const int *d_sites, int cap, int pmax, int B, double *d_txyz, double *d_trjs, int *d_tnsp);
// With a screen (screened != 0, one model, two deviates per proposal): stage 1 of every slot is
// decided before the exact energies (mc_screen_batch) and the settlement applies delayed
// acceptance in order, a slot rejected by the screen settling without its exact energies; the
// screen cache of an accepted slot's sites is committed with its exact energies.
int mc_resolve_batch(tgap_context *ctx, McDev *d_st, const NeighborBatch &nb, int n_models, const int *d_sites,
                     int cap, int B, const double *d_etrial, double *d_ecache, double *d_positions, double *d_dacc,
                     const double *d_prop_u, int u_stride, double temperature, double rc_sel, double skin,
                     McLogs logs, int screened = 0, const float *d_es_trial = nullptr, float *d_es_cache = nullptr);

// Delayed acceptance, stage 1, for every slot of a speculative batch (one model): the screen's
// energy change over the slot's rows (screen energies es_trial [B cap], cache es_cache [atoms])
// against u1 of the proposal the slot holds. tile_skip[t] (n_tiles row tiles of 128 trial rows)
// is set when no slot with rows in tile t passes, so the exact GAP kernel skips that tile; rows
// of a skipped tile keep stale energies that the settlement never reads.
int mc_screen_batch(tgap_context *ctx, McDev *d_st, const int *d_sites, int cap, int B, const float *d_es_trial,
                    const float *d_es_cache, const double *d_prop_u, double temperature, int *d_tile_skip,
                    int n_tiles);

// Start of a run of n proposals (keeps a pending rebuild request), and the reset after a list
// rebuild.
int mc_begin(tgap_context *ctx, McDev *d_st, long long n_prop);
int mc_lists_rebuilt(tgap_context *ctx, McDev *d_st, double *d_dacc, int n_atoms);

}  // namespace tgap
