// Pair and triplet GAP terms resident on the device (pair_terms.cu): the distance_2b GAP
// (gap.f90:329-460), the core potential (gap.f90:552-686) and the angle_3b GAP (gap.f90:756-1015),
// evaluated on a resident neighbor list and added into energies, forces and virial.
#pragma once

#include <vector>

#include "tgap_internal.h"

namespace tgap {

struct Term2b {
    int sp1 = 0, sp2 = 0, n_sparse = 0;
    DevBuf alphas, cutoff, Qs;
    double rcut = 0, buffer = 0.5, delta = 1, sigma = 1, e0 = 0;
};

struct TermCore {
    int sp1 = 0, sp2 = 0, n = 0;
    DevBuf x, V, y2;
    double yp1 = 0, ypn = 0, rcut = 0;  // rcut = max(x)
};

struct Term3b {
    int sp0 = 0, sp1 = 0, sp2 = 0, n_sparse = 0, kernel = 0;  // kernel 0 "exp", 1 "pol"
    DevBuf pref, Qs;  // pref = 2 delta^2 alphas cutoff (gap.f90:829); Qs [3][n_sparse]
    double rcut = 0, buffer = 0.5, is[3] = {1, 1, 1}, e0 = 0;  // is = 1 / sigma^2
};

struct TermSet {
    std::vector<Term2b> t2b;
    std::vector<TermCore> core;
    std::vector<Term3b> t3b;
    double rcut_max() const
    {
        double r = 0;
        for (const auto &b : t2b) r = b.rcut > r ? b.rcut : r;
        for (const auto &c : core) r = c.rcut > r ? c.rcut : r;
        for (const auto &b : t3b) r = b.rcut > r ? b.rcut : r;
        return r;
    }
    void release()
    {
        for (auto &b : t2b)
            for (DevBuf *p : {&b.alphas, &b.cutoff, &b.Qs}) p->release();
        for (auto &c : core)
            for (DevBuf *p : {&c.x, &c.V, &c.y2}) p->release();
        for (auto &b : t3b)
            for (DevBuf *p : {&b.pref, &b.Qs}) p->release();
    }
};

// Adds every term of t on a resident list (site species and structure per site, neighbor species
// and folded atom per pair) into the outputs; the virial of structure s is d_virial[9 s .. 9 s + 9).
int terms_compute(tgap_context *ctx, const TermSet &t, int n_sites, const int64_t *d_start, const double *d_rjs,
                  const double *d_xyz, const int *d_site_species, const int *d_nsp, const int *d_jatom,
                  const int *d_site_struct, int do_forces, double *d_energies, double *d_forces, double *d_virial);

}  // namespace tgap
