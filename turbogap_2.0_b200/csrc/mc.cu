// Metropolis Monte Carlo with local updates: proposal selection, trial geometry and acceptance
// (mc_utils.f90:172-180, 215-277; mc_interface.f90:183-447). Built with --fmad=false like the
// neighbor build, so the trial pair vectors carry the same bits as a full rebuild at the trial
// positions would.
#include "mc_kernels.h"
#include "neighbors_device.cuh"

namespace tgap {

// Position of supercell atom j (1-based within structure S) with primitive atom `moved` (global
// index) at pos_new, by the replication arithmetic of sc_position.
__device__ __forceinline__ void sc_position_moved(const StructDesc &S, const double *pos, int j, int moved,
                                                  const double *pos_new, double out[3])
{
    const int a = (j - 1) % S.n, r = (j - 1) / S.n;
    const int k2 = r % S.rep[2], j2 = (r / S.rep[2]) % S.rep[1], i2 = r / (S.rep[2] * S.rep[1]);
    const double *p = (S.atom_off + a == moved) ? pos_new : pos + 3 * (size_t)(S.atom_off + a);
    for (int q = 0; q < 3; ++q) {
        double v = p[q] + (double)i2 * S.pa[q];
        v = v + (double)j2 * S.pb[q];
        v = v + (double)k2 * S.pc[q];
        out[q] = v;
    }
}

__device__ __forceinline__ unsigned mc_lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// One warp. mark[atom] holds the serial of the last proposal that selected it.
__global__ void k_mc_select(McDev *st, const int64_t *__restrict__ start, const int *__restrict__ list,
                            const int *__restrict__ jatom, const int *__restrict__ site_struct,
                            const StructDesc *__restrict__ sd, const double *__restrict__ pos,
                            const int *__restrict__ species_sc, McModelSel sel, double rc_sel, double skin,
                            const int *__restrict__ prop_atom, const double *__restrict__ prop_disp,
                            const double *__restrict__ dacc, long long *mark, int *sites, int cap, int *check)
{
    const int lane = threadIdx.x & 31;
    __shared__ int s_status;
    __shared__ long long s_serial;
    if (lane == 0) {
        int status = st->status;
        if (status == kMcRunning) {
            const long long k = st->next;
            if (k >= st->n_prop) {
                status = kMcDone;
            } else {
                const int a = prop_atom[k];
                const double d0 = prop_disp[3 * k], d1 = prop_disp[3 * k + 1], d2 = prop_disp[3 * k + 2];
                const double dn = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
                // list of cutoff rc + skin stays complete while every pair moved by < skin
                if (st->maxD + dacc[a] + dn >= skin) {
                    status = kMcNeedRebuild;
                } else {
                    st->atom = a;
                    st->pos_new[0] = pos[3 * (size_t)a] + d0;
                    st->pos_new[1] = pos[3 * (size_t)a + 1] + d1;
                    st->pos_new[2] = pos[3 * (size_t)a + 2] + d2;
                    st->dnorm = dn;
                }
            }
            st->status = status;
        }
        if (status != kMcRunning)
            for (int m = 0; m < kMcMaxModels; ++m) st->count[m] = 0;
        st->skip = 0;
        s_status = status;
        // serial of this proposal, unique over the object's lifetime (stamps mark[])
        if (status == kMcRunning) s_serial = ++st->serial;
    }
    __syncwarp();
    if (s_status != kMcRunning) return;
    const long long serial = s_serial;
    const int a = st->atom;
    const double pn[3] = {st->pos_new[0], st->pos_new[1], st->pos_new[2]};
    const StructDesc &S = sd[site_struct[a]];
    const int ia = a - S.atom_off + 1;
    double pa_old[3], pa_new[3];
    sc_position(S, pos, ia, pa_old);
    sc_position_moved(S, pos, ia, a, pn, pa_new);
    int cnt[kMcMaxModels] = {0, 0, 0, 0};
    auto species_of = [&](int g) { return species_sc[S.sc_off + (g - S.atom_off)]; };
    // the moved atom first
    if (lane == 0) mark[a] = serial;
    {
        const int sa = species_of(a);
        for (int m = 0; m < sel.n_models; ++m)
            if (sel.central_species[m] == 0 || sel.central_species[m] == sa) {
                if (lane == 0) sites[m * cap] = a;
                cnt[m] = 1;
            }
    }
    __syncwarp();
    const int64_t kb = start[a], ke = start[a + 1];
    for (int64_t k0 = kb + 1; k0 < ke; k0 += 32) {
        const int64_t k = k0 + lane;
        bool pick = false;
        int g = -1;
        if (k < ke) {
            const int jsc = list[k];
            g = jatom[k];
            double pj_old[3], pj_new[3], dist[3], dd;
            sc_position(S, pos, jsc, pj_old);
            sc_position_moved(S, pos, jsc, a, pn, pj_new);
            get_distance_dev(pa_old, pj_old, S, dist, &dd);
            pick = dd < rc_sel;
            get_distance_dev(pa_new, pj_new, S, dist, &dd);
            pick = pick || dd < rc_sel;
        }
        // one entry per atom: the lowest lane among equal atoms, and only if no earlier chunk
        // (or the moved atom itself) took it
        const unsigned peers = __match_any_sync(0xffffffffu, pick ? g : -2 - lane);
        const bool leader = pick && (__ffs(peers) - 1 == lane);
        const bool fresh = leader && mark[g] != serial;
        __syncwarp();
        if (fresh) mark[g] = serial;
        const int sg = fresh ? species_of(g) : 0;
        for (int m = 0; m < sel.n_models; ++m) {
            const bool in_m = fresh && (sel.central_species[m] == 0 || sel.central_species[m] == sg);
            const unsigned mm = __ballot_sync(0xffffffffu, in_m);
            if (in_m) {
                const int slot = cnt[m] + __popc(mm & mc_lanemask_lt());
                if (slot < cap)
                    sites[m * cap + slot] = g;
                else
                    check_fail(check, kCheckMcOverflow, slot, g);
            }
            cnt[m] += __popc(mm);
        }
        __syncwarp();
    }
    if (lane == 0)
        for (int m = 0; m < kMcMaxModels; ++m) st->count[m] = m < sel.n_models ? min(cnt[m], cap) : 0;
}

// Warp per (model, row).
__global__ void k_mc_trial_geometry(const McDev *st, int n_models, const int *__restrict__ sites, int cap, int pmax,
                                    const int64_t *__restrict__ start, const int *__restrict__ list,
                                    const int *__restrict__ nspecies, const int *__restrict__ site_struct,
                                    const StructDesc *__restrict__ sd, const double *__restrict__ pos,
                                    double *__restrict__ txyz, double *__restrict__ trjs, int *__restrict__ tnsp,
                                    int *check)
{
    const int lane = threadIdx.x & 31;
    const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (w >= n_models * cap) return;
    const int m = w / cap, r = w - m * cap;
    const size_t base = (size_t)w * pmax;
    int ns = 0, g = 0;
    if (st->status == kMcRunning && r < st->count[m]) {
        g = sites[m * cap + r];
        ns = (int)(start[g + 1] - start[g]);
        if (ns > pmax) {
            if (lane == 0) check_fail(check, kCheckMcOverflow, g, ns);
            ns = pmax;
        }
    }
    const int a = st->atom;
    const double pn[3] = {st->pos_new[0], st->pos_new[1], st->pos_new[2]};
    for (int t = lane; t < pmax; t += 32) {
        double x0 = 0.0, x1 = 0.0, x2 = 0.0, rr = 0.0;
        int sp = 0;
        if (t < ns) {
            const int64_t k = start[g] + t;
            sp = nspecies[k];
            if (t > 0) {
                const StructDesc &S = sd[site_struct[g]];
                double pi[3], pj[3], dist[3];
                sc_position_moved(S, pos, g - S.atom_off + 1, a, pn, pi);
                sc_position_moved(S, pos, list[k], a, pn, pj);
                get_distance_dev(pi, pj, S, dist, &rr);
                x0 = dist[0];
                x1 = dist[1];
                x2 = dist[2];
            }
        }
        txyz[3 * (base + t)] = x0;
        txyz[3 * (base + t) + 1] = x1;
        txyz[3 * (base + t) + 2] = x2;
        trjs[base + t] = rr;
        tnsp[base + t] = sp;
    }
}

// kB of mc_utils.f90:176, a default-real literal
__device__ __forceinline__ double mc_kb() { return (double)8.617333262e-5f; }

// One warp: screen dE of the affected sites (model 0) in a fixed reduction order, stage-1 test.
__global__ void k_mc_screen_stage(McDev *st, const int *__restrict__ sites, const float *__restrict__ es_trial,
                                  const float *__restrict__ es_cache, const double *__restrict__ prop_u,
                                  double temperature, McLogs logs)
{
    const int lane = threadIdx.x & 31;
    if (st->status != kMcRunning) return;
    const long long k = st->next;
    const int c = st->count[0];
    double des = 0.0;
    for (int r = lane; r < c; r += 32) des += (double)es_trial[r] - (double)es_cache[sites[r]];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) des += __shfl_xor_sync(0xffffffffu, des, o);
    if (lane == 0) {
        double p = exp(-des / (mc_kb() * temperature));
        p = p < 1.0 ? p : 1.0;
        st->de_screen = des;
        st->s_prop += 1;
        if (logs.de_screen) logs.de_screen[k] = des;
        if (!(p > prop_u[2 * k])) {
            st->skip = 1;
            if (logs.de) logs.de[k] = __longlong_as_double(0x7ff8000000000000ll);
            if (logs.acc) logs.acc[k] = 0;
            if (logs.stage) logs.stage[k] = 1;
            st->next = k + 1;
        }
    }
}

// One warp: dE in a fixed reduction order, then the reference's acceptance test.
__global__ void k_mc_accept(McDev *st, int n_models, const int *__restrict__ sites, int cap,
                            const double *__restrict__ etrial, double *__restrict__ ecache, int n_atoms,
                            double *__restrict__ pos, double *__restrict__ dacc, const double *__restrict__ prop_u,
                            double temperature, McLogs logs, int screened, int u_stride,
                            const float *__restrict__ es_trial, float *__restrict__ es_cache)
{
    const int lane = threadIdx.x & 31;
    if (st->status != kMcRunning || st->skip) return;
    const long long k = st->next;
    double de = 0.0;
    for (int m = 0; m < n_models; ++m) {
        const int c = st->count[m];
        for (int r = lane; r < c; r += 32)
            de += etrial[(size_t)m * cap + r] - ecache[(size_t)m * n_atoms + sites[m * cap + r]];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) de += __shfl_xor_sync(0xffffffffu, de, o);
    int accept = 0;
    if (lane == 0) {
        // mc_utils.f90:172-180 (p = exp(-dE / kB T)); get_mc_acceptance (:255) takes min(1, p);
        // mc_interface.f90:286 accepts when p > ranf. Delayed acceptance replaces dE by dE - dE_s
        // and uses the second deviate.
        const double x = screened ? de - st->de_screen : de;
        double p = exp(-x / (mc_kb() * temperature));
        p = p < 1.0 ? p : 1.0;
        accept = p > (screened ? prop_u[2 * k + 1] : prop_u[(long long)u_stride * k]) ? 1 : 0;
        if (screened) {
            st->s_pass += 1;
            st->s_conf += accept;
        }
        if (logs.de) logs.de[k] = de;
        if (logs.acc) logs.acc[k] = (unsigned char)accept;
        if (logs.stage) logs.stage[k] = 2;
    }
    accept = __shfl_sync(0xffffffffu, accept, 0);
    if (accept) {
        for (int m = 0; m < n_models; ++m) {
            const int c = st->count[m];
            for (int r = lane; r < c; r += 32)
                ecache[(size_t)m * n_atoms + sites[m * cap + r]] = etrial[(size_t)m * cap + r];
        }
        if (screened)
            for (int r = lane; r < st->count[0]; r += 32) es_cache[sites[r]] = es_trial[r];
        if (lane == 0) {
            const int a = st->atom;
            pos[3 * (size_t)a] = st->pos_new[0];
            pos[3 * (size_t)a + 1] = st->pos_new[1];
            pos[3 * (size_t)a + 2] = st->pos_new[2];
            dacc[a] += st->dnorm;
            if (dacc[a] > st->maxD) st->maxD = dacc[a];
            st->accepted += 1;
        }
    }
    __syncwarp();
    if (lane == 0) st->next = k + 1;
}

__global__ void k_mc_begin(McDev *st, long long n_prop)
{
    st->next = 0;
    st->n_pend = 0;
    st->n_prop = n_prop;
    if (st->status != kMcNeedRebuild) st->status = kMcRunning;
}

__global__ void k_mc_lists_rebuilt(McDev *st, double *dacc, int n)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < n) dacc[g] = 0.0;
    if (g == 0) {
        st->maxD = 0.0;
        if (st->status == kMcNeedRebuild) st->status = kMcRunning;
    }
}

// ----------------------------------------------------------------------------- speculative batch

// Block b (one warp) selects the affected sites of slot b's proposal (the deferred ones first, then
// next, next + 1, ...) from the state before the batch; mark[b N + atom] holds the stamp of the last
// batch whose slot b took the atom.
__global__ void k_mc_select_batch(McDev *st, const int64_t *__restrict__ start, const int *__restrict__ list,
                                  const int *__restrict__ jatom, const int *__restrict__ site_struct,
                                  const StructDesc *__restrict__ sd, const double *__restrict__ pos,
                                  const int *__restrict__ species_sc, McModelSel sel, double rc_sel, double skin,
                                  const int *__restrict__ prop_atom, const double *__restrict__ prop_disp,
                                  const double *__restrict__ dacc, long long *mark, int n_atoms, int *sites, int cap,
                                  int B, int *check)
{
    const int lane = threadIdx.x & 31, b = blockIdx.x;
    __shared__ int s_flag;
    if (lane == 0) {
        int flag = 1;
        if (st->status == kMcRunning) {
            const long long k = b < st->n_pend ? st->pend[b] : st->next + (b - st->n_pend);
            if (k < st->n_prop) {
                st->slot_prop[b] = k;
                const int a = prop_atom[k];
                const double d0 = prop_disp[3 * k], d1 = prop_disp[3 * k + 1], d2 = prop_disp[3 * k + 2];
                const double dn = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
                if (st->maxD + dacc[a] + dn >= skin) {
                    flag = 2;
                } else {
                    flag = 0;
                    st->slot_atom[b] = a;
                    for (int q = 0; q < 3; ++q) st->slot_old[b][q] = pos[3 * (size_t)a + q];
                    st->slot_new[b][0] = pos[3 * (size_t)a] + d0;
                    st->slot_new[b][1] = pos[3 * (size_t)a + 1] + d1;
                    st->slot_new[b][2] = pos[3 * (size_t)a + 2] + d2;
                    st->slot_dn[b] = dn;
                }
            }
        }
        st->slot_flag[b] = flag;
        if (flag != 0)
            for (int m = 0; m < kMcMaxModels; ++m) st->slot_count[b][m] = 0;
        s_flag = flag;
    }
    __syncwarp();
    if (s_flag != 0) return;
    const long long stamp = st->serial + 1;  // advanced by the resolve kernel after every batch
    long long *mk = mark + (size_t)b * n_atoms;
    const int a = st->slot_atom[b];
    const double pn[3] = {st->slot_new[b][0], st->slot_new[b][1], st->slot_new[b][2]};
    const StructDesc &S = sd[site_struct[a]];
    const int ia = a - S.atom_off + 1;
    double pa_old[3], pa_new[3];
    sc_position(S, pos, ia, pa_old);
    sc_position_moved(S, pos, ia, a, pn, pa_new);
    int cnt[kMcMaxModels] = {0, 0, 0, 0};
    auto species_of = [&](int g) { return species_sc[S.sc_off + (g - S.atom_off)]; };
    if (lane == 0) mk[a] = stamp;
    {
        const int sa = species_of(a);
        for (int m = 0; m < sel.n_models; ++m)
            if (sel.central_species[m] == 0 || sel.central_species[m] == sa) {
                if (lane == 0) sites[(m * B + b) * cap] = a;
                cnt[m] = 1;
            }
    }
    __syncwarp();
    const int64_t kb = start[a], ke = start[a + 1];
    for (int64_t k0 = kb + 1; k0 < ke; k0 += 32) {
        const int64_t k = k0 + lane;
        bool pick = false;
        int g = -1;
        if (k < ke) {
            const int jsc = list[k];
            g = jatom[k];
            double pj_old[3], pj_new[3], dist[3], dd;
            sc_position(S, pos, jsc, pj_old);
            sc_position_moved(S, pos, jsc, a, pn, pj_new);
            get_distance_dev(pa_old, pj_old, S, dist, &dd);
            pick = dd < rc_sel;
            get_distance_dev(pa_new, pj_new, S, dist, &dd);
            pick = pick || dd < rc_sel;
        }
        const unsigned peers = __match_any_sync(0xffffffffu, pick ? g : -2 - lane);
        const bool leader = pick && (__ffs(peers) - 1 == lane);
        const bool fresh = leader && mk[g] != stamp;
        __syncwarp();
        if (fresh) mk[g] = stamp;
        const int sg = fresh ? species_of(g) : 0;
        for (int m = 0; m < sel.n_models; ++m) {
            const bool in_m = fresh && (sel.central_species[m] == 0 || sel.central_species[m] == sg);
            const unsigned mm = __ballot_sync(0xffffffffu, in_m);
            if (in_m) {
                const int slot = cnt[m] + __popc(mm & mc_lanemask_lt());
                if (slot < cap)
                    sites[(m * B + b) * cap + slot] = g;
                else
                    check_fail(check, kCheckMcOverflow, slot, g);
            }
            cnt[m] += __popc(mm);
        }
        __syncwarp();
    }
    if (lane == 0)
        for (int m = 0; m < kMcMaxModels; ++m) st->slot_count[b][m] = m < sel.n_models ? min(cnt[m], cap) : 0;
}

// Warp per (model, slot, row): the row's pair geometry with its slot's atom at the trial position.
__global__ void k_mc_trial_geometry_batch(const McDev *st, int n_models, const int *__restrict__ sites, int cap,
                                          int pmax, int B, const int64_t *__restrict__ start,
                                          const int *__restrict__ list, const int *__restrict__ nspecies,
                                          const int *__restrict__ site_struct, const StructDesc *__restrict__ sd,
                                          const double *__restrict__ pos, double *__restrict__ txyz,
                                          double *__restrict__ trjs, int *__restrict__ tnsp, int *check)
{
    const int lane = threadIdx.x & 31;
    const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (w >= n_models * B * cap) return;
    const int m = w / (B * cap), rem = w - m * B * cap, b = rem / cap, r = rem - b * cap;
    const size_t base = (size_t)w * pmax;
    int ns = 0, g = 0;
    if (st->slot_flag[b] == 0 && r < st->slot_count[b][m]) {
        g = sites[(m * B + b) * cap + r];
        ns = (int)(start[g + 1] - start[g]);
        if (ns > pmax) {
            if (lane == 0) check_fail(check, kCheckMcOverflow, g, ns);
            ns = pmax;
        }
    }
    const int a = st->slot_atom[b];
    const double pn[3] = {st->slot_new[b][0], st->slot_new[b][1], st->slot_new[b][2]};
    for (int t = lane; t < pmax; t += 32) {
        double x0 = 0.0, x1 = 0.0, x2 = 0.0, rr = 0.0;
        int sp = 0;
        if (t < ns) {
            const int64_t k = start[g] + t;
            sp = nspecies[k];
            if (t > 0) {
                const StructDesc &S = sd[site_struct[g]];
                double pi[3], pj[3], dist[3];
                sc_position_moved(S, pos, g - S.atom_off + 1, a, pn, pi);
                sc_position_moved(S, pos, list[k], a, pn, pj);
                get_distance_dev(pi, pj, S, dist, &rr);
                x0 = dist[0];
                x1 = dist[1];
                x2 = dist[2];
            }
        }
        txyz[3 * (base + t)] = x0;
        txyz[3 * (base + t) + 1] = x1;
        txyz[3 * (base + t) + 2] = x2;
        trjs[base + t] = rr;
        tnsp[base + t] = sp;
    }
}

// One warp: settles the batch's proposals in proposal order. A slot's energies stay valid unless an
// accepted earlier slot of the batch moved an atom within 2 rc + |d_i| + |d_b| of it; such a slot is
// deferred to the next batch, and so is every later slot within that range of a deferred one (its
// move could change the deferred proposal's energies), so each proposal is decided from the state
// that settling them one at a time gives it: the chain is the one-at-a-time chain.
__global__ void k_mc_resolve_batch(McDev *st, int n_models, const int *__restrict__ sites, int cap, int B,
                                   const double *__restrict__ etrial, double *__restrict__ ecache, int n_atoms,
                                   double *__restrict__ pos, double *__restrict__ dacc,
                                   const double *__restrict__ prop_u, int u_stride, double temperature,
                                   double rc_sel, double skin, const int *__restrict__ site_struct,
                                   const StructDesc *__restrict__ sd, McLogs logs, int screened,
                                   const float *__restrict__ es_trial, float *__restrict__ es_cache)
{
    const int lane = threadIdx.x & 31;
    __shared__ int acc_slot[kMcMaxBatch], def_slot[kMcMaxBatch];
    if (st->status != kMcRunning) return;
    int n_acc = 0, n_def = 0, settled = 0;
    int b = 0;
    for (; b < B; ++b) {
        const int flag = st->slot_flag[b];
        if (flag == 1) break;
        if (flag == 2) {
            if (lane == 0) st->status = kMcNeedRebuild;
            break;
        }
        const long long k = st->slot_prop[b];
        const int a = st->slot_atom[b];
        const double dn = st->slot_dn[b];
        // blocked by an accepted or a deferred earlier slot within 2 rc + |d_i| + |d_b|
        bool conflict = false;
        if (lane < n_acc + n_def) {
            const int i = lane < n_acc ? acc_slot[lane] : def_slot[lane - n_acc];
            const int ai = st->slot_atom[i];
            if (ai == a) {
                conflict = true;
            } else if (site_struct[ai] == site_struct[a]) {
                const StructDesc &S = sd[site_struct[a]];
                if (S.rep[0] * S.rep[1] * S.rep[2] > 1) {
                    // a replicated cell moves every replica of the atom: its images repeat with the
                    // primitive cell, which is smaller than twice the list cutoff
                    conflict = true;
                } else {
                    double dist[3], dd;
                    get_distance_dev(st->slot_old[i], st->slot_old[b], S, dist, &dd);
                    conflict = !(dd >= 2.0 * rc_sel + st->slot_dn[i] + dn + 1e-9);
                }
            }
        }
        if (__any_sync(0xffffffffu, conflict)) {
            if (lane == 0) def_slot[n_def] = b;
            ++n_def;
            __syncwarp();
            continue;
        }
        if (st->maxD + dacc[a] + dn >= skin) {
            if (lane == 0) st->status = kMcNeedRebuild;
            break;
        }
        if (screened) {
            // stage 1 was decided before the exact energies (k_mc_screen_batch)
            if (lane == 0) {
                st->s_prop += 1;
                if (logs.de_screen) logs.de_screen[k] = st->slot_des[b];
            }
            if (!st->slot_pass[b]) {
                if (lane == 0) {
                    if (logs.de) logs.de[k] = __longlong_as_double(0x7ff8000000000000ll);
                    if (logs.acc) logs.acc[k] = 0;
                    if (logs.stage) logs.stage[k] = 1;
                }
                __syncwarp();
                ++settled;
                continue;
            }
        }
        // dE in the fixed order of the one-at-a-time kernel
        double de = 0.0;
        for (int m = 0; m < n_models; ++m) {
            const int c = st->slot_count[b][m];
            const int *sm = sites + (size_t)(m * B + b) * cap;
            const double *em = etrial + (size_t)m * B * cap + (size_t)b * cap;
            for (int r = lane; r < c; r += 32) de += em[r] - ecache[(size_t)m * n_atoms + sm[r]];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) de += __shfl_xor_sync(0xffffffffu, de, o);
        int accept = 0;
        if (lane == 0) {
            // delayed acceptance, stage 2 (Christen and Fox): dE - dE_s against the second deviate
            const double x = screened ? de - st->slot_des[b] : de;
            double p = exp(-x / (mc_kb() * temperature));
            p = p < 1.0 ? p : 1.0;
            accept = p > (screened ? prop_u[2 * k + 1] : prop_u[(long long)u_stride * k]) ? 1 : 0;
            if (screened) {
                st->s_pass += 1;
                st->s_conf += accept;
            }
            if (logs.de) logs.de[k] = de;
            if (logs.acc) logs.acc[k] = (unsigned char)accept;
            if (logs.stage) logs.stage[k] = 2;
        }
        accept = __shfl_sync(0xffffffffu, accept, 0);
        if (accept) {
            for (int m = 0; m < n_models; ++m) {
                const int c = st->slot_count[b][m];
                const int *sm = sites + (size_t)(m * B + b) * cap;
                const double *em = etrial + (size_t)m * B * cap + (size_t)b * cap;
                for (int r = lane; r < c; r += 32) ecache[(size_t)m * n_atoms + sm[r]] = em[r];
            }
            if (screened) {
                const int c = st->slot_count[b][0];
                const int *sm = sites + (size_t)b * cap;
                for (int r = lane; r < c; r += 32) es_cache[sm[r]] = es_trial[(size_t)b * cap + r];
            }
            if (lane == 0) {
                for (int q = 0; q < 3; ++q) pos[3 * (size_t)a + q] = st->slot_new[b][q];
                dacc[a] += dn;
                if (dacc[a] > st->maxD) st->maxD = dacc[a];
                st->accepted += 1;
                acc_slot[n_acc] = b;
            }
            ++n_acc;
        }
        __syncwarp();
        ++settled;
    }
    if (lane == 0) {
        // unsettled: the deferred slots and every slot from b on that holds a proposal, in order
        long long pend[kMcMaxBatch];
        int np = 0;
        long long top = st->next;  // one past the largest proposal of the batch
        for (int i = 0; i < n_def; ++i) pend[np++] = st->slot_prop[def_slot[i]];
        for (int i = 0; i < B; ++i)
            if (st->slot_flag[i] != 1) {
                if (i >= b) pend[np++] = st->slot_prop[i];
                if (st->slot_prop[i] + 1 > top) top = st->slot_prop[i] + 1;
            }
        // a run of consecutive proposals ending at top is the plain state next = its first
        bool run = true;
        for (int i = 0; i < np; ++i) run = run && pend[i] == top - np + i;
        if (run) {
            st->next = top - np;
            st->n_pend = 0;
        } else {
            st->next = top;
            st->n_pend = np;
            for (int i = 0; i < np; ++i) st->pend[i] = pend[i];
        }
        st->serial += 1;
        st->batches += 1;
        st->batch_resolved += settled;
    }
}

int mc_select_batch(tgap_context *ctx, McDev *d_st, const NeighborBatch &nb, const McModelSel &sel, double rc_sel,
                    double skin, const int *d_prop_atom, const double *d_prop_disp, const double *d_dacc,
                    long long *d_mark, int *d_sites, int cap, int B)
{
    k_mc_select_batch<<<B, 32, 0, ctx->stream>>>(d_st, nb.start.as<int64_t>(), nb.list.as<int>(), nb.jatom.as<int>(),
                                                 nb.site_struct.as<int>(), nb.d_structs.as<StructDesc>(),
                                                 nb.positions.as<double>(), nb.species_sc.as<int>(), sel, rc_sel,
                                                 skin, d_prop_atom, d_prop_disp, d_dacc, d_mark, nb.n_atoms, d_sites,
                                                 cap, B, ctx->d_check);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

int mc_trial_geometry_batch(tgap_context *ctx, const McDev *d_st, const NeighborBatch &nb, int n_models,
                            const int *d_sites, int cap, int pmax, int B, double *d_txyz, double *d_trjs, int *d_tnsp)
{
    const int warps = n_models * B * cap, T = 128;
    k_mc_trial_geometry_batch<<<(warps + T / 32 - 1) / (T / 32), T, 0, ctx->stream>>>(
        d_st, n_models, d_sites, cap, pmax, B, nb.start.as<int64_t>(), nb.list.as<int>(), nb.nspecies.as<int>(),
        nb.site_struct.as<int>(), nb.d_structs.as<StructDesc>(), nb.positions.as<double>(), d_txyz, d_trjs, d_tnsp,
        ctx->d_check);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

int mc_resolve_batch(tgap_context *ctx, McDev *d_st, const NeighborBatch &nb, int n_models, const int *d_sites,
                     int cap, int B, const double *d_etrial, double *d_ecache, double *d_positions, double *d_dacc,
                     const double *d_prop_u, int u_stride, double temperature, double rc_sel, double skin,
                     McLogs logs, int screened, const float *d_es_trial, float *d_es_cache)
{
    k_mc_resolve_batch<<<1, 32, 0, ctx->stream>>>(d_st, n_models, d_sites, cap, B, d_etrial, d_ecache, nb.n_atoms,
                                                  d_positions, d_dacc, d_prop_u, u_stride, temperature, rc_sel, skin,
                                                  nb.site_struct.as<int>(), nb.d_structs.as<StructDesc>(), logs,
                                                  screened, d_es_trial, d_es_cache);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

// Warp b: slot b's screen energy change over its model-0 rows in a fixed reduction order and the
// stage-1 test against u1 of the slot's proposal (a slot the batch does not settle is evaluated
// again in the next batch). Then one thread
// per row tile of 128 trial rows: the tile is needed when a passing slot's rows fall into it.
__global__ void k_mc_screen_batch(McDev *st, const int *__restrict__ sites, int cap, int B,
                                  const float *__restrict__ es_trial, const float *__restrict__ es_cache,
                                  const double *__restrict__ prop_u, double temperature, int *__restrict__ tile_skip,
                                  int n_tiles)
{
    const int lane = threadIdx.x & 31, b = threadIdx.x >> 5;
    const bool running = st->status == kMcRunning;
    if (b < B) {
        int pass = 0;
        double des = 0.0;
        if (running && st->slot_flag[b] == 0) {
            const int c = st->slot_count[b][0];
            const int *sb = sites + (size_t)b * cap;
            const float *eb = es_trial + (size_t)b * cap;
            for (int r = lane; r < c; r += 32) des += (double)eb[r] - (double)es_cache[sb[r]];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) des += __shfl_xor_sync(0xffffffffu, des, o);
            double p = exp(-des / (mc_kb() * temperature));
            p = p < 1.0 ? p : 1.0;
            pass = p > prop_u[2 * st->slot_prop[b]] ? 1 : 0;
        }
        if (lane == 0) {
            st->slot_des[b] = des;
            st->slot_pass[b] = pass;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n_tiles; t += blockDim.x) {
        int need = 0;
        const int r0 = 128 * t, r1 = 128 * t + 127;
        for (int bb = r0 / cap; bb <= r1 / cap && bb < B; ++bb) need |= st->slot_pass[bb];
        tile_skip[t] = need ? 0 : 1;
    }
}

int mc_screen_batch(tgap_context *ctx, McDev *d_st, const int *d_sites, int cap, int B, const float *d_es_trial,
                    const float *d_es_cache, const double *d_prop_u, double temperature, int *d_tile_skip,
                    int n_tiles)
{
    if (B < 1 || B > kMcMaxBatch) return set_error(ctx, TGAP_ERR_ARGUMENT, "screen batch width");
    k_mc_screen_batch<<<1, 32 * B, 0, ctx->stream>>>(d_st, d_sites, cap, B, d_es_trial, d_es_cache, d_prop_u,
                                                      temperature, d_tile_skip, n_tiles);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

int mc_select(tgap_context *ctx, McDev *d_st, const NeighborBatch &nb, const McModelSel &sel, double rc_sel,
              double skin, const int *d_prop_atom, const double *d_prop_disp, const double *d_dacc,
              long long *d_mark, int *d_sites, int cap)
{
    k_mc_select<<<1, 32, 0, ctx->stream>>>(d_st, nb.start.as<int64_t>(), nb.list.as<int>(), nb.jatom.as<int>(),
                                           nb.site_struct.as<int>(), nb.d_structs.as<StructDesc>(),
                                           nb.positions.as<double>(), nb.species_sc.as<int>(), sel, rc_sel, skin,
                                           d_prop_atom, d_prop_disp, d_dacc, d_mark, d_sites, cap, ctx->d_check);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

int mc_trial_geometry(tgap_context *ctx, const McDev *d_st, const NeighborBatch &nb, int n_models,
                      const int *d_sites, int cap, int pmax, double *d_txyz, double *d_trjs, int *d_tnsp)
{
    const int warps = n_models * cap, T = 128;
    k_mc_trial_geometry<<<(warps + T / 32 - 1) / (T / 32), T, 0, ctx->stream>>>(
        d_st, n_models, d_sites, cap, pmax, nb.start.as<int64_t>(), nb.list.as<int>(), nb.nspecies.as<int>(),
        nb.site_struct.as<int>(), nb.d_structs.as<StructDesc>(), nb.positions.as<double>(), d_txyz, d_trjs, d_tnsp,
        ctx->d_check);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

int mc_screen_stage(tgap_context *ctx, McDev *d_st, const int *d_sites, const float *d_es_trial,
                    const float *d_es_cache, const double *d_prop_u, double temperature, McLogs logs)
{
    k_mc_screen_stage<<<1, 32, 0, ctx->stream>>>(d_st, d_sites, d_es_trial, d_es_cache, d_prop_u, temperature, logs);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

int mc_accept(tgap_context *ctx, McDev *d_st, int n_models, const int *d_sites, int cap, const double *d_etrial,
              double *d_ecache, int n_atoms, double *d_positions, double *d_dacc, const double *d_prop_u,
              double temperature, McLogs logs, int screened, int u_stride, const float *d_es_trial,
              float *d_es_cache)
{
    k_mc_accept<<<1, 32, 0, ctx->stream>>>(d_st, n_models, d_sites, cap, d_etrial, d_ecache, n_atoms, d_positions,
                                           d_dacc, d_prop_u, temperature, logs, screened, u_stride, d_es_trial,
                                           d_es_cache);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

int mc_begin(tgap_context *ctx, McDev *d_st, long long n_prop)
{
    k_mc_begin<<<1, 1, 0, ctx->stream>>>(d_st, n_prop);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

int mc_lists_rebuilt(tgap_context *ctx, McDev *d_st, double *d_dacc, int n_atoms)
{
    k_mc_lists_rebuilt<<<(n_atoms + 255) / 256, 256, 0, ctx->stream>>>(d_st, d_dacc, n_atoms);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

}  // namespace tgap
