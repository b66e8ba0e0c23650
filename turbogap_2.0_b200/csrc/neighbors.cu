// Neighbor-list build for batches of periodic structures (sm_100a).
//
// Reproduces build_neighbors_list (src/neighbors/neighbors_interface.f90:144-524) pair for
// pair: self first; orthorhombic boxes that need no replicas use the linked-cell traversal
// (cell of an atom from the minimum image about the box centre, :311-321; cells visited
// z -> y -> x over +-1 with the mx/my/mz in {1,2} skips, :352-363; atoms of a cell in
// decreasing index, the order of the LIFO linked list, :329-330, :365-382); every other box
// uses the ascending brute-force scan over the supercell (:390-421). Distances follow
// get_distance (:547-643) operation by operation. This file is compiled with --fmad=false so
// no multiply-add is contracted and the accept test d < rcut_max sees the same bits as the
// Fortran arithmetic.
//
// One thread owns one central site in both passes (count, then fill at the scanned offset),
// so the list order inside a site is the sequential order of the reference.
#include <cub/cub.cuh>

#include "neighbors.h"
#include "neighbors_device.cuh"

namespace tgap {

// Cell coordinates (1-based i2, j2, k2) and the linear cell index of a position.
__device__ void cell_of(const double *pos, const StructDesc &S, int *i2, int *j2, int *k2,
                        int *lin)
{
    const double tol = 1.0e-10;
    double centre[3] = {S.a[0] / 2.0, S.b[1] / 2.0, S.c[2] / 2.0};
    double dist[3], d;
    get_distance_dev(centre, pos, S, dist, &d);
    double p[3] = {dist[0] + centre[0], dist[1] + centre[1], dist[2] + centre[2]};
    int ci = (int)(p[0] / (S.a[0] + tol) * S.mx);
    int cj = (int)(p[1] / (S.b[1] + tol) * S.my);
    int ck = (int)(p[2] / (S.c[2] + tol) * S.mz);
    *i2 = 1 + ci;
    *j2 = 1 + cj;
    *k2 = 1 + ck;
    *lin = i_modulo(ci, S.mx) + i_modulo(cj, S.my) * S.mx + i_modulo(ck, S.mz) * S.my * S.mx;
}

__global__ void k_cell_count(int n_atoms_total, const int *site_struct, const StructDesc *sd,
                             const double *pos_sc, int *atom_cell, int *cell_count)
{
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_atoms_total) return;
    const StructDesc &S = sd[site_struct[g]];
    if (S.cell_off < 0) return;
    int local = g - S.atom_off;
    int i2, j2, k2, lin;
    cell_of(pos_sc + 3 * (size_t)(S.sc_off + local), S, &i2, &j2, &k2, &lin);
    atom_cell[g] = S.cell_off + lin;
    atomicAdd(cell_count + S.cell_off + lin, 1);
}

__global__ void k_cell_fill(int n_atoms_total, const int *site_struct, const StructDesc *sd,
                            const int *atom_cell, const int *cell_start, int *cell_cursor,
                            int *cell_atoms)
{
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_atoms_total) return;
    const StructDesc &S = sd[site_struct[g]];
    if (S.cell_off < 0) return;
    int c = atom_cell[g];
    int slot = atomicAdd(cell_cursor + c, 1);
    cell_atoms[cell_start[c] + slot] = g - S.atom_off + 1;  // 1-based local index
}

// Each cell's members (in cell_tmp, in arrival order) written to cell_atoms in decreasing index,
// the LIFO order of the reference linked list. One warp per cell: a member's slot is the number
// of members with a larger index.
__global__ void k_cell_sort(int n_cells, const int *cell_start, const int *cell_tmp, int *cell_atoms)
{
    const int lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (c >= n_cells) return;
    const int b = cell_start[c], e = cell_start[c + 1];
    for (int t0 = b; t0 < e; t0 += 32) {
        const int t = t0 + lane;
        const int v = t < e ? cell_tmp[t] : 0;
        int rank = 0;
        for (int u0 = b; u0 < e; u0 += 32) {
            const int w = u0 + lane < e ? cell_tmp[u0 + lane] : 0;
            const int m = e - u0 < 32 ? e - u0 : 32;
            for (int q = 0; q < m; ++q) rank += __shfl_sync(0xffffffffu, w, q) > v ? 1 : 0;
        }
        if (t < e) cell_atoms[b + rank] = v;
    }
}

__device__ __forceinline__ unsigned nb_lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Width of a site's row in the staging area: the count pass of a linked-cell site with at most this
// many list entries (self included) also writes them, in list order, into its row, and the fill
// pass copies the row instead of walking the cells again.
constexpr int kStageW = 96;

// One warp per site; FILL=false counts the site's pairs, FILL=true writes them in the
// reference order. Linked-cell path: lane c < 27 finds neighbor cell c of the z -> y -> x
// traversal (c = 9 dz + 3 dy + dx) and its member range (members in decreasing index); a warp
// scan of the ranges' lengths lays the 27 cells' candidates end to end, and the warp tests them
// 32 at a time, each accepted pair placed by a ballot prefix, which keeps the cell-by-cell order.
// Brute-force path: the warp strides over the supercell in ascending order and compacts with a
// ballot. With stage (int [n_atoms][kStageW]) and staged (int [n_atoms]) given, the count pass
// also writes the rows that fit and marks them; the fill pass copies a marked row to its place in
// the list (bounded by the site's offsets) and walks the cells only for the other sites.
template <bool FILL>
__global__ void __launch_bounds__(128) k_site_pairs(int n_atoms_total, const int *site_struct,
                                                    const StructDesc *sd, const double *pos_sc,
                                                    const int *cell_start, const int *cell_atoms,
                                                    int64_t *counts, const int64_t *start, int *list,
                                                    int *check, int *stage, int *staged)
{
    const int lane = threadIdx.x & 31;
    const int g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (g >= n_atoms_total) return;
    if (FILL && staged && staged[g]) {
        const int64_t b = start[g], len = start[g + 1] - b;
        const int *row = stage + (size_t)g * kStageW;
        for (int j = lane; j < len && j < kStageW; j += 32) list[b + j] = row[j];
        return;
    }
    const StructDesc &S = sd[site_struct[g]];
    const int i = g - S.atom_off + 1;  // 1-based local site
    const double *pi = pos_sc + 3 * (size_t)(S.sc_off + i - 1);
    const double rc = S.rcut;
    const int64_t w0 = FILL ? start[g] : 0;
    const int64_t w_end = FILL ? start[g + 1] : 0;
    // the fill pass repeats the count pass, so it never reaches w_end; checked all the same
    auto put = [&](int64_t w, int v) {
        if (w < w_end)
            list[w] = v;
        else
            check_fail(check, kCheckListOverrun, g, v);
    };
    if (FILL && lane == 0) put(w0, i);
    if (S.cell_off >= 0) {
        int i2, j2, k2, lin;
        cell_of(pi, S, &i2, &j2, &k2, &lin);
        const int mx = S.mx, my = S.my, mz = S.mz;
        int c = -1;
        if (lane < 27) {
            const int k3 = k2 - 1 + lane / 9, j3 = j2 - 1 + (lane / 3) % 3, i3 = i2 - 1 + lane % 3;
            const bool skip = (mz == 1 && k3 != 1) || (mz == 2 && k2 == 1 && k3 == 0) ||
                              (mz == 2 && k2 == 2 && k3 == 3) || (my == 1 && j3 != 1) ||
                              (my == 2 && j2 == 1 && j3 == 0) || (my == 2 && j2 == 2 && j3 == 3) ||
                              (mx == 1 && i3 != 1) || (mx == 2 && i2 == 1 && i3 == 0) ||
                              (mx == 2 && i2 == 2 && i3 == 3);
            if (!skip)
                c = S.cell_off + i_modulo(i3 - 1, mx) + i_modulo(j3 - 1, my) * mx + i_modulo(k3 - 1, mz) * mx * my;
        }
        const int t0 = c >= 0 ? cell_start[c] : 0, nc = c >= 0 ? cell_start[c + 1] - t0 : 0;
        // the candidates of the 27 cells in traversal order (cell by lane, then the cell's sorted
        // atoms) are walked 32 at a time: lane u takes candidate b + u, the accepted ones keep their
        // order through a ballot, so the list comes out as a cell-by-cell walk would write it
        int incl = nc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        int *row = !FILL && stage ? stage + (size_t)g * kStageW : nullptr;
        if (row && lane == 0) row[0] = i;
        int acc = 0;  // pairs accepted so far (the self entry not counted)
        for (int b = 0; b < total; b += 32) {
            const int u = b + lane;
            // the cell holding candidate u: the first lane whose inclusive count exceeds u
            int L = 0;
#pragma unroll
            for (int st = 16; st > 0; st >>= 1)
                if (__shfl_sync(0xffffffffu, incl, L + st - 1) <= u) L += st;
            const int base = __shfl_sync(0xffffffffu, t0, L) - __shfl_sync(0xffffffffu, incl - nc, L);
            bool ok = false;
            int k = 0;
            if (u < total) {
                k = cell_atoms[base + u];
                if (k != i) {
                    double dist[3], d;
                    get_distance_dev(pi, pos_sc + 3 * (size_t)(S.sc_off + k - 1), S, dist, &d);
                    ok = d < rc;
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            const int w = 1 + acc + __popc(m & nb_lanemask_lt());
            if (ok) {
                if (FILL)
                    put(w0 + w, k);
                else if (row && w < kStageW)
                    row[w] = k;
            }
            acc += __popc(m);
        }
        if (!FILL && lane == 0) {
            counts[g] = 1 + acc;
            if (staged) staged[g] = row && 1 + acc <= kStageW ? 1 : 0;
        }
    } else {
        int64_t w = w0 + 1, n = 1;
        for (int jb = 1; jb <= S.n_sc; jb += 32) {
            const int j = jb + lane;
            bool ok = false;
            if (j <= S.n_sc && j != i) {
                double dist[3], d;
                get_distance_dev(pi, pos_sc + 3 * (size_t)(S.sc_off + j - 1), S, dist, &d);
                ok = d < rc;
            }
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            if (FILL && ok) put(w + __popc(m & nb_lanemask_lt()), j);
            w += __popc(m);
            n += __popc(m);
        }
        if (!FILL && lane == 0) {
            counts[g] = n;
            if (staged) staged[g] = 0;
        }
    }
}

// Geometry of every pair (neighbors_interface.f90:467-510); angles only when requested. With
// FROM_POS the supercell positions are formed from the primitive ones on the fly (no replicate
// pass; only for batches whose supercells are pure replicas). With rjs null only the per-pair
// species and atom maps are written (the descriptor forward writes the geometry itself).
template <bool FROM_POS>
__global__ void k_pair_geometry(int n_atoms_total, const int *site_struct, const StructDesc *sd,
                                const double *pos_sc, const double *pos, const int *species_sc,
                                const int64_t *start, const int *list, double *rjs, double *xyz, double *thetas,
                                double *phis, int *nspecies, int *jatom)
{
    // one warp per site
    const int g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (g >= n_atoms_total) return;
    const StructDesc &S = sd[site_struct[g]];
    const int i = g - S.atom_off + 1;
    double pi_buf[3];
    const double *pi = pos_sc + 3 * (size_t)(S.sc_off + i - 1);
    if (FROM_POS) {
        sc_position(S, pos, i, pi_buf);
        pi = pi_buf;
    }
    const int64_t b = start[g], e = start[g + 1];
    for (int64_t k = b + (threadIdx.x & 31); k < e; k += 32) {
        int j = list[k];
        if (jatom) jatom[k] = S.atom_off + (j - 1) % S.n;
        if (nspecies) nspecies[k] = species_sc[S.sc_off + j - 1];
        if (!rjs) continue;
        if (k == b) {
            rjs[k] = 0.0;
            xyz[3 * k] = xyz[3 * k + 1] = xyz[3 * k + 2] = 0.0;
            if (thetas) thetas[k] = 0.0;
            if (phis) phis[k] = 0.0;
            continue;
        }
        double pj_buf[3];
        const double *pj = pos_sc + 3 * (size_t)(S.sc_off + j - 1);
        if (FROM_POS) {
            sc_position(S, pos, j, pj_buf);
            pj = pj_buf;
        }
        double dist[3], d;
        get_distance_dev(pi, pj, S, dist, &d);
        rjs[k] = d;
        xyz[3 * k] = dist[0];
        xyz[3 * k + 1] = dist[1];
        xyz[3 * k + 2] = dist[2];
        if (thetas) {
            if (fabs(dist[2]) >= d)
                thetas[k] = dist[2] > 0.0 ? 0.0 : acos(-1.0);
            else
                thetas[k] = acos(dist[2] / d);
        }
        if (phis) phis[k] = atan2(dist[1], dist[0]);
    }
}

__global__ void k_start_from_nneigh(int n, const int *n_neigh, int64_t *cnt)
{
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < n) cnt[g] = n_neigh[g];
    if (g == n) cnt[g] = 0;
}

__global__ void k_nneigh_from_counts(int n, const int64_t *cnt, int *n_neigh)
{
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < n) n_neigh[g] = (int)cnt[g];
}

// Device-side rebuild, one CTA: n_neigh from the list offsets, which stay as they are when the
// lists fit the reserved pair capacity cap. Longer lists are recorded in the check word and every
// offset is clamped to cap - 1 (start[i] = min(start[i], cap - 1)): each later pass, the self entry
// that the descriptor kernels read at start[i] included, stays inside the arrays; the tail sites
// get no pairs and the fill records the site it cut. The decision is taken once, from start[n],
// before any offset changes; thread i reading start[i + 1] while another thread clamps it gets
// the same min(., cap - 1) either way. The unclamped total is kept in *total.
__global__ void k_fit_pairs(int n, int64_t *start, int *n_neigh, int64_t cap, int *check, int64_t *total)
{
    __shared__ int over;
    if (threadIdx.x == 0) {
        *total = start[n];
        over = start[n] > cap;
        if (over) check_fail(check, kCheckPairCapacity, n, (long long)start[n]);
    }
    __syncthreads();
    const int64_t lim = cap - 1;
    for (int i = threadIdx.x; i <= n; i += blockDim.x) {
        int64_t a = start[i];
        if (i < n) {
            int64_t b = start[i + 1];
            if (over) {
                a = a < lim ? a : lim;
                b = b < lim ? b : lim;
            }
            n_neigh[i] = (int)(b - a);
        } else if (over) {
            a = a < lim ? a : lim;
        }
        if (over) start[i] = a;
    }
}

// Systems up to this many sites take the list offsets and the capacity fit from one launch.
constexpr int kScanFitMax = 16384;

// The small-system form of the offset scan and k_fit_pairs in one CTA of 1024 threads: start[0, n] =
// the exclusive sum of the per-site counts (start[n] the total, also kept in *total), then the same
// capacity fit. The counts are read in chunks of 1024 consecutive sites (all chunks' loads issued
// first), each chunk scanned across the block and carried into the next.
__global__ void __launch_bounds__(1024) k_scan_fit_pairs(int n, const int64_t *counts, int64_t *start, int *n_neigh,
                                                         int64_t cap, int *check, int64_t *total)
{
    constexpr int R = kScanFitMax / 1024;
    __shared__ int64_t wsum[32];
    __shared__ int over;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int chunks = (n + 1023) / 1024;
    int64_t v[R];
#pragma unroll
    for (int k = 0; k < R; ++k) v[k] = k < chunks && k * 1024 + t < n ? counts[k * 1024 + t] : 0;
    // inclusive prefix within each chunk, the chunks' totals carried forward
    int64_t carry = 0;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        if (k >= chunks) break;
        int64_t x = v[k];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            int64_t z = wsum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t y = __shfl_up_sync(0xffffffffu, z, o);
                if (lane >= o) z += y;
            }
            wsum[lane] = z;
        }
        __syncthreads();
        const int64_t incl = carry + (w > 0 ? wsum[w - 1] : 0) + x;
        carry += wsum[31];
        v[k] = incl - v[k];  // exclusive prefix of site k * 1024 + t
        __syncthreads();     // wsum is rewritten for the next 1024 sites
    }
    const int64_t tot = carry;
    if (t == 0) {
        *total = tot;
        over = tot > cap;
        if (over) check_fail(check, kCheckPairCapacity, n, (long long)tot);
    }
    __syncthreads();
    const int64_t lim = cap - 1;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int i = k * 1024 + t;
        if (k >= chunks || i >= n) break;
        const int64_t a = v[k], z = a + counts[i];
        const int64_t a2 = over && a > lim ? lim : a, z2 = over && z > lim ? lim : z;
        start[i] = a2;
        n_neigh[i] = (int)(z2 - a2);
    }
    if (t == 0) start[n] = over && tot > lim ? lim : tot;
}

static int scan_i64(tgap_context *ctx, DevBuf &tmp, const int64_t *in, int64_t *out, int n)
{
    size_t bytes = 0;
    TGAP_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, ctx->stream));
    if (tmp.ensure(bytes)) return set_error(ctx, TGAP_ERR_NOMEM, "scan workspace");
    TGAP_CUDA(ctx, cub::DeviceScan::ExclusiveSum(tmp.ptr, bytes, in, out, n, ctx->stream));
    ctx->launches++;
    return TGAP_OK;
}

static int scan_i32(tgap_context *ctx, DevBuf &tmp, const int *in, int *out, int n)
{
    size_t bytes = 0;
    TGAP_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, ctx->stream));
    if (tmp.ensure(bytes)) return set_error(ctx, TGAP_ERR_NOMEM, "scan workspace");
    TGAP_CUDA(ctx, cub::DeviceScan::ExclusiveSum(tmp.ptr, bytes, in, out, n, ctx->stream));
    ctx->launches++;
    return TGAP_OK;
}

// ---------------------------------------------------------------------------- host side

static void host_dot_inverse(const double *a, const double *b, const double *c, double *inv)
{
    // neighbors_interface.f90:592-613, same operation order (host code is built without
    // floating-point contraction).
    auto dot = [](const double *x, const double *y) {
        double s = 0.0;
        s = s + x[0] * y[0];
        s = s + x[1] * y[1];
        s = s + x[2] * y[2];
        return s;
    };
    double m[3][3];
    m[0][0] = dot(a, a);
    m[0][1] = dot(a, b);
    m[0][2] = dot(a, c);
    m[1][0] = m[0][1];
    m[1][1] = dot(b, b);
    m[1][2] = dot(b, c);
    m[2][0] = m[0][2];
    m[2][1] = m[1][2];
    m[2][2] = dot(c, c);
    volatile double md = -(m[0][2] * m[0][2] * m[1][1]);
    md = md + 2.0 * m[0][1] * m[0][2] * m[1][2];
    md = md - m[0][0] * (m[1][2] * m[1][2]);
    md = md - m[0][1] * m[0][1] * m[2][2];
    md = md + m[0][0] * m[1][1] * m[2][2];
    double r[3][3];
    r[0][0] = m[1][1] * m[2][2] - m[1][2] * m[1][2];
    r[0][1] = m[0][2] * m[1][2] - m[0][1] * m[2][2];
    r[0][2] = m[0][1] * m[1][2] - m[0][2] * m[1][1];
    r[1][0] = r[0][1];
    r[1][1] = m[0][0] * m[2][2] - m[0][2] * m[0][2];
    r[1][2] = m[0][1] * m[0][2] - m[0][0] * m[1][2];
    r[2][0] = r[0][2];
    r[2][1] = r[1][2];
    r[2][2] = m[0][0] * m[1][1] - m[0][1] * m[0][1];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) inv[3 * i + j] = r[i][j] / md;
}

int make_struct_desc(const double a[3], const double b[3], const double c[3], int box_small,
                     double rcut, StructDesc *S)
{
    const double d_tol = 1.0e-6;
    std::memcpy(S->a, a, sizeof(S->a));
    std::memcpy(S->b, b, sizeof(S->b));
    std::memcpy(S->c, c, sizeof(S->c));
    S->ortho = std::fabs(a[1]) < d_tol && std::fabs(a[2]) < d_tol && std::fabs(b[0]) < d_tol &&
               std::fabs(b[2]) < d_tol && std::fabs(c[0]) < d_tol && std::fabs(c[1]) < d_tol;
    if (S->ortho) {
        S->a[1] = S->a[2] = S->b[0] = S->b[2] = S->c[0] = S->c[1] = 0.0;
    } else {
        host_dot_inverse(S->a, S->b, S->c, S->inv);
    }
    S->rcut = rcut;
    S->cell_off = -1;
    S->mx = S->my = S->mz = 0;
    if (S->ortho && !box_small) {
        S->mx = (int)(S->a[0] / rcut);
        S->my = (int)(S->b[1] / rcut);
        S->mz = (int)(S->c[2] / rcut);
        if (S->mx < 1 || S->my < 1 || S->mz < 1) return TGAP_ERR_ARGUMENT;
        S->cell_off = 0;  // set by the caller when batching
    }
    return TGAP_OK;
}

// The counting half of a rebuild: cell lists, per-site pair counts and their exclusive scan
// (start[0..n]). Stream-ordered only.
// scan = false leaves the offsets to the caller (counts only).
static int rebuild_count(tgap_context *ctx, NeighborBatch *nb, bool scan = true)
{
    const int n = nb->n_atoms;
    const int T = 128;
    const int grid = (n + T - 1) / T;
    const int wgrid = (n + T / 32 - 1) / (T / 32);  // one warp per site
    StructDesc *d_sd = nb->d_structs.as<StructDesc>();
    // cells
    if (nb->n_cells > 0) {
        TGAP_CUDA(ctx, cudaMemsetAsync(nb->cell_count.ptr, 0, sizeof(int) * (nb->n_cells + 1), ctx->stream));
        k_cell_count<<<grid, T, 0, ctx->stream>>>(n, nb->site_struct.as<int>(), d_sd, nb->pos_sc.as<double>(),
                                                  nb->atom_cell.as<int>(), nb->cell_count.as<int>());
        TGAP_LAUNCH_CHECK(ctx);
        int rc = scan_i32(ctx, nb->scan_tmp, nb->cell_count.as<int>(), nb->cell_start.as<int>(), nb->n_cells + 1);
        if (rc) return rc;
        TGAP_CUDA(ctx, cudaMemsetAsync(nb->cell_cursor.ptr, 0, sizeof(int) * nb->n_cells, ctx->stream));
        k_cell_fill<<<grid, T, 0, ctx->stream>>>(n, nb->site_struct.as<int>(), d_sd, nb->atom_cell.as<int>(),
                                                 nb->cell_start.as<int>(), nb->cell_cursor.as<int>(),
                                                 nb->cell_tmp.as<int>());
        TGAP_LAUNCH_CHECK(ctx);
        k_cell_sort<<<(nb->n_cells + T / 32 - 1) / (T / 32), T, 0, ctx->stream>>>(
            nb->n_cells, nb->cell_start.as<int>(), nb->cell_tmp.as<int>(), nb->cell_atoms.as<int>());
        TGAP_LAUNCH_CHECK(ctx);
    }
    // the staging rows (sized with the batch; no allocation once a list exists)
    if (nb->stage.ensure(sizeof(int) * (size_t)n * kStageW) || nb->staged.ensure(sizeof(int) * (size_t)n))
        return set_error(ctx, TGAP_ERR_NOMEM, "pair staging rows");
    k_site_pairs<false><<<wgrid, T, 0, ctx->stream>>>(n, nb->site_struct.as<int>(), d_sd, nb->pos_sc.as<double>(),
                                                      nb->cell_start.as<int>(), nb->cell_atoms.as<int>(),
                                                      nb->counts.as<int64_t>(), nullptr, nullptr, nullptr,
                                                      nb->stage.as<int>(), nb->staged.as<int>());
    TGAP_LAUNCH_CHECK(ctx);
    if (!scan) return TGAP_OK;
    TGAP_CUDA(ctx, cudaMemsetAsync(nb->counts.as<int64_t>() + n, 0, sizeof(int64_t), ctx->stream));
    return scan_i64(ctx, nb->scan_tmp, nb->counts.as<int64_t>(), nb->start.as<int64_t>(), n + 1);
}

// The filling half: each warp writes its site's pairs inside [start[g], start[g + 1]) (a site cut
// short is recorded in check when given).
static int rebuild_fill(tgap_context *ctx, NeighborBatch *nb, int *check)
{
    const int n = nb->n_atoms;
    const int T = 128;
    const int wgrid = (n + T / 32 - 1) / (T / 32);
    k_site_pairs<true><<<wgrid, T, 0, ctx->stream>>>(n, nb->site_struct.as<int>(), nb->d_structs.as<StructDesc>(),
                                                     nb->pos_sc.as<double>(), nb->cell_start.as<int>(),
                                                     nb->cell_atoms.as<int>(), nullptr, nb->start.as<int64_t>(),
                                                     nb->list.as<int>(), check, nb->stage.as<int>(),
                                                     nb->staged.as<int>());
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

int neighbors_rebuild_lists(tgap_context *ctx, NeighborBatch *nb, int64_t capacity, int64_t *n_pairs_out)
{
    const int n = nb->n_atoms;
    if (n <= 0) {
        *n_pairs_out = 0;
        return TGAP_OK;
    }
    const int T = 128;
    const int grid = (n + T - 1) / T;
    StageScope sc(ctx, "neighbors_rebuild");
    if (const int rc = rebuild_count(ctx, nb)) return rc;
    int64_t total = 0;
    TGAP_CUDA(ctx, cudaMemcpyAsync(&total, nb->start.as<int64_t>() + n, sizeof(int64_t), cudaMemcpyDeviceToHost,
                                   ctx->stream));
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *n_pairs_out = total;
    if (capacity >= 0 && total > capacity) return TGAP_ERR_CAPACITY;
    if (nb->ensure_pairs(total)) return set_error(ctx, TGAP_ERR_NOMEM, "pair arrays");
    nb->n_pairs = total;
    nb->count_on_device = false;
    k_nneigh_from_counts<<<grid, T, 0, ctx->stream>>>(n, nb->counts.as<int64_t>(), nb->n_neigh.as<int>());
    TGAP_LAUNCH_CHECK(ctx);
    return rebuild_fill(ctx, nb, ctx->d_check);
}

int neighbors_rebuild_lists_device(tgap_context *ctx, NeighborBatch *nb, bool report)
{
    const int n = nb->n_atoms;
    if (n <= 0) return TGAP_OK;
    if (!nb->list.ptr) return set_error(ctx, TGAP_ERR_ARGUMENT, "device-side list rebuild before any list was built");
    StageScope sc(ctx, "neighbors_rebuild");
    const bool small = n <= kScanFitMax;
    if (const int rc = rebuild_count(ctx, nb, !small)) return rc;
    int *check = report ? ctx->d_check : nullptr;
    if (small)
        k_scan_fit_pairs<<<1, 1024, 0, ctx->stream>>>(n, nb->counts.as<int64_t>(), nb->start.as<int64_t>(),
                                                      nb->n_neigh.as<int>(), nb->pair_capacity(), check,
                                                      nb->counts.as<int64_t>() + n);
    else
        k_fit_pairs<<<1, 1024, 0, ctx->stream>>>(n, nb->start.as<int64_t>(), nb->n_neigh.as<int>(),
                                                 nb->pair_capacity(), check, nb->counts.as<int64_t>() + n);
    TGAP_LAUNCH_CHECK(ctx);
    nb->count_on_device = true;
    return rebuild_fill(ctx, nb, check);
}

int neighbors_sync_count(tgap_context *ctx, NeighborBatch *nb)
{
    if (!nb->count_on_device) return TGAP_OK;
    int64_t total = 0;
    TGAP_CUDA(ctx, cudaMemcpyAsync(&total, nb->start.as<int64_t>() + nb->n_atoms, sizeof(int64_t),
                                   cudaMemcpyDeviceToHost, ctx->stream));
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    nb->n_pairs = total;
    nb->count_on_device = false;
    return TGAP_OK;
}

int neighbors_geometry(tgap_context *ctx, NeighborBatch *nb, bool with_angles, bool from_positions)
{
    const int n = nb->n_atoms;
    if (n <= 0) return TGAP_OK;
    const int T = 128;
    StageScope sc(ctx, "neighbors_geometry");
    auto kern = from_positions ? k_pair_geometry<true> : k_pair_geometry<false>;
    kern<<<(n + T / 32 - 1) / (T / 32), T, 0, ctx->stream>>>(
        n, nb->site_struct.as<int>(), nb->d_structs.as<StructDesc>(), nb->pos_sc.as<double>(),
        nb->positions.as<double>(), nb->species_sc.as<int>(), nb->start.as<int64_t>(), nb->list.as<int>(),
        nb->rjs.as<double>(), nb->xyz.as<double>(), with_angles ? nb->thetas.as<double>() : nullptr,
        with_angles ? nb->phis.as<double>() : nullptr, nb->nspecies.as<int>(), nb->jatom.as<int>());
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

int neighbors_maps(tgap_context *ctx, NeighborBatch *nb)
{
    const int n = nb->n_atoms;
    if (n <= 0) return TGAP_OK;
    const int T = 128;
    StageScope sc(ctx, "neighbors_maps");
    k_pair_geometry<false><<<(n + T / 32 - 1) / (T / 32), T, 0, ctx->stream>>>(
        n, nb->site_struct.as<int>(), nb->d_structs.as<StructDesc>(), nb->pos_sc.as<double>(), nullptr,
        nb->species_sc.as<int>(),
        nb->start.as<int64_t>(), nb->list.as<int>(), nullptr, nullptr, nullptr, nullptr, nb->nspecies.as<int>(),
        nb->jatom.as<int>());
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

int neighbors_refresh(tgap_context *ctx, NeighborBatch *nb)
{
    if (nb->replicated) return neighbors_geometry(ctx, nb, false, true);
    const int rc = neighbors_sync_positions(ctx, nb);
    return rc ? rc : neighbors_geometry(ctx, nb, false, false);
}

int neighbors_build(tgap_context *ctx, NeighborBatch *nb, int rebuild, int64_t capacity,
                    int64_t *n_pairs_out, bool with_angles)
{
    if (rebuild) {
        const int rc = neighbors_rebuild_lists(ctx, nb, capacity, n_pairs_out);
        if (rc) return rc;
    } else {
        if (const int rc = neighbors_sync_count(ctx, nb)) return rc;
        *n_pairs_out = nb->n_pairs;
    }
    return neighbors_geometry(ctx, nb, with_angles, false);
}

// Start offsets from a caller-provided n_neigh (geometry-only refresh of a given list).
int neighbors_set_counts(tgap_context *ctx, NeighborBatch *nb)
{
    const int n = nb->n_atoms;
    const int T = 128;
    k_start_from_nneigh<<<(n + 1 + T - 1) / T, T, 0, ctx->stream>>>(n, nb->n_neigh.as<int>(),
                                                                       nb->counts.as<int64_t>());
    TGAP_LAUNCH_CHECK(ctx);
    return scan_i64(ctx, nb->scan_tmp, nb->counts.as<int64_t>(), nb->start.as<int64_t>(), n + 1);
}

int NeighborBatch::ensure_pairs(int64_t P)
{
    // a quarter of headroom: the pair count of a running simulation fluctuates, and every
    // reallocation synchronizes the device and invalidates captured graphs
    size_t p = (size_t)(P > 0 ? P : 1);
    if (!list.ptr || p * sizeof(int) > list.bytes) p += p / 4 + 256;
    if (list.ensure(p * sizeof(int))) return 1;
    if (rjs.ensure(p * sizeof(double))) return 1;
    if (xyz.ensure(3 * p * sizeof(double))) return 1;
    if (thetas.ensure(p * sizeof(double))) return 1;
    if (phis.ensure(p * sizeof(double))) return 1;
    if (nspecies.ensure(p * sizeof(int))) return 1;
    if (jatom.ensure(p * sizeof(int))) return 1;
    return 0;
}

// Lay out the structures: supercell replication (read_xyz.f90:323-373, replica order
// a -> b -> c outer, atoms inner), cell grids, per-site structure ids. Host arrays in.
int neighbors_setup(tgap_context *ctx, NeighborBatch *nb, int n_structures, const int *offsets,
                    const double *positions, const double *boxes, const int *species,
                    double rcut, const int *force_small)
{
    std::vector<StructDesc> sd(n_structures);
    std::vector<double> pos_sc;
    std::vector<int> sp_sc, site_struct;
    int n_cells = 0, sc_total = 0;
    for (int b = 0; b < n_structures; ++b) {
        const int n = offsets[b + 1] - offsets[b];
        const double *bx = boxes + 9 * b;
        int idx[3];
        tgap_number_of_unit_cells(bx, bx + 3, bx + 6, rcut, idx);
        int small = idx[0] > 1 || idx[1] > 1 || idx[2] > 1;
        if (force_small && force_small[b]) small = 1;
        double a[3], bb[3], c[3];
        for (int q = 0; q < 3; ++q) {
            a[q] = bx[q];
            bb[q] = bx[3 + q];
            c[q] = bx[6 + q];
        }
        const int rep = idx[0] * idx[1] * idx[2];
        StructDesc &S = sd[b];
        S.atom_off = offsets[b];
        S.n = n;
        S.sc_off = sc_total;
        S.n_sc = n * rep;
        for (int i2 = 1; i2 <= idx[0]; ++i2)
            for (int j2 = 1; j2 <= idx[1]; ++j2)
                for (int k2 = 1; k2 <= idx[2]; ++k2)
                    for (int i = 0; i < n; ++i) {
                        const double *p = positions + 3 * (size_t)(offsets[b] + i);
                        for (int q = 0; q < 3; ++q) {
                            volatile double v = p[q] + (double)(i2 - 1) * a[q];
                            v = v + (double)(j2 - 1) * bb[q];
                            v = v + (double)(k2 - 1) * c[q];
                            pos_sc.push_back((double)v);
                        }
                        sp_sc.push_back(species[offsets[b] + i]);
                    }
        for (int q = 0; q < 3; ++q) {
            a[q] = (double)idx[0] * a[q];
            bb[q] = (double)idx[1] * bb[q];
            c[q] = (double)idx[2] * c[q];
        }
        for (int q = 0; q < 3; ++q) {
            S.pa[q] = bx[q];
            S.pb[q] = bx[3 + q];
            S.pc[q] = bx[6 + q];
        }
        int rc = make_struct_desc(a, bb, c, small, rcut, &S);
        if (rc) return set_error(ctx, rc, "structure %d: cell smaller than the cutoff", b);
        S.rep[0] = idx[0];
        S.rep[1] = idx[1];
        S.rep[2] = idx[2];
        if (S.cell_off >= 0) {
            S.cell_off = n_cells;
            n_cells += S.mx * S.my * S.mz;
        }
        sc_total += S.n_sc;
        for (int i = 0; i < n; ++i) site_struct.push_back(b);
    }
    nb->n_structures = n_structures;
    nb->n_atoms = offsets[n_structures];
    nb->replicated = true;  // supercells built here are replicas of the primitive cells
    nb->n_sc_total = sc_total;
    nb->n_cells = n_cells;
    nb->host_structs = sd;
    size_t N = (size_t)nb->n_atoms;
    if (nb->d_structs.ensure(sizeof(StructDesc) * n_structures) ||
        nb->pos_sc.ensure(sizeof(double) * 3 * (size_t)sc_total) ||
        nb->species_sc.ensure(sizeof(int) * (size_t)sc_total) ||
        nb->site_struct.ensure(sizeof(int) * N) || nb->atom_cell.ensure(sizeof(int) * N) ||
        nb->cell_count.ensure(sizeof(int) * (n_cells + 1)) ||
        nb->cell_start.ensure(sizeof(int) * (n_cells + 1)) ||
        nb->cell_cursor.ensure(sizeof(int) * (n_cells + 1)) ||
        nb->cell_atoms.ensure(sizeof(int) * (N + 1)) || nb->cell_tmp.ensure(sizeof(int) * (N + 1)) ||
        nb->counts.ensure(sizeof(int64_t) * (N + 1)) ||
        nb->start.ensure(sizeof(int64_t) * (N + 1)) || nb->n_neigh.ensure(sizeof(int) * N) ||
        nb->positions.ensure(sizeof(double) * 3 * N))
        return set_error(ctx, TGAP_ERR_NOMEM, "neighbor set-up");
    TGAP_CUDA(ctx, cudaMemcpyAsync(nb->d_structs.ptr, sd.data(), sizeof(StructDesc) * n_structures,
                                   cudaMemcpyHostToDevice, ctx->stream));
    TGAP_CUDA(ctx, cudaMemcpyAsync(nb->pos_sc.ptr, pos_sc.data(), sizeof(double) * pos_sc.size(),
                                   cudaMemcpyHostToDevice, ctx->stream));
    TGAP_CUDA(ctx, cudaMemcpyAsync(nb->species_sc.ptr, sp_sc.data(), sizeof(int) * sp_sc.size(),
                                   cudaMemcpyHostToDevice, ctx->stream));
    TGAP_CUDA(ctx, cudaMemcpyAsync(nb->site_struct.ptr, site_struct.data(), sizeof(int) * N,
                                   cudaMemcpyHostToDevice, ctx->stream));
    TGAP_CUDA(ctx, cudaMemcpyAsync(nb->positions.ptr, positions, sizeof(double) * 3 * N,
                                   cudaMemcpyHostToDevice, ctx->stream));
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return TGAP_OK;
}

// Replicate the resident positions into the supercell copy (after an MD update).
__global__ void k_replicate(int n_atoms_total, const int *site_struct, const StructDesc *sd,
                            const double *pos, double *pos_sc)
{
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_atoms_total) return;
    const StructDesc &S = sd[site_struct[g]];
    const int i = g - S.atom_off;
    const int reps = S.rep[0] * S.rep[1] * S.rep[2];
    for (int r = 0; r < reps; ++r) sc_position(S, pos, r * S.n + i + 1, pos_sc + 3 * (size_t)(S.sc_off + r * S.n + i));
}

int neighbors_setup_supercell(tgap_context *ctx, NeighborBatch *nb, int n_sites, int n_sc,
                              const double *positions_sc, const double a[3], const double b[3],
                              const double c[3], int box_small, double rcut,
                              const int *species_sc)
{
    StructDesc S;
    std::memset(&S, 0, sizeof(S));
    int rc = make_struct_desc(a, b, c, box_small, rcut, &S);
    if (rc) return set_error(ctx, rc, "cell smaller than the cutoff on the linked-cell path");
    S.atom_off = 0;
    S.n = n_sites;
    S.sc_off = 0;
    S.n_sc = n_sc;
    S.rep[0] = S.rep[1] = S.rep[2] = 1;
    for (int q = 0; q < 3; ++q) {
        S.pa[q] = S.a[q];
        S.pb[q] = S.b[q];
        S.pc[q] = S.c[q];
    }
    int n_cells = S.cell_off >= 0 ? S.mx * S.my * S.mz : 0;
    nb->n_structures = 1;
    nb->n_atoms = n_sites;
    nb->replicated = false;  // caller-given supercell: pos_sc is the source of truth
    nb->n_sc_total = n_sc;
    nb->n_cells = n_cells;
    nb->host_structs.assign(1, S);
    size_t N = (size_t)n_sites;
    if (nb->d_structs.ensure(sizeof(StructDesc)) ||
        nb->pos_sc.ensure(sizeof(double) * 3 * (size_t)n_sc) ||
        nb->species_sc.ensure(sizeof(int) * (size_t)n_sc) ||
        nb->site_struct.ensure(sizeof(int) * N) || nb->atom_cell.ensure(sizeof(int) * N) ||
        nb->cell_count.ensure(sizeof(int) * (n_cells + 1)) ||
        nb->cell_start.ensure(sizeof(int) * (n_cells + 1)) ||
        nb->cell_cursor.ensure(sizeof(int) * (n_cells + 1)) ||
        nb->cell_atoms.ensure(sizeof(int) * (N + 1)) || nb->cell_tmp.ensure(sizeof(int) * (N + 1)) ||
        nb->counts.ensure(sizeof(int64_t) * (N + 1)) ||
        nb->start.ensure(sizeof(int64_t) * (N + 1)) || nb->n_neigh.ensure(sizeof(int) * N) ||
        nb->positions.ensure(sizeof(double) * 3 * N))
        return set_error(ctx, TGAP_ERR_NOMEM, "neighbor set-up");
    TGAP_CUDA(ctx, cudaMemcpyAsync(nb->d_structs.ptr, &S, sizeof(StructDesc), cudaMemcpyHostToDevice,
                                   ctx->stream));
    TGAP_CUDA(ctx, cudaMemcpyAsync(nb->pos_sc.ptr, positions_sc, sizeof(double) * 3 * (size_t)n_sc,
                                   cudaMemcpyHostToDevice, ctx->stream));
    if (species_sc)
        TGAP_CUDA(ctx, cudaMemcpyAsync(nb->species_sc.ptr, species_sc, sizeof(int) * (size_t)n_sc,
                                       cudaMemcpyHostToDevice, ctx->stream));
    else
        TGAP_CUDA(ctx, cudaMemsetAsync(nb->species_sc.ptr, 0, sizeof(int) * (size_t)n_sc, ctx->stream));
    TGAP_CUDA(ctx, cudaMemsetAsync(nb->site_struct.ptr, 0, sizeof(int) * N, ctx->stream));
    TGAP_CUDA(ctx, cudaMemcpyAsync(nb->positions.ptr, positions_sc, sizeof(double) * 3 * N,
                                   cudaMemcpyHostToDevice, ctx->stream));
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return TGAP_OK;
}

int neighbors_sync_positions(tgap_context *ctx, NeighborBatch *nb)
{
    const int n = nb->n_atoms;
    const int T = 128;
    StageScope sc(ctx, "replicate_positions");
    k_replicate<<<(n + T - 1) / T, T, 0, ctx->stream>>>(n, nb->site_struct.as<int>(),
                                                          nb->d_structs.as<StructDesc>(),
                                                          nb->positions.as<double>(),
                                                          nb->pos_sc.as<double>());
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

}  // namespace tgap
