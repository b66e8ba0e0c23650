// Pair and triplet GAP terms on the neighbor list (FP64): the distance_2b GAP (gap.f90:329-460),
// the tabulated core potential with its cubic spline (gap.f90:552-686; splines.f90:33-156) and the
// angle_3b GAP (gap.f90:756-1015, cov_pp of :1022-1081).
//
// Pair terms: one warp per site, lanes over the site's pairs (the self slot skipped, as the
// reference's j = 2 .. n_neigh loop does). Each lane sums its pairs' energy, force and virial terms;
// the warp reduces them in a fixed order, writes the site's energy and force (a full neighbor list
// gives each pair to both of its atoms, so the force of a site comes from its own pairs only) and
// adds its virial share with FP64 atomics. They are a few hundred flops per pair: latency-bound
// passes over the list. The triplet term (k_triplet_3b) is described at its kernel.
#include <cuda_runtime.h>

#include <vector>

#include "pair_kernels.h"
#include "tgap_internal.h"

namespace tgap {

namespace {

__device__ __forceinline__ bool pair_matches(int si, int sj, int sp1, int sp2)
{
    return (si == sp1 && sj == sp2) || (si == sp2 && sj == sp1);
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// virial[k1 + 3 k2] -= 1/2 (f_k1 r_k2 + f_k2 r_k1) in the 6 independent components
// (xx yy zz xy xz yz)
__device__ __forceinline__ void virial_sym_add(double v[6], const double f[3], const double r[3])
{
    v[0] -= f[0] * r[0];
    v[1] -= f[1] * r[1];
    v[2] -= f[2] * r[2];
    v[3] -= 0.5 * (f[0] * r[1] + f[1] * r[0]);
    v[4] -= 0.5 * (f[0] * r[2] + f[2] * r[0]);
    v[5] -= 0.5 * (f[1] * r[2] + f[2] * r[1]);
}

// Site energy and force, and 1/2 of the pair virial (the reference's final halving), written out
// (add != 0: added to the outputs, the resident evaluation summing several terms).
__device__ __forceinline__ void site_out(int i, int lane, double e, double f[3], double v[6], double e_base,
                                         int do_forces, int add, double *energies, double *forces, double *virial,
                                         const int *site_struct)
{
    e = warp_sum(e);
    if (lane == 0) energies[i] = (add ? energies[i] : 0.0) + e_base + e;
    if (!do_forces) return;
    for (int c = 0; c < 3; ++c) f[c] = warp_sum(f[c]);
    for (int c = 0; c < 6; ++c) v[c] = warp_sum(v[c]);
    if (lane == 0) {
        for (int c = 0; c < 3; ++c) forces[3 * (size_t)i + c] = (add ? forces[3 * (size_t)i + c] : 0.0) + f[c];
        if (site_struct) virial += 9 * (size_t)site_struct[i];  // per structure of a batch
        const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
        for (int c = 0; c < 6; ++c) {
            const double h = 0.5 * v[c];
            atomicAdd(virial + ia[c] + 3 * ib[c], h);
            if (ia[c] != ib[c]) atomicAdd(virial + ib[c] + 3 * ia[c], h);
        }
    }
}

__global__ void k_pair_2b(int n_sites, const int64_t *__restrict__ start, const double *__restrict__ rjs,
                          const double *__restrict__ xyz, const int *__restrict__ species,
                          const int *__restrict__ nsp, int sp1, int sp2, int n_sparse,
                          const double *__restrict__ alphas, const double *__restrict__ cutoff,
                          const double *__restrict__ Qs, double rcut, double buffer, double delta, double sigma,
                          double e0, int do_forces, int add, double *__restrict__ energies,
                          double *__restrict__ forces, double *__restrict__ virial, const int *__restrict__ site_struct)
{
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (i >= n_sites) return;
    const double pi = 3.141592653589793, d2 = delta * delta, is2 = 1.0 / (sigma * sigma);
    double e = 0.0, f[3] = {0.0, 0.0, 0.0}, v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const int si = species[i];
    if (si == sp1 || si == sp2) {
        for (int64_t k = start[i] + 1 + lane; k < start[i + 1]; k += 32) {
            const double r = rjs[k];
            if (!pair_matches(si, nsp[k], sp1, sp2) || !(r < rcut)) continue;
            double fcut = 1.0, dfcut = 0.0;
            if (!(r < rcut - buffer)) {
                const double t = pi * (r - rcut + buffer) / buffer;
                fcut = (cos(t) + 1.0) / 2.0;
                dfcut = pi / 2.0 / buffer * sin(t);
            }
            double h = 0.0;
            for (int s = 0; s < n_sparse; ++s) {
                const double dr = r - Qs[s];
                const double g = d2 * alphas[s] * cutoff[s] * exp(-0.5 * dr * dr * is2);
                e += g * fcut;
                h += g * (dr * is2 * fcut + dfcut);
            }
            if (do_forces) {
                const double rk[3] = {xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2]};
                double fk[3];
                for (int c = 0; c < 3; ++c) fk[c] = -2.0 * h * rk[c] / r;
                for (int c = 0; c < 3; ++c) f[c] += fk[c];
                virial_sym_add(v, fk, rk);
            }
        }
    }
    site_out(i, lane, e, f, v, e0, do_forces, add, energies, forces, virial, site_struct);
}

// Cubic spline of splines.f90 at r (x strictly increasing, n >= 2): value and derivative.
__device__ __forceinline__ void spline_eval(int n, const double *__restrict__ x, const double *__restrict__ y,
                                            const double *__restrict__ y2, double yp1, double ypn, double r,
                                            double *s, double *ds)
{
    if (r < x[0]) {
        *s = y[0] + (r - x[0]) * yp1;
        *ds = yp1;
        return;
    }
    if (r > x[n - 1]) {
        *s = y[n - 1] + (r - x[n - 1]) * ypn;
        *ds = ypn;
        return;
    }
    // the reference's first j with r < x(j + 1), by bisection on the increasing grid
    int lo = 0, hi = n - 2;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (r < x[mid + 1])
            hi = mid;
        else
            lo = mid + 1;
    }
    const int j = lo;
    const double h = x[j + 1] - x[j], h26 = h * h / 6.0, h6 = h / 6.0;
    const double A = (x[j + 1] - r) / h, B = 1.0 - A;
    *s = A * y[j] + B * y[j + 1] + (A * A * A - A) * h26 * y2[j] + (B * B * B - B) * h26 * y2[j + 1];
    *ds = -y[j] / h + y[j + 1] / h + (1.0 - 3.0 * A * A) * h6 * y2[j] + (3.0 * B * B - 1.0) * h6 * y2[j + 1];
}

__global__ void k_pair_core_pot(int n_sites, const int64_t *__restrict__ start, const double *__restrict__ rjs,
                                const double *__restrict__ xyz, const int *__restrict__ species,
                                const int *__restrict__ nsp, int sp1, int sp2, int n, const double *__restrict__ x,
                                const double *__restrict__ V, double yp1, double ypn,
                                const double *__restrict__ dVdx2, double rcut, int do_forces, int add,
                                double *__restrict__ energies, double *__restrict__ forces,
                                double *__restrict__ virial, const int *__restrict__ site_struct)
{
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (i >= n_sites) return;
    double e = 0.0, f[3] = {0.0, 0.0, 0.0}, v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const int si = species[i];
    if (si == sp1 || si == sp2) {
        for (int64_t k = start[i] + 1 + lane; k < start[i + 1]; k += 32) {
            const double r = rjs[k];
            if (!pair_matches(si, nsp[k], sp1, sp2) || !(r < rcut)) continue;
            double s, ds;
            spline_eval(n, x, V, dVdx2, yp1, ypn, r, &s, &ds);
            e += 0.5 * s;
            if (do_forces) {
                const double rk[3] = {xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2]};
                double fk[3];
                for (int c = 0; c < 3; ++c) fk[c] = ds * rk[c] / r;
                for (int c = 0; c < 3; ++c) f[c] += fk[c];
                virial_sym_add(v, fk, rk);
            }
        }
    }
    site_out(i, lane, e, f, v, 0.0, do_forces, add, energies, forces, virial, site_struct);
}

constexpr int k3bMaxPairs = 512;  // eligible pairs of one site held in shared memory
constexpr int k3bWarps = 4;

// cov_pp (d = 3, q = 1) and its derivative with the 1/r factor (gap.f90:1022-1081)
__device__ __forceinline__ double cov_pp31(double r)
{
    if (r >= 1.0) return 0.0;
    if (r <= 0.0) return 1.0;
    const double u = 1.0 - r;
    return u * u * u * u * (4.0 * r + 1.0);
}
__device__ __forceinline__ double cov_pp31_der(double r)
{
    if (r >= 1.0 || r <= 0.0) return 0.0;
    const double u = 1.0 - r;
    return (-4.0 * u * u * u * (4.0 * r + 1.0) + u * u * u * u * 4.0) / r;
}

// One warp per site of species sp0. Its pairs with a neighbor of species sp1 or sp2 inside rcut
// are compacted in list order; lanes then take the triplets (a < b in that order), each summing
// over the sparse points K0 = sum kernel and G_c = sum w dr/dq_c (w = kernel for "exp", -kernel'
// for "pol"), from which the three forces follow in closed form.
__global__ void __launch_bounds__(32 * k3bWarps) k_triplet_3b(
    int n_sites0, int n_sites, const int64_t *__restrict__ start, const double *__restrict__ rjs,
    const double *__restrict__ xyz, const int *__restrict__ nl, const int *__restrict__ species,
    const int *__restrict__ nsp, int sp0, int sp1, int sp2, int n_sparse, const double *__restrict__ pref,
    const double *__restrict__ Qs, double is0, double is1, double is2, double rcut, double buffer, int kernel_pol,
    double e0, int do_forces, int add, const int *__restrict__ jatom, double *__restrict__ energies,
    double *__restrict__ forces, double *__restrict__ virial, const int *__restrict__ site_struct, int *check)
{
    __shared__ int pk[k3bWarps][k3bMaxPairs];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * k3bWarps + w;
    if (i >= n_sites) return;
    const double pi = 3.141592653589793;
    double e = 0.0, v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (species[i] == sp0) {
        const int64_t kb = start[i], ke = start[i + 1];
        // folded atoms: the list's atom map (resident lists) or mod(neighbors_list - 1, n_sites0)
        const int i3 = jatom ? jatom[kb] : (nl[kb] - 1) % n_sites0;
        int n = 0;
        for (int64_t k0 = kb + 1; k0 < ke; k0 += 32) {
            const int64_t k = k0 + lane;
            const bool ok = k < ke && (nsp[k] == sp1 || nsp[k] == sp2) && rjs[k] < rcut;
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            const int slot = n + __popc(m & ((1u << lane) - 1u));
            if (ok) {
                if (slot < k3bMaxPairs)
                    pk[w][slot] = (int)(k - kb);
                else
                    check_fail(check, kCheckListOverrun, k, i);
            }
            n += __popc(m);
        }
        __syncwarp();
        n = min(n, k3bMaxPairs);
        const int T = n * (n - 1) / 2;
        for (int t = lane; t < T; t += 32) {
            int a = 0, rem = t;
            while (rem >= n - 1 - a) {
                rem -= n - 1 - a;
                ++a;
            }
            const int64_t k = kb + pk[w][a], k2 = kb + pk[w][a + 1 + rem];
            const int sj = nsp[k], sk = nsp[k2];
            if (!((sj == sp1 && sk == sp2) || (sj == sp2 && sk == sp1))) continue;
            const double r12 = rjs[k], r13 = rjs[k2];
            const double x12[3] = {xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2]};
            const double x13[3] = {xyz[3 * k2], xyz[3 * k2 + 1], xyz[3 * k2 + 2]};
            double x12r[3], x13r[3], x23[3];
            for (int c = 0; c < 3; ++c) {
                x12r[c] = x12[c] / r12;
                x13r[c] = x13[c] / r13;
                x23[c] = x13[c] - x12[c];
            }
            const double r23 = sqrt(x23[0] * x23[0] + x23[1] * x23[1] + x23[2] * x23[2]);
            double fc12 = 1.0, fc13 = 1.0, dfc12[3] = {0.0, 0.0, 0.0}, dfc13[3] = {0.0, 0.0, 0.0};
            if (!(r12 < rcut - buffer)) {
                const double t12 = pi * (r12 - rcut + buffer) / buffer;
                fc12 = (cos(t12) + 1.0) / 2.0;
                for (int c = 0; c < 3; ++c) dfc12[c] = sin(t12) / 2.0 * pi / buffer * x12r[c];
            }
            if (!(r13 < rcut - buffer)) {
                const double t13 = pi * (r13 - rcut + buffer) / buffer;
                fc13 = (cos(t13) + 1.0) / 2.0;
                for (int c = 0; c < 3; ++c) dfc13[c] = sin(t13) / 2.0 * pi / buffer * x13r[c];
            }
            const double fcut = fc12 * fc13;
            const double q0 = r12 + r13, q1 = (r12 - r13) * (r12 - r13), q2 = r23;
            double K0 = 0.0, G0 = 0.0, G1 = 0.0, G2 = 0.0;
            for (int s = 0; s < n_sparse; ++s) {
                const double d0 = q0 - Qs[s], d1 = q1 - Qs[n_sparse + s], d2 = q2 - Qs[2 * n_sparse + s];
                const double a2 = d0 * d0 * is0 + d1 * d1 * is1 + d2 * d2 * is2;
                double kern, wgt;
                if (kernel_pol) {
                    const double rr = sqrt(a2);
                    kern = pref[s] * cov_pp31(rr);
                    wgt = -pref[s] * cov_pp31_der(rr);
                } else {
                    kern = pref[s] * exp(-0.5 * a2);
                    wgt = kern;
                }
                K0 += kern;
                G0 += wgt * d0 * is0;
                G1 += wgt * d1 * is1;
                G2 += wgt * d2 * is2;
            }
            e += fcut * K0;
            if (!do_forces) continue;
            const int j3 = jatom ? jatom[k] : (nl[k] - 1) % n_sites0;
            const int k3 = jatom ? jatom[k2] : (nl[k2] - 1) % n_sites0;
            double f1[3], f2[3], f3[3];
            const double x23r[3] = {x23[0] / r23, x23[1] / r23, x23[2] / r23};
            for (int l = 0; l < 3; ++l) {
                const double dfc = fc12 * dfc13[l] + fc13 * dfc12[l];
                const double s1 = G0 * (x12r[l] + x13r[l]) + G1 * 2.0 * (r12 - r13) * (x12r[l] - x13r[l]);
                const double s2 = -G0 * x12r[l] - G1 * 2.0 * (r12 - r13) * x12r[l] + G2 * x23r[l];
                const double s3 = -G0 * x13r[l] - G1 * 2.0 * (r13 - r12) * x13r[l] - G2 * x23r[l];
                f1[l] = -(K0 * dfc + fcut * s1);
                f2[l] = -(-K0 * fc13 * dfc12[l] + fcut * s2);
                f3[l] = -(-K0 * fc12 * dfc13[l] + fcut * s3);
            }
            for (int c = 0; c < 3; ++c) {
                atomicAdd(forces + 3 * (size_t)i3 + c, f1[c]);
                atomicAdd(forces + 3 * (size_t)j3 + c, f2[c]);
                atomicAdd(forces + 3 * (size_t)k3 + c, f3[c]);
            }
            v[0] += f2[0] * x12[0] + f3[0] * x13[0];
            v[1] += f2[1] * x12[1] + f3[1] * x13[1];
            v[2] += f2[2] * x12[2] + f3[2] * x13[2];
            v[3] += 0.5 * (f2[0] * x12[1] + f2[1] * x12[0] + f3[0] * x13[1] + f3[1] * x13[0]);
            v[4] += 0.5 * (f2[0] * x12[2] + f2[2] * x12[0] + f3[0] * x13[2] + f3[2] * x13[0]);
            v[5] += 0.5 * (f2[1] * x12[2] + f2[2] * x12[1] + f3[1] * x13[2] + f3[2] * x13[1]);
        }
    }
    e = warp_sum(e);
    if (lane == 0) energies[i] = (add ? energies[i] : 0.0) + e0 + e;
    if (!do_forces) return;
    for (int c = 0; c < 6; ++c) v[c] = warp_sum(v[c]);
    if (lane == 0) {
        if (site_struct) virial += 9 * (size_t)site_struct[i];
        const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
        for (int c = 0; c < 6; ++c) {
            atomicAdd(virial + ia[c] + 3 * ib[c], v[c]);
            if (ia[c] != ib[c]) atomicAdd(virial + ib[c] + 3 * ia[c], v[c]);
        }
    }
}

int up(tgap_context *ctx, DevBuf &b, const void *h, size_t bytes)
{
    if (b.ensure(bytes ? bytes : 8)) return set_error(ctx, TGAP_ERR_NOMEM, "pair-term buffers");
    if (bytes) TGAP_CUDA(ctx, cudaMemcpyAsync(b.ptr, h, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return TGAP_OK;
}

#define PRC(x)                \
    do {                      \
        int _rc = (x);        \
        if (_rc) return _rc;  \
    } while (0)

struct PairBufs {
    DevBuf start, rjs, xyz, species, nsp, nl, a, b, c, out;
    ~PairBufs()
    {
        for (DevBuf *p : {&start, &rjs, &xyz, &species, &nsp, &nl, &a, &b, &c, &out}) p->release();
    }
};

// Uploads the list arrays shared by both terms; out gets room for energies, forces and virial.
int upload_list(tgap_context *ctx, PairBufs &B, int n_sites, int n_atom_pairs, const int *n_neigh,
                const double *rjs, const double *xyz, const int *species, const int *nsp, int n_sites0)
{
    std::vector<int64_t> st((size_t)n_sites + 1, 0);
    for (int i = 0; i < n_sites; ++i) st[i + 1] = st[i] + n_neigh[i];
    if (st[n_sites] != n_atom_pairs) return set_error(ctx, TGAP_ERR_ARGUMENT, "sum(n_neigh) != n_atom_pairs");
    PRC(up(ctx, B.start, st.data(), sizeof(int64_t) * st.size()));
    PRC(up(ctx, B.rjs, rjs, sizeof(double) * (size_t)n_atom_pairs));
    PRC(up(ctx, B.xyz, xyz, sizeof(double) * 3 * (size_t)n_atom_pairs));
    PRC(up(ctx, B.species, species, sizeof(int) * (size_t)n_sites));
    PRC(up(ctx, B.nsp, nsp, sizeof(int) * (size_t)n_atom_pairs));
    if (B.out.ensure(sizeof(double) * ((size_t)n_sites + 3 * (size_t)n_sites0 + 9)))
        return set_error(ctx, TGAP_ERR_NOMEM, "pair-term outputs");
    TGAP_CUDA(ctx, cudaMemsetAsync(B.out.ptr, 0, B.out.bytes, ctx->stream));
    return TGAP_OK;
}

int download_out(tgap_context *ctx, PairBufs &B, int n_sites, int n_sites0, int do_forces, double *energies,
                 double *forces, double *virial)
{
    const double *o = B.out.as<double>();
    TGAP_CUDA(ctx, cudaMemcpyAsync(energies, o, sizeof(double) * n_sites, cudaMemcpyDeviceToHost, ctx->stream));
    if (do_forces) {
        TGAP_CUDA(ctx, cudaMemcpyAsync(forces, o + n_sites, sizeof(double) * 3 * (size_t)n_sites0,
                                       cudaMemcpyDeviceToHost, ctx->stream));
        TGAP_CUDA(ctx, cudaMemcpyAsync(virial, o + n_sites + 3 * (size_t)n_sites0, sizeof(double) * 9,
                                       cudaMemcpyDeviceToHost, ctx->stream));
    }
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return read_device_check(ctx);
}

}  // namespace

int terms_compute(tgap_context *ctx, const TermSet &t, int n_sites, const int64_t *d_start, const double *d_rjs,
                  const double *d_xyz, const int *d_site_species, const int *d_nsp, const int *d_jatom,
                  const int *d_site_struct, int do_forces, double *d_energies, double *d_forces, double *d_virial)
{
    if (n_sites <= 0) return TGAP_OK;
    const int grid = (n_sites + 3) / 4;
    for (const Term2b &b : t.t2b) {
        StageScope sc(ctx, "pair_2b_f64");
        k_pair_2b<<<grid, 128, 0, ctx->stream>>>(n_sites, d_start, d_rjs, d_xyz, d_site_species, d_nsp, b.sp1, b.sp2,
                                                 b.n_sparse, b.alphas.as<double>(), b.cutoff.as<double>(),
                                                 b.Qs.as<double>(), b.rcut, b.buffer, b.delta, b.sigma, b.e0,
                                                 do_forces, 1, d_energies, d_forces, d_virial, d_site_struct);
        TGAP_LAUNCH_CHECK(ctx);
    }
    for (const TermCore &c : t.core) {
        StageScope sc(ctx, "pair_core_pot_f64");
        k_pair_core_pot<<<grid, 128, 0, ctx->stream>>>(n_sites, d_start, d_rjs, d_xyz, d_site_species, d_nsp, c.sp1,
                                                       c.sp2, c.n, c.x.as<double>(), c.V.as<double>(), c.yp1, c.ypn,
                                                       c.y2.as<double>(), c.rcut, do_forces, 1, d_energies, d_forces,
                                                       d_virial, d_site_struct);
        TGAP_LAUNCH_CHECK(ctx);
    }
    for (const Term3b &b : t.t3b) {
        StageScope sc(ctx, "triplet_3b_f64");
        k_triplet_3b<<<(n_sites + k3bWarps - 1) / k3bWarps, 32 * k3bWarps, 0, ctx->stream>>>(
            1, n_sites, d_start, d_rjs, d_xyz, nullptr, d_site_species, d_nsp, b.sp0, b.sp1, b.sp2, b.n_sparse,
            b.pref.as<double>(), b.Qs.as<double>(), b.is[0], b.is[1], b.is[2], b.rcut, b.buffer, b.kernel, b.e0,
            do_forces, 1, d_jatom, d_energies, d_forces, d_virial, d_site_struct, ctx->d_check);
        TGAP_LAUNCH_CHECK(ctx);
    }
    return TGAP_OK;
}

}  // namespace tgap

using namespace tgap;

extern "C" int tgap_get_2b_energy_and_forces(tgap_context *ctx, int n_sites, int n_atom_pairs, const double *rjs,
                                             const double *xyz, int n_sparse, const double *alphas,
                                             const double *cutoff, double rcut, double buffer, double delta,
                                             double sigma, double e0, const double *Qs, const int *n_neigh,
                                             int do_forces, const int *species, const int *neighbor_species,
                                             int species1, int species2, int n_sites0, double *energies,
                                             double *forces, double *virial)
{
    if (!ctx) return TGAP_ERR_ARGUMENT;
    if (n_sites < 0 || n_atom_pairs < 0 || n_sparse < 1 || !rjs || !xyz || !alphas || !cutoff || !Qs || !n_neigh ||
        !species || !neighbor_species || !energies || !(sigma > 0.0) || !(buffer > 0.0) ||
        (do_forces && (!forces || !virial || n_sites0 < n_sites)))
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_get_2b_energy_and_forces: bad arguments");
    TGAP_CUDA(ctx, cudaSetDevice(ctx->device));
    if (n_sites == 0) return TGAP_OK;
    const int n0 = do_forces ? n_sites0 : 0;
    PairBufs B;
    PRC(upload_list(ctx, B, n_sites, n_atom_pairs, n_neigh, rjs, xyz, species, neighbor_species, n0));
    PRC(up(ctx, B.a, alphas, sizeof(double) * n_sparse));
    PRC(up(ctx, B.b, cutoff, sizeof(double) * n_sparse));
    PRC(up(ctx, B.c, Qs, sizeof(double) * n_sparse));
    double *o = B.out.as<double>();
    {
        StageScope sc(ctx, "pair_2b_f64");
        k_pair_2b<<<(n_sites + 3) / 4, 128, 0, ctx->stream>>>(
            n_sites, B.start.as<int64_t>(), B.rjs.as<double>(), B.xyz.as<double>(), B.species.as<int>(),
            B.nsp.as<int>(), species1, species2, n_sparse, B.a.as<double>(), B.b.as<double>(), B.c.as<double>(), rcut,
            buffer, delta, sigma, e0, do_forces, 0, o, o + n_sites, o + n_sites + 3 * (size_t)n0, nullptr);
        TGAP_LAUNCH_CHECK(ctx);
    }
    return download_out(ctx, B, n_sites, n0, do_forces, energies, forces, virial);
}

extern "C" int tgap_get_core_pot_energy_and_forces(tgap_context *ctx, int n_sparse, int n_sites, int n_atom_pairs,
                                                   int n_sites0, const double *rjs, const double *xyz,
                                                   const double *x, const double *V, double yp1, double ypn,
                                                   const double *dVdx2, const int *n_neigh, int do_forces,
                                                   const int *species, const int *neighbor_species, int species1,
                                                   int species2, double *energies, double *forces, double *virial)
{
    if (!ctx) return TGAP_ERR_ARGUMENT;
    if (n_sparse < 2 || n_sites < 0 || n_atom_pairs < 0 || !rjs || !xyz || !x || !V || !dVdx2 || !n_neigh ||
        !species || !neighbor_species || !energies || (do_forces && (!forces || !virial || n_sites0 < n_sites)))
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_get_core_pot_energy_and_forces: bad arguments");
    double rcut = x[0];
    for (int s = 1; s < n_sparse; ++s) {
        // splines.f90 stops on h = 0: the table must increase
        if (!(x[s] > x[s - 1]))
            return set_error(ctx, TGAP_ERR_ARGUMENT, "core_pot table: x must increase (x[%d] <= x[%d])", s, s - 1);
        rcut = x[s] > rcut ? x[s] : rcut;
    }
    TGAP_CUDA(ctx, cudaSetDevice(ctx->device));
    if (n_sites == 0) return TGAP_OK;
    const int n0 = do_forces ? n_sites0 : 0;
    PairBufs B;
    PRC(upload_list(ctx, B, n_sites, n_atom_pairs, n_neigh, rjs, xyz, species, neighbor_species, n0));
    PRC(up(ctx, B.a, x, sizeof(double) * n_sparse));
    PRC(up(ctx, B.b, V, sizeof(double) * n_sparse));
    PRC(up(ctx, B.c, dVdx2, sizeof(double) * n_sparse));
    double *o = B.out.as<double>();
    {
        StageScope sc(ctx, "pair_core_pot_f64");
        k_pair_core_pot<<<(n_sites + 3) / 4, 128, 0, ctx->stream>>>(
            n_sites, B.start.as<int64_t>(), B.rjs.as<double>(), B.xyz.as<double>(), B.species.as<int>(),
            B.nsp.as<int>(), species1, species2, n_sparse, B.a.as<double>(), B.b.as<double>(), yp1, ypn,
            B.c.as<double>(), rcut, do_forces, 0, o, o + n_sites, o + n_sites + 3 * (size_t)n0, nullptr);
        TGAP_LAUNCH_CHECK(ctx);
    }
    return download_out(ctx, B, n_sites, n0, do_forces, energies, forces, virial);
}

extern "C" int tgap_get_3b_energy_and_forces(tgap_context *ctx, int n_sites0, int n_sites, int n_atom_pairs,
                                             const double *rjs, const double *xyz, int n_sparse,
                                             const double *alphas, const double *cutoff, double rcut, double buffer,
                                             double delta, const double *sigma, double e0, const double *Qs,
                                             const int *n_neigh, const int *neighbors_list, int do_forces,
                                             int kernel_type, const int *species, const int *neighbor_species,
                                             int species_center, int species1, int species2, double *energies,
                                             double *forces, double *virial)
{
    if (!ctx) return TGAP_ERR_ARGUMENT;
    if (n_sites < 0 || n_atom_pairs < 0 || n_sparse < 1 || n_sites0 < 1 || !rjs || !xyz || !alphas || !cutoff ||
        !sigma || !Qs || !n_neigh || !neighbors_list || !species || !neighbor_species || !energies ||
        !(sigma[0] > 0.0 && sigma[1] > 0.0 && sigma[2] > 0.0) || !(buffer > 0.0) ||
        (kernel_type != 0 && kernel_type != 1) || (do_forces && (!forces || !virial)))
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_get_3b_energy_and_forces: bad arguments");
    TGAP_CUDA(ctx, cudaSetDevice(ctx->device));
    if (n_sites == 0) return TGAP_OK;
    const int n0 = do_forces ? n_sites0 : 0;
    PairBufs B;
    PRC(upload_list(ctx, B, n_sites, n_atom_pairs, n_neigh, rjs, xyz, species, neighbor_species, n0));
    PRC(up(ctx, B.nl, neighbors_list, sizeof(int) * (size_t)n_atom_pairs));
    std::vector<double> pref(n_sparse);
    for (int s = 0; s < n_sparse; ++s) pref[s] = 2.0 * delta * delta * alphas[s] * cutoff[s];  // gap.f90:829
    PRC(up(ctx, B.a, pref.data(), sizeof(double) * n_sparse));
    PRC(up(ctx, B.b, Qs, sizeof(double) * 3 * (size_t)n_sparse));
    double *o = B.out.as<double>();
    {
        StageScope sc(ctx, "triplet_3b_f64");
        k_triplet_3b<<<(n_sites + k3bWarps - 1) / k3bWarps, 32 * k3bWarps, 0, ctx->stream>>>(
            n_sites0, n_sites, B.start.as<int64_t>(), B.rjs.as<double>(), B.xyz.as<double>(), B.nl.as<int>(),
            B.species.as<int>(), B.nsp.as<int>(), species_center, species1, species2, n_sparse, B.a.as<double>(),
            B.b.as<double>(), 1.0 / (sigma[0] * sigma[0]), 1.0 / (sigma[1] * sigma[1]), 1.0 / (sigma[2] * sigma[2]),
            rcut, buffer, kernel_type, e0, do_forces, 0, nullptr, o, o + n_sites, o + n_sites + 3 * (size_t)n0,
            nullptr, ctx->d_check);
        TGAP_LAUNCH_CHECK(ctx);
    }
    return download_out(ctx, B, n_sites, n0, do_forces, energies, forces, virial);
}
