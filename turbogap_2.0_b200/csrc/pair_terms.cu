// Pairwise GAP terms on the neighbor list (FP64): the distance_2b GAP (gap.f90:329-460) and the
// tabulated core potential with its cubic spline (gap.f90:552-686; splines.f90:33-156).
//
// One warp per site, lanes over the site's pairs (the self slot skipped, as the reference's
// j = 2 .. n_neigh loop does). Each lane sums its pairs' energy, force and virial terms; the warp
// reduces them in a fixed order, writes the site's energy and force (a full neighbor list gives
// each pair to both of its atoms, so the force of a site comes from its own pairs only) and adds
// its virial share with FP64 atomics. Both terms are a few hundred flops per pair: they are
// latency-bound passes over the list, not worth fusing into the SOAP kernels.
#include <cuda_runtime.h>

#include <vector>

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

// Site energy and force, and 1/2 of the pair virial (the reference's final halving), written out.
__device__ __forceinline__ void site_out(int i, int lane, double e, double f[3], double v[6], double e_base,
                                         int do_forces, double *energies, double *forces, double *virial)
{
    e = warp_sum(e);
    if (lane == 0) energies[i] = e_base + e;
    if (!do_forces) return;
    for (int c = 0; c < 3; ++c) f[c] = warp_sum(f[c]);
    for (int c = 0; c < 6; ++c) v[c] = warp_sum(v[c]);
    if (lane == 0) {
        for (int c = 0; c < 3; ++c) forces[3 * (size_t)i + c] = f[c];
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
                          double e0, int do_forces, double *__restrict__ energies, double *__restrict__ forces,
                          double *__restrict__ virial)
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
    site_out(i, lane, e, f, v, e0, do_forces, energies, forces, virial);
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
                                const double *__restrict__ dVdx2, double rcut, int do_forces,
                                double *__restrict__ energies, double *__restrict__ forces,
                                double *__restrict__ virial)
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
    site_out(i, lane, e, f, v, 0.0, do_forces, energies, forces, virial);
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
    DevBuf start, rjs, xyz, species, nsp, a, b, c, d, e, f, out;
    ~PairBufs()
    {
        for (DevBuf *p : {&start, &rjs, &xyz, &species, &nsp, &a, &b, &c, &d, &e, &f, &out}) p->release();
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
            buffer, delta, sigma, e0, do_forces, o, o + n_sites, o + n_sites + 3 * (size_t)n0);
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
            B.c.as<double>(), rcut, do_forces, o, o + n_sites, o + n_sites + 3 * (size_t)n0);
        TGAP_LAUNCH_CHECK(ctx);
    }
    return download_out(ctx, B, n_sites, n0, do_forces, energies, forces, virial);
}
