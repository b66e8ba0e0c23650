// SOAP poly3 descriptor kernels (sm_100a): forward expansion + power spectrum, adjoint
// back-scatter of dE/dq to forces and virial, and the materialised dq/dr of the reference
// get_soap surface (soap_cart_der, call site src/gap/gap_interface.f90:301-306).
//
// Forward and adjoint (soap_warp.cuh): one warp owns one central site, one lane one pair, with
// l_max a template parameter (0..10). The expansion c_{n,lm} = sum_j R_n(r_j) A_lm(r_j) is a
// small (n_max x 32) x (32 x nlm) product out of the warp's shared memory per group of 32
// pairs. The materialised dq/dr keeps one CTA of 256 threads per site, four lanes per pair
// splitting the quadrature nodes and harmonic orders. The templates run in FP64 (plain path)
// or FP32 (mixed path); positions, pair vectors, forces and the virial stay FP64.
#include <cuda_bf16.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <type_traits>

#include "soap_device.cuh"
#include "soap_kernels.h"

namespace tgap {

__constant__ YlmConst c_ylm;

constexpr int kThreads = 256;
constexpr int kPairsPerChunk = kThreads / kLanesPerPair;

int upload_ylm_constants()
{
    const YlmConst &h = ylm_host_constants();
    return cudaMemcpyToSymbol(c_ylm, &h, sizeof(h)) == cudaSuccess ? 0 : 1;
}

// Harmonics of the orders m = sub (mod 4): calls fn(k, l, Y, gx, gy, gz) for every real
// harmonic index k = l^2 + {0 | 2m-1 | 2m} with (gx, gy, gz) = dY/du (components of u taken
// independent; project onto the tangent plane for the gradient with respect to r).
template <class T, bool GRAD, class F>
__device__ __forceinline__ void ylm_lane(int L, T ux, T uy, T uz, int sub, F &&fn)
{
    T Cc = 1, Sc = 0, Cp = 0, Sp = 0;
#pragma unroll
    for (int m = 0; m <= kMaxL; ++m) {
        if (m > 0) {
            Cp = Cc;
            Sp = Sc;
            T cn = ux * Cc - uy * Sc;
            T sn = ux * Sc + uy * Cc;
            Cc = cn;
            Sc = sn;
        }
        if (m > L) break;
        if ((m & 3) != sub) continue;
        T Q2 = 0, Q1 = 0, dQ2 = 0, dQ1 = 0;
        const T qmm = (T)c_ylm.dfact[m];
        for (int l = m; l <= L; ++l) {
            T Q, dQ;
            if (l == m) {
                Q = qmm;
                dQ = 0;
            } else if (l == m + 1) {
                Q = (T)(2 * m + 1) * uz * qmm;
                dQ = (T)(2 * m + 1) * qmm;
            } else {
                const T inv = (T)1 / (T)(l - m);
                Q = ((T)(2 * l - 1) * uz * Q1 - (T)(l + m - 1) * Q2) * inv;
                dQ = ((T)(2 * l - 1) * (Q1 + uz * dQ1) - (T)(l + m - 1) * dQ2) * inv;
            }
            Q2 = Q1;
            Q1 = Q;
            dQ2 = dQ1;
            dQ1 = dQ;
            const T N = (T)c_ylm.norm[l * (l + 1) / 2 + m];
            const int base = l * l;
            if (m == 0) {
                fn(base, l, N * Q, (T)0, (T)0, GRAD ? N * dQ : (T)0);
            } else {
                const T NQ = N * Q;
                const T mm = (T)m;
                if (GRAD) {
                    fn(base + 2 * m - 1, l, NQ * Cc, NQ * mm * Cp, -NQ * mm * Sp, N * dQ * Cc);
                    fn(base + 2 * m, l, NQ * Sc, NQ * mm * Sp, NQ * mm * Cp, N * dQ * Sc);
                } else {
                    fn(base + 2 * m - 1, l, NQ * Cc, (T)0, (T)0, (T)0);
                    fn(base + 2 * m, l, NQ * Sc, (T)0, (T)0, (T)0);
                }
            }
        }
    }
}

// Pair classification shared by the kernels.
template <class T>
__device__ __forceinline__ bool pair_setup(const SoapParams &P, int64_t k, int64_t kb, int64_t ke,
                                           const double *__restrict__ rjs,
                                           const double *__restrict__ xyz,
                                           const int *__restrict__ nsp, int *s_out, T *r_out,
                                           T u[3], T rv[3])
{
    bool valid = (k < ke) && (k != kb);
    int s = 0;
    T r = 1;
    if (valid) {
        s = nsp[k] - 1;
        if (s < 0 || s >= P.n_species) valid = false;
    }
    if (valid) {
        const double rd = rjs[k];
        if (!(rd < P.rcut_hard[s]) || !(rd > 0.0)) valid = false;
        r = (T)rd;
        rv[0] = (T)xyz[3 * k];
        rv[1] = (T)xyz[3 * k + 1];
        rv[2] = (T)xyz[3 * k + 2];
        const T ir = (T)1 / r;
        u[0] = rv[0] * ir;
        u[1] = rv[1] * ir;
        u[2] = rv[2] * ir;
    }
    if (!valid) {
        s = 0;
        r = 1;
        u[0] = 0;
        u[1] = 0;
        u[2] = 1;
        rv[0] = rv[1] = rv[2] = 0;
    }
    *s_out = s;
    *r_out = r;
    return valid;
}

template <class T>
__device__ __forceinline__ T block_sum(T v, T *red)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    T t = 0;
    if (threadIdx.x < 32) {
        t = threadIdx.x < (kThreads / 32) ? red[threadIdx.x] : (T)0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) red[0] = t;
    }
    __syncthreads();
    t = red[0];
    __syncthreads();
    return t;
}

// Decode power-spectrum index d -> (n, n', l) with n <= n'.
__device__ __forceinline__ void ps_decode(int d, int nmax, int L, int *n, int *np, int *l)
{
    int pidx = d / (L + 1);
    *l = d - pidx * (L + 1);
    int a = 0;
    while (pidx >= nmax - a) {
        pidx -= nmax - a;
        ++a;
    }
    *n = a;
    *np = a + pidx;
}

__device__ __forceinline__ int ps_index(int n, int np, int nmax, int L, int l)
{
    if (n > np) {
        int t = n;
        n = np;
        np = t;
    }
    return (n * nmax - n * (n - 1) / 2 + (np - n)) * (L + 1) + l;
}

// ----------------------------------------------------------------------------- dq/dr

// Reference layout: der[(pair * dim + d) * 3 + x]; self slot = -sum of the site's others.
__global__ void __launch_bounds__(kThreads) k_soap_cart_der(
    SoapParams P, const double *__restrict__ xq, const double *__restrict__ tq,
    const int *__restrict__ sites, int n_rows, const int64_t *__restrict__ start,
    const double *__restrict__ rjs, const double *__restrict__ xyz, const int *__restrict__ nsp,
    const double *__restrict__ c_in, const double *__restrict__ q_in, int q_ld,
    const double *__restrict__ norm_in, double *__restrict__ der)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *smem = reinterpret_cast<double *>(smem_raw);
    const int nmax = P.n_max, L = P.l_max, nlm = (L + 1) * (L + 1), dim = P.dim;
    double *cs = smem;                 // [nmax][nlm]
    double *Ap = cs + nmax * nlm;      // [nlm]
    double *dAp = Ap + nlm;            // [nlm][3]
    double *Rp = dAp + 3 * nlm;        // [kMaxAlpha]
    double *dRp = Rp + kMaxAlpha;      // [kMaxAlpha]
    double *red = dRp + kMaxAlpha;     // [32]
    double *misc = red + 32;           // [8]

    const int row = blockIdx.x;
    if (row >= n_rows) return;
    const int site = sites ? sites[row] : row;
    const int64_t kb = start[site], ke = start[site + 1];
    const int t = threadIdx.x;
    const int nout = nmax * nlm;
    for (int o = t; o < nout; o += kThreads) cs[o] = c_in[(size_t)row * nout + o];
    const double nrm = norm_in[row];
    const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
    constexpr int kSlots = (kMaxNmax * (kMaxNmax + 1) / 2 * (kMaxL + 1) + kThreads - 1) / kThreads;
    double self_acc[kSlots][3];
#pragma unroll
    for (int j = 0; j < kSlots; ++j) self_acc[j][0] = self_acc[j][1] = self_acc[j][2] = 0.0;
    __syncthreads();

    for (int64_t k = kb + 1; k < ke; ++k) {
        int s;
        double r, u[3], rv[3];
        const bool valid = pair_setup<double>(P, k, kb, ke, rjs, xyz, nsp, &s, &r, u, rv);
        double *out = der + (size_t)k * dim * 3;
        if (!valid || nrm == 0.0) {
            for (int i = t; i < dim * 3; i += kThreads) out[i] = 0.0;
            continue;
        }
        if (t < 32) {
            const int sub = t & 3;
            const double rc = P.rcut_hard[s];
            const double x = r / rc;
            const double sig = (P.sigma_r[s] + P.sigma_r_scaling[s] * r) / rc;
            const double dsig = P.sigma_r_scaling[s];
            double sum[kMaxAlpha], dsum[kMaxAlpha];
            radial_node_sums<double, true>(P, s, true, xq, tq, x, sig, dsig, sub, sum, dsum);
            if (t < 4) {
                double A, dA;
                radial_amplitude<double>(P, s, x, sig, dsig, &A, &dA);
                const double gs = P.global_scaling[s];
                if (t == 0) {
#pragma unroll
                    for (int n = 0; n < kMaxAlpha; ++n) {
                        Rp[n] = gs * A * sum[n];
                        dRp[n] = gs * (dA * sum[n] + A * dsum[n]) / rc;
                    }
                }
                const double st = P.sigma_t[s] + P.sigma_t_scaling[s] * r;
                const double kap = r * r / (st * st);
                const double dkap = 2.0 * r / (st * st) - 2.0 * r * r * P.sigma_t_scaling[s] / (st * st * st);
                double f[kMaxL + 2];
                bessel_ratios<double>(L, kap, f);
                const double ir = 1.0 / r;
                ylm_lane<double, true>(L, u[0], u[1], u[2], sub,
                                       [&](int kk, int l, double Y, double gx, double gy, double gz) {
                    const double fl = f[l];
                    const double dfl = (f[l + 1] + (double)l / kap * fl - fl * f[1]) * dkap;
                    const double ug = u[0] * gx + u[1] * gy + u[2] * gz;
                    Ap[kk] = fl * Y;
                    dAp[3 * kk] = dfl * u[0] * Y + fl * (gx - u[0] * ug) * ir;
                    dAp[3 * kk + 1] = dfl * u[1] * Y + fl * (gy - u[1] * ug) * ir;
                    dAp[3 * kk + 2] = dfl * u[2] * Y + fl * (gz - u[2] * ug) * ir;
                });
            }
        }
        __syncthreads();
        const int off = P.n_off[s], am = P.alpha_max[s];
        double dp[kSlots][3];
        double qd0 = 0, qd1 = 0, qd2 = 0;
#pragma unroll
        for (int j = 0; j < kSlots; ++j) {
            dp[j][0] = dp[j][1] = dp[j][2] = 0.0;
            const int d = t + j * kThreads;
            if (d < dim) {
                int n, np, l;
                ps_decode(d, nmax, L, &n, &np, &l);
                const bool in_n = n >= off && n < off + am, in_np = np >= off && np < off + am;
                double a0 = 0, a1 = 0, a2 = 0;
                for (int kk = l * l; kk < (l + 1) * (l + 1); ++kk) {
                    if (in_n) {
                        const double cn = cs[np * nlm + kk];
                        const double R = Rp[n - off], dR = dRp[n - off];
                        a0 += (dR * u[0] * Ap[kk] + R * dAp[3 * kk]) * cn;
                        a1 += (dR * u[1] * Ap[kk] + R * dAp[3 * kk + 1]) * cn;
                        a2 += (dR * u[2] * Ap[kk] + R * dAp[3 * kk + 2]) * cn;
                    }
                    if (in_np) {
                        const double cn = cs[n * nlm + kk];
                        const double R = Rp[np - off], dR = dRp[np - off];
                        a0 += (dR * u[0] * Ap[kk] + R * dAp[3 * kk]) * cn;
                        a1 += (dR * u[1] * Ap[kk] + R * dAp[3 * kk + 1]) * cn;
                        a2 += (dR * u[2] * Ap[kk] + R * dAp[3 * kk + 2]) * cn;
                    }
                }
                const double mult = (n == np) ? 1.0 : 1.4142135623730951;
                dp[j][0] = mult * a0;
                dp[j][1] = mult * a1;
                dp[j][2] = mult * a2;
                const double qv = q_in[(size_t)row * q_ld + d];
                qd0 += qv * dp[j][0];
                qd1 += qv * dp[j][1];
                qd2 += qv * dp[j][2];
            }
        }
        qd0 = block_sum<double>(qd0, red);
        qd1 = block_sum<double>(qd1, red);
        qd2 = block_sum<double>(qd2, red);
#pragma unroll
        for (int j = 0; j < kSlots; ++j) {
            const int d = t + j * kThreads;
            if (d < dim) {
                const double qv = q_in[(size_t)row * q_ld + d];
                const double v0 = (dp[j][0] - qv * qd0) * inv;
                const double v1 = (dp[j][1] - qv * qd1) * inv;
                const double v2 = (dp[j][2] - qv * qd2) * inv;
                out[3 * d] = v0;
                out[3 * d + 1] = v1;
                out[3 * d + 2] = v2;
                self_acc[j][0] -= v0;
                self_acc[j][1] -= v1;
                self_acc[j][2] -= v2;
            }
        }
        __syncthreads();
    }
    (void)misc;
    double *out = der + (size_t)kb * dim * 3;
#pragma unroll
    for (int j = 0; j < kSlots; ++j) {
        const int d = t + j * kThreads;
        if (d < dim) {
            out[3 * d] = self_acc[j][0];
            out[3 * d + 1] = self_acc[j][1];
            out[3 * d + 2] = self_acc[j][2];
        }
    }
}

// ----------------------------------------------------------------------------- host

static size_t der_smem(const SoapParams &P)
{
    const int nlm = (P.l_max + 1) * (P.l_max + 1);
    return sizeof(double) * ((size_t)P.n_max * nlm + 4 * (size_t)nlm + 2 * kMaxAlpha + 40);
}

const YlmConst &ylm_host_constants()
{
    static const YlmConst h = [] {
        YlmConst y;
        double df = 1.0;
        for (int m = 0; m <= kMaxL; ++m) {
            if (m > 0) df *= (2.0 * m - 1.0);
            y.dfact[m] = df;
            y.inv_int[m] = m > 0 ? 1.0 / m : 0.0;
        }
        for (int l = 0; l <= kMaxL; ++l) {
            double fr = 1.0;
            for (int m = 0; m <= l; ++m) {
                if (m > 0) fr /= (double)(l + m) * (double)(l - m + 1);
                const double N = std::sqrt((2.0 * l + 1.0) / (4.0 * M_PI) * fr);
                y.norm[l * (l + 1) / 2 + m] = m == 0 ? N : N * M_SQRT2;
            }
        }
        for (int m = 0; m <= kMaxL; ++m) {
            y.qb0[m] = y.norm[m * (m + 1) / 2 + m] * y.dfact[m];
            for (int l = m + 1; l <= kMaxL + 1; ++l) {
                const double dl = l, dm = m;
                const int i = rec_off(m) + l - m - 1;
                y.ra[i] = std::sqrt((4.0 * dl * dl - 1.0) / (dl * dl - dm * dm));
                y.rb[i] = l == m + 1 ? 0.0
                                     : std::sqrt((2.0 * dl + 1.0) * (dl + dm - 1.0) * (dl - dm - 1.0) /
                                                 ((2.0 * dl - 3.0) * (dl + dm) * (dl - dm)));
            }
        }
        for (int i = 0; i <= kMaxL; ++i) {
            y.dfact_f[i] = (float)y.dfact[i];
            y.inv_int_f[i] = (float)y.inv_int[i];
            y.qb0_f[i] = (float)y.qb0[i];
        }
        for (int i = 0; i < (kMaxL + 1) * (kMaxL + 2) / 2; ++i) y.norm_f[i] = (float)y.norm[i];
        for (int i = 0; i < kRecN; ++i) {
            y.ra_f[i] = (float)y.ra[i];
            y.rb_f[i] = (float)y.rb[i];
        }
        return y;
    }();
    return h;
}

int soap_forward(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites,
                 int n_rows, int precision, SoapOut &o)
{
    if (n_rows <= 0) return TGAP_OK;
    StageScope sc(ctx, precision == TGAP_FP64 ? "soap_forward_f64" : "soap_forward_f32");
    const bool cmp = ds.p.cmp_row != nullptr;
    if (precision == TGAP_FP64)
        return (cmp ? soap_fwd_f64_cmp : soap_fwd_f64)(ctx, ds, pv, d_sites, n_rows, o);
    return (cmp ? soap_fwd_f32_cmp : soap_fwd_f32)(ctx, ds, pv, d_sites, n_rows, o);
}

int soap_backward(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites,
                  int n_rows, int precision, const SoapOut &o, const void *d_g, int g_ld,
                  int g_is_double, const int *site_struct, double *d_forces, double *d_virial)
{
    if (n_rows <= 0) return TGAP_OK;
    StageScope sc(ctx, precision == TGAP_FP64 ? "soap_backward_f64" : "soap_backward_f32");
    const bool cmp = ds.p.cmp_row != nullptr;
    if (precision == TGAP_FP64)
        return (cmp ? soap_bwd_f64_cmp : soap_bwd_f64)(ctx, ds, pv, d_sites, n_rows, o, d_g, g_ld, site_struct,
                                                       d_forces, d_virial);
    return (cmp ? soap_bwd_f32_cmp : soap_bwd_f32)(ctx, ds, pv, d_sites, n_rows, o, d_g, g_ld, g_is_double,
                                                   site_struct, d_forces, d_virial);
}

// Cubic Hermite coefficients of R_n on interval i of species s from FP64 quadrature values and
// derivatives at both ends: R(t) = a + b t + c t^2 + d t^3, t in [0, 1], h = rcut_hard / kTabIntervals.
__global__ void k_radial_table(const __grid_constant__ SoapParams P, const double *__restrict__ xq,
                               const double *__restrict__ tq, float4 *__restrict__ tab)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= P.n_species * kTabIntervals) return;
    const int s = g / kTabIntervals, i = g - s * kTabIntervals;
    const double h = P.rcut_hard[s] / kTabIntervals;
    double R0[kMaxAlpha], dR0[kMaxAlpha], R1[kMaxAlpha], dR1[kMaxAlpha];
    radial_quad<double, kMaxAlpha, true>(P, s, i * h, xq, tq, R0, dR0);
    radial_quad<double, kMaxAlpha, true>(P, s, (i + 1) * h, xq, tq, R1, dR1);
    float4 *e = tab + (size_t)g * P.am_pad;
    for (int n = 0; n < P.am_pad; ++n) {
        float4 c = make_float4(0.f, 0.f, 0.f, 0.f);
        if (n < P.alpha_max[s]) {
            const double a = R0[n], b = h * dR0[n];
            const double cc = 3.0 * (R1[n] - R0[n]) - h * (2.0 * dR0[n] + dR1[n]);
            const double d = 2.0 * (R0[n] - R1[n]) + h * (dR0[n] + dR1[n]);
            c = make_float4((float)a, (float)b, (float)cc, (float)d);
        }
        e[n] = c;
    }
}

int soap_cart_der(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites,
                  int n_rows, const SoapOut &o, double *d_der)
{
    if (n_rows <= 0) return TGAP_OK;
    StageScope sc(ctx, "soap_cart_der_f64");
    const size_t sm = der_smem(ds.p);
    TGAP_CUDA(ctx, cudaFuncSetAttribute(k_soap_cart_der, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_soap_cart_der<<<n_rows, kThreads, sm, ctx->stream>>>(
        ds.p, ds.xq.as<double>(), ds.tq.as<double>(), d_sites, n_rows, pv.start, pv.rjs, pv.xyz,
        pv.species, (const double *)o.c, (const double *)o.q, o.q_ld, (const double *)o.norm, d_der);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

// One CTA per site: q_c = P q / |P q| from the normalised uncompressed q (the normalisation of p
// cancels: P p / |P p| = P q / |P q|) and, for each of the site's pairs, the derivative of that
// map, dq_c = (P dq - q_c (q_c . P dq)) / |P q| (linear in dq, so the self slot stays minus the sum
// of the others). Rows of P are summed in the order their entries were given.
__global__ void __launch_bounds__(128) k_compress_rows(int n_sites, int dim, int dim_out, const int *__restrict__ row,
                                                       const int *__restrict__ col, const double *__restrict__ val,
                                                       const int64_t *__restrict__ start, const double *__restrict__ q,
                                                       const double *__restrict__ der, double *__restrict__ qc_out,
                                                       double *__restrict__ derc)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *qc = reinterpret_cast<double *>(smem_raw);  // [dim_out]
    double *vb = qc + dim_out;                           // [dim_out][3]
    double *red = vb + 3 * dim_out;                      // [4][4]: per-warp partial sums
    const int i = blockIdx.x, t = threadIdx.x, lane = t & 31, w = t >> 5;
    if (i >= n_sites) return;
    const double *qi = q + (size_t)i * dim;
    // the block's sum of (up to) three values, in a fixed order
    auto block_sum3 = [&](double a[3]) {
#pragma unroll
        for (int x = 0; x < 3; ++x)
            for (int o = 16; o > 0; o >>= 1) a[x] += __shfl_xor_sync(0xffffffffu, a[x], o);
        __syncthreads();
        if (lane == 0)
            for (int x = 0; x < 3; ++x) red[4 * w + x] = a[x];
        __syncthreads();
        for (int x = 0; x < 3; ++x) a[x] = red[x] + red[4 + x] + red[8 + x] + red[12 + x];
    };
    double s[3] = {0.0, 0.0, 0.0};
    for (int r = t; r < dim_out; r += blockDim.x) {
        double acc = 0.0;
        for (int e = row[r]; e < row[r + 1]; ++e) acc += val[e] * qi[col[e]];
        qc[r] = acc;
        s[0] += acc * acc;
    }
    block_sum3(s);
    const double nr = sqrt(s[0]), inv = nr > 0.0 ? 1.0 / nr : 0.0;
    for (int r = t; r < dim_out; r += blockDim.x) {
        qc[r] *= inv;
        qc_out[(size_t)i * dim_out + r] = qc[r];
    }
    __syncthreads();
    if (!der) return;
    for (int64_t k = start[i]; k < start[i + 1]; ++k) {
        const double *dk = der + (size_t)k * dim * 3;
        double a[3] = {0.0, 0.0, 0.0};
        for (int r = t; r < dim_out; r += blockDim.x) {
            double v[3] = {0.0, 0.0, 0.0};
            for (int e = row[r]; e < row[r + 1]; ++e)
                for (int x = 0; x < 3; ++x) v[x] += val[e] * dk[3 * col[e] + x];
            for (int x = 0; x < 3; ++x) {
                vb[3 * r + x] = v[x];
                a[x] += qc[r] * v[x];
            }
        }
        block_sum3(a);
        double *out = derc + (size_t)k * dim_out * 3;
        for (int r = t; r < dim_out; r += blockDim.x)
            for (int x = 0; x < 3; ++x) out[3 * r + x] = (vb[3 * r + x] - qc[r] * a[x]) * inv;
        __syncthreads();
    }
}

int soap_compress_rows(tgap_context *ctx, const DeviceSoap &ds, int n_sites, const int64_t *d_start,
                       const double *d_q, const double *d_der, double *d_qc, double *d_derc)
{
    if (n_sites <= 0) return TGAP_OK;
    const int dim_out = ds.p.dim_out;
    const size_t sm = sizeof(double) * (4 * (size_t)dim_out + 16);
    if (sm > 227 * 1024) return set_error(ctx, TGAP_ERR_UNSUPPORTED, "compressed length %d too large", dim_out);
    StageScope sc(ctx, "soap_compress_f64");
    TGAP_CUDA(ctx, cudaFuncSetAttribute(k_compress_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_compress_rows<<<n_sites, 128, sm, ctx->stream>>>(n_sites, ds.p.dim, dim_out, ds.p.cmp_row, ds.p.cmp_rcol,
                                                       ds.p.cmp_rval, d_start, d_q, d_der, d_qc, d_derc);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

int upload_soap(tgap_context *ctx, const SoapParams &p, const SoapTables &t, DeviceSoap *d)
{
    d->p = p;
    const size_t nx = t.xq.size(), nt = t.tq.size(), nc = t.central.size();
    if (d->xq.ensure(nx * 8) || d->tq.ensure(nt * 8) || d->central.ensure(nc * 8) ||
        d->xq32.ensure(nx * 4) || d->tq32.ensure(nt * 4) || d->central32.ensure(nc * 4))
        return set_error(ctx, TGAP_ERR_NOMEM, "descriptor tables");
    std::vector<float> xf(t.xq.begin(), t.xq.end()), tf(t.tq.begin(), t.tq.end()),
        cf(t.central.begin(), t.central.end());
    TGAP_CUDA(ctx, cudaMemcpy(d->xq.ptr, t.xq.data(), nx * 8, cudaMemcpyHostToDevice));
    TGAP_CUDA(ctx, cudaMemcpy(d->tq.ptr, t.tq.data(), nt * 8, cudaMemcpyHostToDevice));
    TGAP_CUDA(ctx, cudaMemcpy(d->central.ptr, t.central.data(), nc * 8, cudaMemcpyHostToDevice));
    TGAP_CUDA(ctx, cudaMemcpy(d->xq32.ptr, xf.data(), nx * 4, cudaMemcpyHostToDevice));
    TGAP_CUDA(ctx, cudaMemcpy(d->tq32.ptr, tf.data(), nt * 4, cudaMemcpyHostToDevice));
    TGAP_CUDA(ctx, cudaMemcpy(d->central32.ptr, cf.data(), nc * 4, cudaMemcpyHostToDevice));
    // radial table of the mixed path
    const int n_int = p.n_species * kTabIntervals;
    if (d->rtab.ensure(sizeof(float4) * (size_t)n_int * p.am_pad))
        return set_error(ctx, TGAP_ERR_NOMEM, "radial table");
    k_radial_table<<<(n_int + 127) / 128, 128, 0, ctx->stream>>>(p, d->xq.as<double>(), d->tq.as<double>(),
                                                                 d->rtab.as<float4>());
    TGAP_LAUNCH_CHECK(ctx);
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return TGAP_OK;
}

}  // namespace tgap
