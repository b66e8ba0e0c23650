// SOAP poly3 descriptor kernels (sm_100a): forward expansion + power spectrum, adjoint
// back-scatter of dE/dq to forces and virial, and the materialised dq/dr of the reference
// get_soap surface (soap_cart_der, call site src/gap/gap_interface.f90:301-306).
//
// One CTA of 256 threads owns one central site. Pairs are processed in chunks of 64; the
// four lanes of a pair split the radial quadrature nodes and the harmonic orders m, so a
// chunk fills the CTA. The expansion c_{n,lm} = sum_j R_n(r_j) A_lm(r_j) is then a small
// (n_max x 64) x (64 x nlm) product out of shared memory. The templates run in FP64 (plain
// path) or FP32 (mixed path); positions, pair vectors, forces and the virial stay FP64.
#include <cuda_bf16.h>

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
    YlmConst h;
    double df = 1.0;
    for (int m = 0; m <= kMaxL; ++m) {
        if (m > 0) df *= (2.0 * m - 1.0);
        h.dfact[m] = df;
    }
    for (int l = 0; l <= kMaxL; ++l) {
        double fr = 1.0;
        for (int m = 0; m <= l; ++m) {
            if (m > 0) fr /= (double)(l + m) * (double)(l - m + 1);
            double N = std::sqrt((2.0 * l + 1.0) / (4.0 * M_PI) * fr);
            h.norm[l * (l + 1) / 2 + m] = m == 0 ? N : N * M_SQRT2;
        }
    }
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

// ----------------------------------------------------------------------------- forward

template <class T, bool SPLIT>
__global__ void __launch_bounds__(kThreads) k_soap_forward(
    SoapParams P, const T *__restrict__ xq, const T *__restrict__ tq, const T *__restrict__ central,
    const int *__restrict__ sites, int n_rows, const int64_t *__restrict__ start,
    const double *__restrict__ rjs, const double *__restrict__ xyz, const int *__restrict__ nsp,
    T *__restrict__ c_out, T *__restrict__ q_out, int q_ld, T *__restrict__ norm_out,
    __nv_bfloat16 *__restrict__ q_hi, __nv_bfloat16 *__restrict__ q_lo)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *smem = reinterpret_cast<T *>(smem_raw);
    const int nmax = P.n_max, L = P.l_max, nlm = (L + 1) * (L + 1), dim = P.dim;
    T *Rs = smem;                               // [64][nmax]
    T *As = Rs + kPairsPerChunk * nmax;         // [64][nlm]
    T *cs = As + kPairsPerChunk * nlm;          // [nmax][nlm]
    T *ps = cs + nmax * nlm;                    // [dim]
    T *red = ps + dim;                          // [32]

    const int row = blockIdx.x;
    if (row >= n_rows) return;
    const int site = sites ? sites[row] : row;
    const int64_t kb = start[site], ke = start[site + 1];
    const int t = threadIdx.x, pl = t >> 2, sub = t & 3;
    const int nout = nmax * nlm;
    constexpr int kMaxOut = (kMaxNmax * kNlmMax + kThreads - 1) / kThreads;
    T creg[kMaxOut];
#pragma unroll
    for (int j = 0; j < kMaxOut; ++j) creg[j] = 0;

    for (int64_t cb = kb; cb < ke; cb += kPairsPerChunk) {
        for (int i = t; i < kPairsPerChunk * (nmax + nlm); i += kThreads) Rs[i] = 0;
        __syncthreads();
        const int64_t k = cb + pl;
        int s;
        T r, u[3], rv[3];
        const bool valid = pair_setup<T>(P, k, kb, ke, rjs, xyz, nsp, &s, &r, u, rv);
        const T rc = (T)P.rcut_hard[s];
        const T x = r / rc;
        const T sig = ((T)P.sigma_r[s] + (T)P.sigma_r_scaling[s] * r) / rc;
        const T dsig = (T)P.sigma_r_scaling[s];
        T sum[kMaxAlpha], dsum[kMaxAlpha];
        radial_node_sums<T, false>(P, s, valid, xq, tq, x, sig, dsig, sub, sum, dsum);
        if (valid) {
            T A, dA;
            radial_amplitude<T>(P, s, x, sig, dsig, &A, &dA);
            const T g = (T)P.global_scaling[s] * A;
            if (sub == 0) {
                const int off = P.n_off[s];
#pragma unroll
                for (int n = 0; n < kMaxAlpha; ++n)
                    if (n < P.alpha_max[s]) Rs[pl * nmax + off + n] = g * sum[n];
            }
            const T st = (T)P.sigma_t[s] + (T)P.sigma_t_scaling[s] * r;
            T f[kMaxL + 2];
            bessel_ratios<T>(L, r * r / (st * st), f);
            T *Arow = As + pl * nlm;
            ylm_lane<T, false>(L, u[0], u[1], u[2], sub,
                               [&](int kk, int l, T Y, T, T, T) { Arow[kk] = f[l] * Y; });
        }
        __syncthreads();
        // c += R^T A over the chunk
#pragma unroll
        for (int j = 0; j < kMaxOut; ++j) {
            const int o = t + j * kThreads;
            if (o < nout) {
                const int n = o / nlm, kk = o - n * nlm;
                T acc = 0;
#pragma unroll 8
                for (int p = 0; p < kPairsPerChunk; ++p) acc += Rs[p * nmax + n] * As[p * nlm + kk];
                creg[j] += acc;
            }
        }
        __syncthreads();
    }
    // central atom (self slot species) on l = 0
    const int s_self = nsp[kb] - 1;
#pragma unroll
    for (int j = 0; j < kMaxOut; ++j) {
        const int o = t + j * kThreads;
        if (o < nout) {
            const int n = o / nlm, kk = o - n * nlm;
            T v = creg[j];
            if (kk == 0 && s_self >= 0 && s_self < P.n_species && n >= P.n_off[s_self] &&
                n < P.n_off[s_self] + P.alpha_max[s_self])
                v += central[n];
            cs[o] = v;
            c_out[(size_t)row * nout + o] = v;
        }
    }
    __syncthreads();
    // power spectrum
    T part = 0;
    for (int d = t; d < dim; d += kThreads) {
        int n, np, l;
        ps_decode(d, nmax, L, &n, &np, &l);
        const T *a = cs + n * nlm, *b = cs + np * nlm;
        T acc = 0;
        for (int kk = l * l; kk < (l + 1) * (l + 1); ++kk) acc += a[kk] * b[kk];
        const T v = (n == np) ? acc : acc * (T)1.4142135623730951;
        ps[d] = v;
        part += v * v;
    }
    const T nrm2 = block_sum<T>(part, red);
    const T nrm = t_sqrt<T>(nrm2);
    const T inv = nrm > (T)0 ? (T)1 / nrm : (T)0;
    for (int d = t; d < q_ld; d += kThreads) {
        T qv = d < dim ? ps[d] * inv : (T)0;
        q_out[(size_t)row * q_ld + d] = qv;
        if (SPLIT) {
            const float qf = (float)qv;
            const __nv_bfloat16 h = __float2bfloat16_rn(qf);
            q_hi[(size_t)row * q_ld + d] = h;
            q_lo[(size_t)row * q_ld + d] = __float2bfloat16_rn(qf - __bfloat162float(h));
        }
    }
    if (t == 0) norm_out[row] = nrm;
}

// ----------------------------------------------------------------------------- adjoint

// g: dE/dq per row (GT = double or float). forces: 3 per global atom, virial: 9 per structure.
template <class T, class GT>
__global__ void __launch_bounds__(kThreads) k_soap_backward(
    SoapParams P, const T *__restrict__ xq, const T *__restrict__ tq, const int *__restrict__ sites,
    int n_rows, const int64_t *__restrict__ start, const double *__restrict__ rjs,
    const double *__restrict__ xyz, const int *__restrict__ nsp, const int *__restrict__ jatom,
    const int *__restrict__ site_struct, const T *__restrict__ c_in, const T *__restrict__ q_in,
    int q_ld, const T *__restrict__ norm_in, const GT *__restrict__ g_in, int g_ld,
    double *__restrict__ forces, double *__restrict__ virial)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *dred = reinterpret_cast<double *>(smem_raw);  // [9][8] per-warp partials
    T *smem = reinterpret_cast<T *>(smem_raw + 80 * sizeof(double));
    const int nmax = P.n_max, L = P.l_max, nlm = (L + 1) * (L + 1), dim = P.dim;
    T *cs = smem;               // [nmax][nlm]
    T *Gc = cs + nmax * nlm;    // [nmax][nlm]
    T *hs = Gc + nmax * nlm;    // [dim]
    T *red = hs + dim;          // [32]

    const int row = blockIdx.x;
    if (row >= n_rows) return;
    const int site = sites ? sites[row] : row;
    const int64_t kb = start[site], ke = start[site + 1];
    const int t = threadIdx.x, pl = t >> 2, sub = t & 3;
    const int nout = nmax * nlm;
    for (int o = t; o < nout; o += kThreads) cs[o] = c_in[(size_t)row * nout + o];
    T part = 0;
    for (int d = t; d < dim; d += kThreads)
        part += q_in[(size_t)row * q_ld + d] * (T)g_in[(size_t)row * g_ld + d];
    const T qg = block_sum<T>(part, red);
    const T nrm = norm_in[row];
    const T inv = nrm > (T)0 ? (T)1 / nrm : (T)0;
    for (int d = t; d < dim; d += kThreads)
        hs[d] = ((T)g_in[(size_t)row * g_ld + d] - q_in[(size_t)row * q_ld + d] * qg) * inv;
    __syncthreads();
    // dE/dc_{n,lm} = sum_n' M_l[n][n'] c_{n',lm}
    for (int o = t; o < nout; o += kThreads) {
        const int n = o / nlm, kk = o - n * nlm;
        int l = 0;
        while ((l + 1) * (l + 1) <= kk) ++l;
        T acc = 0;
        for (int np = 0; np < nmax; ++np) {
            const T h = hs[ps_index(n, np, nmax, L, l)];
            const T coef = (np == n) ? (T)2 * h : (T)1.4142135623730951 * h;
            acc += coef * cs[np * nlm + kk];
        }
        Gc[o] = acc;
    }
    __syncthreads();

    double fself[3] = {0, 0, 0}, vir[6] = {0, 0, 0, 0, 0, 0};
    for (int64_t cb = kb; cb < ke; cb += kPairsPerChunk) {
        const int64_t k = cb + pl;
        int s;
        T r, u[3], rv[3];
        const bool valid = pair_setup<T>(P, k, kb, ke, rjs, xyz, nsp, &s, &r, u, rv);
        const T rc = (T)P.rcut_hard[s];
        const T x = r / rc;
        const T sig = ((T)P.sigma_r[s] + (T)P.sigma_r_scaling[s] * r) / rc;
        const T dsig = (T)P.sigma_r_scaling[s];
        T sum[kMaxAlpha], dsum[kMaxAlpha];
        radial_node_sums<T, true>(P, s, valid, xq, tq, x, sig, dsig, sub, sum, dsum);
        T w0 = 0, w1 = 0, w2 = 0;
        if (valid) {
            T A, dA;
            radial_amplitude<T>(P, s, x, sig, dsig, &A, &dA);
            const T gs = (T)P.global_scaling[s];
            T R[kMaxAlpha], dR[kMaxAlpha];
#pragma unroll
            for (int n = 0; n < kMaxAlpha; ++n) {
                R[n] = gs * A * sum[n];
                dR[n] = gs * (dA * sum[n] + A * dsum[n]) / rc;
            }
            const T st = (T)P.sigma_t[s] + (T)P.sigma_t_scaling[s] * r;
            const T kap = r * r / (st * st);
            const T dkap = (T)2 * r / (st * st) -
                           (T)2 * r * r * (T)P.sigma_t_scaling[s] / (st * st * st);
            T f[kMaxL + 2];
            bessel_ratios<T>(L, kap, f);
            const T ir = (T)1 / r;
            const int off = P.n_off[s], am = P.alpha_max[s];
            ylm_lane<T, true>(L, u[0], u[1], u[2], sub, [&](int kk, int l, T Y, T gx, T gy, T gz) {
                T U = 0, V = 0;
#pragma unroll
                for (int n = 0; n < kMaxAlpha; ++n) {
                    if (n < am) {
                        const T gcv = Gc[(off + n) * nlm + kk];
                        U += gcv * R[n];
                        V += gcv * dR[n];
                    }
                }
                const T fl = f[l];
                const T dfl = (f[l + 1] + (T)l / kap * fl - fl * f[1]) * dkap;
                const T ug = u[0] * gx + u[1] * gy + u[2] * gz;
                const T Ak = fl * Y;
                const T radial_part = Ak * V + U * dfl * Y;
                const T tang = U * fl * ir;
                w0 += u[0] * radial_part + tang * (gx - u[0] * ug);
                w1 += u[1] * radial_part + tang * (gy - u[1] * ug);
                w2 += u[2] * radial_part + tang * (gz - u[2] * ug);
            });
        }
        w0 += __shfl_xor_sync(0xffffffffu, w0, 1);
        w0 += __shfl_xor_sync(0xffffffffu, w0, 2);
        w1 += __shfl_xor_sync(0xffffffffu, w1, 1);
        w1 += __shfl_xor_sync(0xffffffffu, w1, 2);
        w2 += __shfl_xor_sync(0xffffffffu, w2, 1);
        w2 += __shfl_xor_sync(0xffffffffu, w2, 2);
        if (valid && sub == 0) {
            // w = dE_i/dr_ij; force on j is -w, on i is +w (self slot of the reference)
            const double f0 = -(double)w0, f1 = -(double)w1, f2 = -(double)w2;
            const int j = jatom[k];
            atomicAdd(forces + 3 * (size_t)j, f0);
            atomicAdd(forces + 3 * (size_t)j + 1, f1);
            atomicAdd(forces + 3 * (size_t)j + 2, f2);
            fself[0] -= f0;
            fself[1] -= f1;
            fself[2] -= f2;
            const double x0 = xyz[3 * k], x1 = xyz[3 * k + 1], x2 = xyz[3 * k + 2];
            vir[0] += f0 * x0;
            vir[1] += f1 * x1;
            vir[2] += f2 * x2;
            vir[3] += 0.5 * (f0 * x1 + f1 * x0);
            vir[4] += 0.5 * (f0 * x2 + f2 * x0);
            vir[5] += 0.5 * (f1 * x2 + f2 * x1);
        }
    }
    // reduce self force and virial over the CTA
    double vals[9] = {fself[0], fself[1], fself[2], vir[0], vir[1], vir[2], vir[3], vir[4], vir[5]};
    const int lane = t & 31, wid = t >> 5;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        double v = vals[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) dred[i * 8 + wid] = v;
    }
    __syncthreads();
    if (t < 9) {
        double v = 0;
        for (int w = 0; w < kThreads / 32; ++w) v += dred[t * 8 + w];
        if (t < 3) {
            atomicAdd(forces + 3 * (size_t)jatom[kb] + t, v);
        } else {
            const int st = site_struct ? site_struct[site] : 0;
            double *V = virial + 9 * (size_t)st;
            // xx yy zz xy xz yz -> column-major 3x3 (symmetric)
            const int idx[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
            const int a = idx[t - 3][0], b = idx[t - 3][1];
            atomicAdd(V + a + 3 * b, v);
            if (a != b) atomicAdd(V + b + 3 * a, v);
        }
    }
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

static size_t fwd_smem(const SoapParams &P, size_t tsz)
{
    const int nlm = (P.l_max + 1) * (P.l_max + 1);
    return tsz * ((size_t)kPairsPerChunk * (P.n_max + nlm) + (size_t)P.n_max * nlm + P.dim + 32);
}

static size_t bwd_smem(const SoapParams &P, size_t tsz)
{
    const int nlm = (P.l_max + 1) * (P.l_max + 1);
    return tsz * ((size_t)2 * P.n_max * nlm + P.dim + 34) + sizeof(double) * 80;
}

static size_t der_smem(const SoapParams &P)
{
    const int nlm = (P.l_max + 1) * (P.l_max + 1);
    return sizeof(double) * ((size_t)P.n_max * nlm + 4 * (size_t)nlm + 2 * kMaxAlpha + 40);
}

template <class T, bool SPLIT>
static int launch_forward(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv,
                          const int *d_sites, int n_rows, SoapOut &o)
{
    const size_t sm = fwd_smem(ds.p, sizeof(T));
    auto kern = k_soap_forward<T, SPLIT>;
    TGAP_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    const T *xq = std::is_same<T, double>::value ? (const T *)ds.xq.ptr : (const T *)ds.xq32.ptr;
    const T *tq = std::is_same<T, double>::value ? (const T *)ds.tq.ptr : (const T *)ds.tq32.ptr;
    const T *ce = std::is_same<T, double>::value ? (const T *)ds.central.ptr : (const T *)ds.central32.ptr;
    kern<<<n_rows, kThreads, sm, ctx->stream>>>(ds.p, xq, tq, ce, d_sites, n_rows, pv.start, pv.rjs,
                                                pv.xyz, pv.species, (T *)o.c, (T *)o.q, o.q_ld,
                                                (T *)o.norm, o.q_hi, o.q_lo);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

int soap_forward(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites,
                 int n_rows, int precision, SoapOut &o)
{
    if (n_rows <= 0) return TGAP_OK;
    StageScope sc(ctx, precision == TGAP_FP64 ? "soap_forward_f64" : "soap_forward_f32");
    if (precision == TGAP_FP64) return launch_forward<double, false>(ctx, ds, pv, d_sites, n_rows, o);
    if (o.q_hi) return launch_forward<float, true>(ctx, ds, pv, d_sites, n_rows, o);
    return launch_forward<float, false>(ctx, ds, pv, d_sites, n_rows, o);
}

int soap_backward(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites,
                  int n_rows, int precision, const SoapOut &o, const void *d_g, int g_ld,
                  int g_is_double, const int *site_struct, double *d_forces, double *d_virial)
{
    if (n_rows <= 0) return TGAP_OK;
    StageScope sc(ctx, precision == TGAP_FP64 ? "soap_backward_f64" : "soap_backward_f32");
    if (precision == TGAP_FP64) {
        const size_t sm = bwd_smem(ds.p, sizeof(double));
        auto kern = k_soap_backward<double, double>;
        TGAP_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        kern<<<n_rows, kThreads, sm, ctx->stream>>>(
            ds.p, ds.xq.as<double>(), ds.tq.as<double>(), d_sites, n_rows, pv.start, pv.rjs, pv.xyz,
            pv.species, pv.jatom, site_struct, (const double *)o.c, (const double *)o.q, o.q_ld,
            (const double *)o.norm, (const double *)d_g, g_ld, d_forces, d_virial);
    } else {
        const size_t sm = bwd_smem(ds.p, sizeof(float));
        if (g_is_double) {
            auto kern = k_soap_backward<float, double>;
            TGAP_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            kern<<<n_rows, kThreads, sm, ctx->stream>>>(
                ds.p, ds.xq32.as<float>(), ds.tq32.as<float>(), d_sites, n_rows, pv.start, pv.rjs,
                pv.xyz, pv.species, pv.jatom, site_struct, (const float *)o.c, (const float *)o.q,
                o.q_ld, (const float *)o.norm, (const double *)d_g, g_ld, d_forces, d_virial);
        } else {
            auto kern = k_soap_backward<float, float>;
            TGAP_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            kern<<<n_rows, kThreads, sm, ctx->stream>>>(
                ds.p, ds.xq32.as<float>(), ds.tq32.as<float>(), d_sites, n_rows, pv.start, pv.rjs,
                pv.xyz, pv.species, pv.jatom, site_struct, (const float *)o.c, (const float *)o.q,
                o.q_ld, (const float *)o.norm, (const float *)d_g, g_ld, d_forces, d_virial);
        }
    }
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
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
    return TGAP_OK;
}

}  // namespace tgap
