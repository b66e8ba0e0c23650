// Device-side pieces of the SOAP poly3 descriptor shared by the forward, adjoint and
// materialised-derivative kernels.
//
// Per neighbor j of site i (species channel s, distance r < rcut_hard(s), unit vector u):
//   radial   R_n(r)  = gs * A(x) * sum_q T[q][n] exp(-(x_q - x)^2 / 2 sigma^2),  x = r/rcut_hard
//   angular  A_lm(r) = f_l(k) Y_lm(u), k = r^2 / sigma_t^2, f_l = i_l(k)/i_0(k)
//   c_{n l m} += R_n A_lm
// T[q][n] = w_q g_n(x_q) filter(x_q) is tabulated on the host (orthonormal poly3 basis at
// Gauss-Legendre nodes). Four lanes share one pair: lane `sub` sums the nodes q = sub mod 4
// and owns the harmonics of order m = sub mod 4.
#pragma once

#include "tgap_internal.h"

namespace tgap {

constexpr int kLanesPerPair = 4;
constexpr int kNlmMax = (kMaxL + 1) * (kMaxL + 1);

// Fully normalised Legendre recurrence (Qb_l = N_lm Q_l, Q the polynomial part of P_l^m):
//   Qb_m = N_mm (2m-1)!!,  Qb_l = ra_lm uz Qb_{l-1} - rb_lm Qb_{l-2}  (l > m)
//   ra_lm = sqrt((4l^2 - 1) / (l^2 - m^2)),
//   rb_lm = sqrt((2l+1) (l+m-1) (l-m-1) / ((2l-3) (l+m) (l-m)))  (0 for l = m + 1),
// the three-term recurrence of the unnormalised Q divided through by the normalisations. The
// coefficients of order m for target degrees l = m+1 .. kMaxL+1 sit at rec_off(m) + l - m - 1.
constexpr int kRecN = (kMaxL + 1) * (kMaxL + 2) / 2;
__host__ __device__ constexpr int rec_off(int m) { return m * (kMaxL + 1) - m * (m - 1) / 2; }

// (2m-1)!! and the normalisation sqrt((2l+1)/(4 pi) (l-m)!/(l+m)!) (times sqrt 2 for m > 0).
struct YlmConst {
    double dfact[kMaxL + 1];
    double norm[(kMaxL + 1) * (kMaxL + 2) / 2];  // index l (l+1)/2 + m
    double inv_int[kMaxL + 1];                   // 1 / k (0 for k = 0)
    double qb0[kMaxL + 1];                       // Qb_m = N_mm (2m-1)!!
    double ra[kRecN], rb[kRecN];                 // recurrence coefficients, packed by rec_off
    float dfact_f[kMaxL + 1];                    // single-precision copies
    float norm_f[(kMaxL + 1) * (kMaxL + 2) / 2];
    float inv_int_f[kMaxL + 1];
    float qb0_f[kMaxL + 1];
    float ra_f[kRecN], rb_f[kRecN];
};

// Constants in the arithmetic type of the caller.
template <class T> __device__ __forceinline__ T yc_dfact(const YlmConst &Y, int i);
template <> __device__ __forceinline__ double yc_dfact<double>(const YlmConst &Y, int i) { return Y.dfact[i]; }
template <> __device__ __forceinline__ float yc_dfact<float>(const YlmConst &Y, int i) { return Y.dfact_f[i]; }
template <class T> __device__ __forceinline__ T yc_norm(const YlmConst &Y, int i);
template <> __device__ __forceinline__ double yc_norm<double>(const YlmConst &Y, int i) { return Y.norm[i]; }
template <> __device__ __forceinline__ float yc_norm<float>(const YlmConst &Y, int i) { return Y.norm_f[i]; }
template <class T> __device__ __forceinline__ T yc_inv(const YlmConst &Y, int i);
template <> __device__ __forceinline__ double yc_inv<double>(const YlmConst &Y, int i) { return Y.inv_int[i]; }
template <> __device__ __forceinline__ float yc_inv<float>(const YlmConst &Y, int i) { return Y.inv_int_f[i]; }
template <class T> __device__ __forceinline__ T yc_qb0(const YlmConst &Y, int m);
template <> __device__ __forceinline__ double yc_qb0<double>(const YlmConst &Y, int m) { return Y.qb0[m]; }
template <> __device__ __forceinline__ float yc_qb0<float>(const YlmConst &Y, int m) { return Y.qb0_f[m]; }
template <class T> __device__ __forceinline__ T yc_ra(const YlmConst &Y, int i);
template <> __device__ __forceinline__ double yc_ra<double>(const YlmConst &Y, int i) { return Y.ra[i]; }
template <> __device__ __forceinline__ float yc_ra<float>(const YlmConst &Y, int i) { return Y.ra_f[i]; }
template <class T> __device__ __forceinline__ T yc_rb(const YlmConst &Y, int i);
template <> __device__ __forceinline__ double yc_rb<double>(const YlmConst &Y, int i) { return Y.rb[i]; }
template <> __device__ __forceinline__ float yc_rb<float>(const YlmConst &Y, int i) { return Y.rb_f[i]; }

// Host copy of the harmonic constants (computed once); passed to the warp kernels by value.
const YlmConst &ylm_host_constants();

template <class T> __device__ __forceinline__ T t_exp(T x);
template <> __device__ __forceinline__ double t_exp<double>(double x) { return exp(x); }
template <> __device__ __forceinline__ float t_exp<float>(float x) { return __expf(x); }
template <class T> __device__ __forceinline__ T t_sqrt(T x);
template <> __device__ __forceinline__ double t_sqrt<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float t_sqrt<float>(float x) { return sqrtf(x); }
template <class T> __device__ __forceinline__ T t_pow(T x, T y);
template <> __device__ __forceinline__ double t_pow<double>(double x, double y) { return pow(x, y); }
template <> __device__ __forceinline__ float t_pow<float>(float x, float y) { return powf(x, y); }
template <class T> __device__ __forceinline__ T t_tanh_inv(T x);  // 1 / tanh(x)
template <> __device__ __forceinline__ double t_tanh_inv<double>(double x) { return 1.0 / tanh(x); }
template <> __device__ __forceinline__ float t_tanh_inv<float>(float x) { return 1.0f / tanhf(x); }

// Amplitude A(x) and dA/dx for scaling_mode "polynomial" and radial_enhancement 0..2.
template <class T>
__device__ __forceinline__ void radial_amplitude(const SoapParams &P, int s, T x, T sig, T dsig,
                                                 T *A, T *dA)
{
    const T as = (T)P.amplitude_scaling[s];
    T a, da;
    if (as == (T)0) {
        a = (T)1 / sig;
        da = -dsig / (sig * sig);
    } else {
        T g = (T)1 + (T)2 * x * x * x - (T)3 * x * x;
        if (g <= (T)1.0e-10) {
            a = 0;
            da = 0;
        } else if (as == (T)1) {
            a = g / sig;
            da = (T)6 / sig * (x * x - x) - dsig / sig * a;
        } else {
            a = t_pow<T>(g, as) / sig;
            da = (T)6 * as / sig * (x * x - x) * t_pow<T>(g, as - (T)1) - dsig / sig * a;
        }
    }
    if (P.radial_enhancement == 1) {
        const T c1 = (T)0.79788456080286536;  // sqrt(2/pi)
        T e = x + c1 * sig, de = (T)1 + c1 * dsig;
        da = a * de + da * e;
        a = a * e;
    } else if (P.radial_enhancement == 2) {
        const T c2 = (T)1.5957691216057308;  // sqrt(8/pi)
        T e = x * x + sig * sig + c2 * sig * x;
        T de = (T)2 * x + (T)2 * sig * dsig + c2 * (sig + x * dsig);
        da = a * de + da * e;
        a = a * e;
    }
    *A = a;
    *dA = da;
}

// Partial node sums of one lane; DERIV adds the x-derivative of the Gaussian.
template <class T, bool DERIV>
__device__ __forceinline__ void radial_node_sums(const SoapParams &P, int s, bool valid,
                                                 const T *__restrict__ xq,
                                                 const T *__restrict__ tq, T x, T sig, T dsig,
                                                 int sub, T *sum, T *dsum)
{
    const int am = P.alpha_max[s];
    const int nn = valid ? P.n_nodes[s] : 0;
    const T *xs = xq + P.node_off[s];
    const T *tqs = tq + P.tq_off[s];
#pragma unroll
    for (int n = 0; n < kMaxAlpha; ++n) {
        sum[n] = 0;
        if (DERIV) dsum[n] = 0;
    }
    const T inv2s2 = (T)1 / ((T)2 * sig * sig);
    const T is2 = (T)1 / (sig * sig);
    const T ds3 = dsig / (sig * sig * sig);
    for (int q = sub; q < nn; q += kLanesPerPair) {
        const T u = xs[q] - x;
        const T G = t_exp<T>(-u * u * inv2s2);
        const T *t = tqs + (size_t)q * am;
        T dG = 0;
        if (DERIV) dG = G * (u * is2 + u * u * ds3);
#pragma unroll
        for (int n = 0; n < kMaxAlpha; ++n) {
            if (n < am) {
                const T tv = t[n];
                sum[n] += tv * G;
                if (DERIV) dsum[n] += tv * dG;
            }
        }
    }
    // combine the four lanes of the pair (warp-uniform bound: every lane shuffles)
#pragma unroll
    for (int n = 0; n < kMaxAlpha; ++n) {
        if (n < P.max_alpha) {
            sum[n] += __shfl_xor_sync(0xffffffffu, sum[n], 1);
            sum[n] += __shfl_xor_sync(0xffffffffu, sum[n], 2);
            if (DERIV) {
                dsum[n] += __shfl_xor_sync(0xffffffffu, dsum[n], 1);
                dsum[n] += __shfl_xor_sync(0xffffffffu, dsum[n], 2);
            }
        }
    }
}

// f_l = i_l(k)/i_0(k) for l = 0..L+1 (upward recurrence when k > L+2, continued fraction
// from l = L+33 otherwise).
template <class T>
__device__ __forceinline__ void bessel_ratios(int L, T k, T *f)
{
    const int top = L + 1;
    if (k < (T)1.0e-12) {
#pragma unroll
        for (int l = 0; l <= kMaxL + 1; ++l) f[l] = (l == 0) ? (T)1 : (T)0;
        return;
    }
    if (k > (T)(L + 2)) {
        f[0] = 1;
        f[1] = t_tanh_inv<T>(k) - (T)1 / k;
#pragma unroll
        for (int l = 1; l <= kMaxL; ++l)
            if (l < top) f[l + 1] = f[l - 1] - (T)(2 * l + 1) / k * f[l];
    } else {
        T rho = 0;
        T ratio[kMaxL + 2];
        for (int l = top + 32; l > top; --l) rho = k / ((T)(2 * l + 1) + k * rho);
#pragma unroll
        for (int l = kMaxL + 1; l >= 1; --l) {
            if (l <= top) {
                rho = k / ((T)(2 * l + 1) + k * rho);
                ratio[l] = rho;
            }
        }
        f[0] = 1;
#pragma unroll
        for (int l = 1; l <= kMaxL + 1; ++l)
            if (l <= top) f[l] = f[l - 1] * ratio[l];
    }
}

// Radial values (and d/dr) by quadrature: R_n = gs A(x) sum_q T[q][n] exp(-(x_q - x)^2 / 2 sig^2).
template <class T, int AMB, bool DERIV>
__device__ __forceinline__ void radial_quad(const SoapParams &P, int s, T r, const T *__restrict__ xq,
                                            const T *__restrict__ tq, T R[AMB], T dR[AMB])
{
    const int am = P.alpha_max[s];
    const T rc = (T)P.rcut_hard[s];
    const T x = r / rc;
    const T sig = ((T)P.sigma_r[s] + (T)P.sigma_r_scaling[s] * r) / rc;
    const T dsig = (T)P.sigma_r_scaling[s];
    T A, dA;
    radial_amplitude<T>(P, s, x, sig, dsig, &A, &dA);
    T sum[AMB], dsum[AMB];
#pragma unroll
    for (int n = 0; n < AMB; ++n) {
        sum[n] = 0;
        dsum[n] = 0;
    }
    const T inv2s2 = (T)1 / ((T)2 * sig * sig);
    const T is2 = (T)1 / (sig * sig);
    const T ds3 = dsig / (sig * sig * sig);
    const T *xs = xq + P.node_off[s];
    const T *ts = tq + P.tq_off[s];
    const int nn = P.n_nodes[s];
    for (int q = 0; q < nn; ++q) {
        const T u = xs[q] - x;
        const T G = t_exp<T>(-u * u * inv2s2);
        const T *t = ts + q * am;
        const T dG = DERIV ? G * (u * is2 + u * u * ds3) : (T)0;
#pragma unroll
        for (int n = 0; n < AMB; ++n) {
            if (n < am) {
                const T tv = t[n];
                sum[n] += tv * G;
                if (DERIV) dsum[n] += tv * dG;
            }
        }
    }
    const T gs = (T)P.global_scaling[s];
#pragma unroll
    for (int n = 0; n < AMB; ++n) {
        R[n] = gs * A * sum[n];
        dR[n] = DERIV ? gs * (dA * sum[n] + A * dsum[n]) / rc : (T)0;
    }
}

}  // namespace tgap
