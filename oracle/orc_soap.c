/*
 * ORACLE — test infrastructure only (see tgap_oracle.h).
 *
 * SOAP "poly3" descriptor, restated from the published method (M. A. Caro, Phys. Rev. B
 * 100, 024112 (2019)) because the soap_turbo sources that TurboGAP calls
 * (src/gap/gap_interface.f90:301-306) are not available. Parity vs soap_turbo: UNPINNED.
 * Parameter meanings follow the model reader (src/gap/read_gap.f90:156-432).
 *
 * Definition (all radial quantities in units of rcut_hard of the neighbor's species s):
 *   x = r / rcut_hard,  sigma(x) = (atom_sigma_r + atom_sigma_r_scaling r) / rcut_hard
 *   basis    phi_a(x) = sqrt(2a+5) (1-x)^(a+2), a = 1..alpha_max ("poly3"),
 *            g_n = sum_a W_na phi_a with W = S^{-1/2}, S_ab = sqrt((2a+5)(2b+5))/(a+b+5)
 *   density  rho_j(x) = A(x_j) exp(-(x-x_j)^2 / 2 sigma^2) on [0, xs], xs = rcut_soft/rcut_hard,
 *            times the filter exp(-(x-xs)^2 / 2 sf^2), sf = (1-xs)/nf, on [xs, 1]
 *   amplitude (scaling_mode "polynomial") A = (1 + 2x^3 - 3x^2)^amplitude_scaling / sigma,
 *            times (x + sqrt(2/pi) sigma) or (x^2 + sigma^2 + sqrt(8/pi) sigma x) for
 *            radial_enhancement 1 or 2
 *   radial   R_n(r) = global_scaling * int_0^1 g_n(x) rho_j(x) dx
 *   angular  f_l(k) Y_lm(r_hat), k = r^2 / sigma_t^2, f_l = i_l(k)/i_0(k) (modified spherical
 *            Bessel ratio: the spherical-harmonic expansion of a Gaussian of angular width
 *            sigma_t/r on the sphere), Y_lm real orthonormal harmonics
 *   c_nlm    = sum_j R_n(r_j) f_l Y_lm(r_hat_j) + central_weight R_n(0) Y_00 (the site itself)
 *   p_nn'l   = m_nn' sum_m c_nlm c_n'lm, n <= n', m_nn' = 1 (n = n') or sqrt(2); q = p / |p|
 *
 * The radial integral is evaluated by Gauss-Legendre quadrature on [0, xs] and [xs, 1]
 * against the orthonormal basis tabulated once per species in binary128. Expanding the
 * integral in raw phi_a and applying W would amplify rounding by ~1e6 (lambda_min(S) ~ 6e-13
 * for alpha_max = 8); the tabulated form does not.
 */
#include "tgap_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef __float128 quad;

#define ORC_MAX_ALPHA 16
#define ORC_MAX_L 12
#define ORC_MAX_NODES 192

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ---------------------------------------------------------------- binary128 helpers */

static quad q_sqrt(quad x)
{
    if (x <= 0) return 0;
    quad y = (quad)sqrt((double)x);
    for (int it = 0; it < 4; ++it) y = (y + x / y) / 2;
    return y;
}

static quad q_abs(quad x) { return x < 0 ? -x : x; }

/* Cyclic Jacobi eigen-decomposition of a symmetric n x n matrix (row-major). */
static void q_jacobi(int n, quad *A, quad *V)
{
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) V[i * n + j] = (i == j) ? 1 : 0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        quad off = 0, tot = 0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                tot += A[i * n + j] * A[i * n + j];
                if (i != j) off += A[i * n + j] * A[i * n + j];
            }
        if (off <= tot * (quad)1e-66Q) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                quad apq = A[p * n + q];
                if (apq == 0) continue;
                quad theta = (A[q * n + q] - A[p * n + p]) / (2 * apq);
                quad t = 1 / (q_abs(theta) + q_sqrt(theta * theta + 1));
                if (theta < 0) t = -t;
                quad c = 1 / q_sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < n; ++k) {
                    quad akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = c * akp - s * akq;
                    A[k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    quad apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = c * apk - s * aqk;
                    A[q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    quad vkp = V[k * n + p], vkq = V[k * n + q];
                    V[k * n + p] = c * vkp - s * vkq;
                    V[k * n + q] = s * vkp + c * vkq;
                }
            }
    }
}

static void q_poly3_w(int am, quad *W)
{
    quad S[ORC_MAX_ALPHA * ORC_MAX_ALPHA], V[ORC_MAX_ALPHA * ORC_MAX_ALPHA];
    for (int a = 1; a <= am; ++a)
        for (int b = 1; b <= am; ++b)
            S[(a - 1) * am + (b - 1)] = q_sqrt((quad)((2 * a + 5) * (2 * b + 5))) / (quad)(a + b + 5);
    q_jacobi(am, S, V);
    for (int i = 0; i < am; ++i)
        for (int j = 0; j < am; ++j) {
            quad s = 0;
            for (int k = 0; k < am; ++k) s += V[i * am + k] * V[j * am + k] / q_sqrt(S[k * am + k]);
            W[i * am + j] = s;
        }
}

void orc_poly3_w(int alpha_max, double *W)
{
    quad Wq[ORC_MAX_ALPHA * ORC_MAX_ALPHA];
    q_poly3_w(alpha_max, Wq);
    for (int i = 0; i < alpha_max * alpha_max; ++i) W[i] = (double)Wq[i];
}

/* ---------------------------------------------------------------- quadrature */

/* Gauss-Legendre nodes/weights on [-1, 1] by Newton iteration on P_n. */
static void gauss_legendre(int n, double *t, double *w)
{
    for (int i = 0; i < n; ++i) {
        double z = cos(M_PI * (i + 0.75) / (n + 0.5));
        double pp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; ++j) {
                double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
            double z1 = z;
            z = z1 - p1 / pp;
            if (fabs(z - z1) < 1e-16) break;
        }
        t[i] = -z;
        w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
    }
}

static int round_up4(int n) { return (n + 3) / 4 * 4; }

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

int orc_radial_nodes(const orc_soap_hypers *h, int s, double *xq, double *tq, int cap)
{
    int am = h->alpha_max[s];
    double rc = h->rcut_hard[s];
    double xs = h->rcut_soft[s] / rc;
    double sig0 = h->atom_sigma_r[s] / rc;
    int n_in = round_up4(clampi((int)ceil(4.5 * xs / sig0), 24, 128));
    int n_buf = 0;
    double sf = 0.0;
    if (xs < 1.0) {
        sf = (1.0 - xs) / h->nf[s];
        double sc = sig0 * sf / sqrt(sig0 * sig0 + sf * sf);
        n_buf = round_up4(clampi((int)ceil(4.5 * (1.0 - xs) / sc), 16, 64));
    }
    int n = n_in + n_buf;
    if (n > cap) return -1;
    quad W[ORC_MAX_ALPHA * ORC_MAX_ALPHA];
    q_poly3_w(am, W);
    double t[128], w[128];
    for (int part = 0; part < 2; ++part) {
        int m = part == 0 ? n_in : n_buf;
        if (m == 0) continue;
        double lo = part == 0 ? 0.0 : xs, hi = part == 0 ? xs : 1.0;
        gauss_legendre(m, t, w);
        for (int i = 0; i < m; ++i) {
            int q = part == 0 ? i : n_in + i;
            double x = lo + (hi - lo) * (t[i] + 1.0) * 0.5;
            double wx = w[i] * (hi - lo) * 0.5;
            double filt = part == 0 ? 1.0 : exp(-(x - xs) * (x - xs) / (2.0 * sf * sf));
            xq[q] = x;
            for (int nn = 0; nn < am; ++nn) {
                quad g = 0, om = 1 - (quad)x, pw = om * om;
                for (int a = 1; a <= am; ++a) {
                    pw *= om; /* (1-x)^(a+2) */
                    g += W[nn * am + (a - 1)] * q_sqrt((quad)(2 * a + 5)) * pw;
                }
                tq[q * am + nn] = (double)(g * (quad)wx * (quad)filt);
            }
        }
    }
    return n;
}

/* ---------------------------------------------------------------- radial */

typedef struct {
    int n;
    double xq[ORC_MAX_NODES];
    double tq[ORC_MAX_NODES * ORC_MAX_ALPHA];
} radial_table;

static void amplitude(const orc_soap_hypers *h, int s, double x, double sig, double dsig,
                      double *A, double *dA)
{
    double as = h->amplitude_scaling[s];
    double a, da;
    if (as == 0.0) {
        a = 1.0 / sig;
        da = -dsig / (sig * sig);
    } else {
        double g = 1.0 + 2.0 * x * x * x - 3.0 * x * x;
        if (g <= 1.0e-10) {
            a = 0.0;
            da = 0.0;
        } else if (as == 1.0) {
            a = g / sig;
            da = 6.0 / sig * (x * x - x) - dsig / sig * a;
        } else {
            a = pow(g, as) / sig;
            da = 6.0 * as / sig * (x * x - x) * pow(g, as - 1.0) - dsig / sig * a;
        }
    }
    if (h->radial_enhancement == 1) {
        double e = x + sqrt(2.0 / M_PI) * sig, de = 1.0 + sqrt(2.0 / M_PI) * dsig;
        da = a * de + da * e;
        a = a * e;
    } else if (h->radial_enhancement == 2) {
        double e = x * x + sig * sig + sqrt(8.0 / M_PI) * sig * x;
        double de = 2.0 * x + 2.0 * sig * dsig + sqrt(8.0 / M_PI) * (sig + x * dsig);
        da = a * de + da * e;
        a = a * e;
    }
    *A = a;
    *dA = da;
}

static void radial_eval(const orc_soap_hypers *h, int s, const radial_table *tb, double r,
                        int central, double *R, double *dR)
{
    int am = h->alpha_max[s];
    double rc = h->rcut_hard[s];
    double x = central ? 0.0 : r / rc;
    double sig = (h->atom_sigma_r[s] + h->atom_sigma_r_scaling[s] * (central ? 0.0 : r)) / rc;
    double dsig = h->atom_sigma_r_scaling[s];
    double A, dA;
    amplitude(h, s, x, sig, dsig, &A, &dA);
    double sum[ORC_MAX_ALPHA], dsum[ORC_MAX_ALPHA];
    for (int n = 0; n < am; ++n) sum[n] = dsum[n] = 0.0;
    double inv2s2 = 1.0 / (2.0 * sig * sig);
    for (int q = 0; q < tb->n; ++q) {
        double u = tb->xq[q] - x;
        double G = exp(-u * u * inv2s2);
        double dG = G * (u / (sig * sig) + u * u * dsig / (sig * sig * sig));
        const double *t = tb->tq + q * am;
        for (int n = 0; n < am; ++n) {
            sum[n] += t[n] * G;
            dsum[n] += t[n] * dG;
        }
    }
    double gs = h->global_scaling[s] * (central ? h->central_weight[s] : 1.0);
    for (int n = 0; n < am; ++n) {
        R[n] = gs * A * sum[n];
        if (dR) dR[n] = central ? 0.0 : gs * (dA * sum[n] + A * dsum[n]) / rc;
    }
}

static radial_table *make_tables(const orc_soap_hypers *h)
{
    radial_table *tb = (radial_table *)calloc((size_t)(h->n_species > 0 ? h->n_species : 1), sizeof(radial_table));
    for (int s = 0; s < h->n_species; ++s)
        tb[s].n = orc_radial_nodes(h, s, tb[s].xq, tb[s].tq, ORC_MAX_NODES);
    return tb;
}

void orc_radial(const orc_soap_hypers *h, int s, double r, int central, double *R, double *dR)
{
    radial_table *tb = make_tables(h);
    radial_eval(h, s, tb + s, r, central, R, dR);
    free(tb);
}

/* ---------------------------------------------------------------- angular */

/* f_l = i_l(k)/i_0(k), l = 0..L, and df_l/dk. */
static void bessel_ratios(int L, double k, double *f, double *df)
{
    double fl[ORC_MAX_L + 3];
    if (k < 1.0e-12) {
        for (int l = 0; l <= L; ++l) {
            f[l] = l == 0 ? 1.0 : 0.0;
            df[l] = l == 1 ? 1.0 / 3.0 : 0.0;
        }
        return;
    }
    int top = L + 1;
    if (k > (double)(L + 2)) {
        fl[0] = 1.0;
        fl[1] = 1.0 / tanh(k) - 1.0 / k;
        for (int l = 1; l < top; ++l) fl[l + 1] = fl[l - 1] - (2.0 * l + 1.0) / k * fl[l];
    } else {
        double rho = 0.0;
        double ratio[ORC_MAX_L + 3];
        for (int l = top + 32; l >= 1; --l) {
            rho = k / (2.0 * l + 1.0 + k * rho);
            if (l <= top) ratio[l] = rho;
        }
        fl[0] = 1.0;
        for (int l = 1; l <= top; ++l) fl[l] = fl[l - 1] * ratio[l];
    }
    for (int l = 0; l <= L; ++l) {
        f[l] = fl[l];
        df[l] = fl[l + 1] + (double)l / k * fl[l] - fl[l] * fl[1];
    }
}

/* Real orthonormal spherical harmonics of a unit vector and their gradient with respect to
 * the three (independent) components of u; index l^2 + {0 | 2m-1 (cos) | 2m (sin)}. */
static void ylm_real(int L, const double u[3], double *Y, double *dY)
{
    double C[ORC_MAX_L + 1], S[ORC_MAX_L + 1];
    C[0] = 1.0;
    S[0] = 0.0;
    for (int m = 1; m <= L; ++m) {
        C[m] = u[0] * C[m - 1] - u[1] * S[m - 1];
        S[m] = u[0] * S[m - 1] + u[1] * C[m - 1];
    }
    double z = u[2];
    double Q[ORC_MAX_L + 1][ORC_MAX_L + 1], dQ[ORC_MAX_L + 1][ORC_MAX_L + 1];
    double qmm = 1.0;
    for (int m = 0; m <= L; ++m) {
        if (m > 0) qmm *= (2.0 * m - 1.0);
        Q[m][m] = qmm;
        dQ[m][m] = 0.0;
        if (m + 1 <= L) {
            Q[m + 1][m] = (2.0 * m + 1.0) * z * qmm;
            dQ[m + 1][m] = (2.0 * m + 1.0) * qmm;
        }
        for (int l = m + 2; l <= L; ++l) {
            Q[l][m] = ((2.0 * l - 1.0) * z * Q[l - 1][m] - (l + m - 1.0) * Q[l - 2][m]) / (l - m);
            dQ[l][m] = ((2.0 * l - 1.0) * (Q[l - 1][m] + z * dQ[l - 1][m]) -
                        (l + m - 1.0) * dQ[l - 2][m]) / (l - m);
        }
    }
    for (int l = 0; l <= L; ++l) {
        double fr = 1.0; /* (l-m)!/(l+m)! */
        for (int m = 0; m <= l; ++m) {
            if (m > 0) fr /= (double)(l + m) * (double)(l - m + 1);
            double N = sqrt((2.0 * l + 1.0) / (4.0 * M_PI) * fr);
            int base = l * l;
            if (m == 0) {
                Y[base] = N * Q[l][0];
                dY[3 * base] = 0.0;
                dY[3 * base + 1] = 0.0;
                dY[3 * base + 2] = N * dQ[l][0];
            } else {
                double Nr = M_SQRT2 * N;
                int kc = base + 2 * m - 1, ks = base + 2 * m;
                Y[kc] = Nr * Q[l][m] * C[m];
                Y[ks] = Nr * Q[l][m] * S[m];
                dY[3 * kc] = Nr * Q[l][m] * m * C[m - 1];
                dY[3 * kc + 1] = -Nr * Q[l][m] * m * S[m - 1];
                dY[3 * kc + 2] = Nr * dQ[l][m] * C[m];
                dY[3 * ks] = Nr * Q[l][m] * m * S[m - 1];
                dY[3 * ks + 1] = Nr * Q[l][m] * m * C[m - 1];
                dY[3 * ks + 2] = Nr * dQ[l][m] * S[m];
            }
        }
    }
}

/* Angular factor A_lm(r_vec) = f_l Y_lm(u) and its gradient with respect to r_vec. */
static void angular_eval(const orc_soap_hypers *h, int s, double r, const double u[3], double *A,
                         double *dA)
{
    int L = h->l_max, nlm = (L + 1) * (L + 1);
    double st = h->atom_sigma_t[s] + h->atom_sigma_t_scaling[s] * r;
    double k = r * r / (st * st);
    double dk = 2.0 * r / (st * st) - 2.0 * r * r * h->atom_sigma_t_scaling[s] / (st * st * st);
    double f[ORC_MAX_L + 1], df[ORC_MAX_L + 1];
    bessel_ratios(L, k, f, df);
    double Y[(ORC_MAX_L + 1) * (ORC_MAX_L + 1)], dY[3 * (ORC_MAX_L + 1) * (ORC_MAX_L + 1)];
    ylm_real(L, u, Y, dY);
    for (int l = 0; l <= L; ++l)
        for (int kk = l * l; kk < (l + 1) * (l + 1); ++kk) {
            A[kk] = f[l] * Y[kk];
            if (dA) {
                const double *g = dY + 3 * kk;
                double ug = u[0] * g[0] + u[1] * g[1] + u[2] * g[2];
                for (int x = 0; x < 3; ++x) {
                    double grad = (g[x] - u[x] * ug) / r;
                    dA[3 * kk + x] = df[l] * dk * u[x] * Y[kk] + f[l] * grad;
                }
            }
        }
    (void)nlm;
}

void orc_angular(const orc_soap_hypers *h, int s, double r, const double u[3], double *A,
                 double *dA)
{
    angular_eval(h, s, r, u, A, dA);
}

/* ---------------------------------------------------------------- get_soap */

int orc_soap_dim(const orc_soap_hypers *h)
{
    if (h->n_compress > 0) return h->dim_out;
    int nmax = 0;
    for (int s = 0; s < h->n_species; ++s) nmax += h->alpha_max[s];
    return nmax * (nmax + 1) / 2 * (h->l_max + 1);
}

int orc_get_soap(const orc_soap_hypers *h, int n_sites, const int *n_neigh, int n_atom_pairs,
                 const unsigned char *mask, const double *rjs, const double *thetas,
                 const double *phis, double *soap, double *soap_cart_der)
{
    const int ns = h->n_species, L = h->l_max, nlm = (L + 1) * (L + 1);
    int noff[ORC_MAX_ALPHA + 1];
    int nmax = 0;
    for (int s = 0; s < ns; ++s) {
        if (h->alpha_max[s] > ORC_MAX_ALPHA) return 1;
        noff[s] = nmax;
        nmax += h->alpha_max[s];
    }
    if (L > ORC_MAX_L) return 1;
    const int D = nmax * (nmax + 1) / 2 * (L + 1);
    /* output length: the compressed one when P is given (entries outside the ranges are refused) */
    const int cmp = h->n_compress > 0;
    const int Dout = cmp ? h->dim_out : D;
    for (int e = 0; cmp && e < h->n_compress; ++e)
        if (h->compress_P_i[e] < 1 || h->compress_P_i[e] > Dout || h->compress_P_j[e] < 1 || h->compress_P_j[e] > D)
            return 1;
    radial_table *tb = make_tables(h);
    for (int s = 0; s < ns; ++s)
        if (tb[s].n <= 0) {
            free(tb);
            return 1;
        }
    int64_t *start = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n_sites + 1));
    start[0] = 0;
    for (int i = 0; i < n_sites; ++i) start[i + 1] = start[i] + n_neigh[i];
    (void)n_atom_pairs;
    const int P = n_atom_pairs;

#pragma omp parallel
    {
        double *c = (double *)malloc(sizeof(double) * (size_t)nmax * nlm);
        double *dc = (double *)malloc(sizeof(double) * 3 * (size_t)nmax * nlm);
        double *p = (double *)malloc(sizeof(double) * (size_t)D);
        double *dp = (double *)malloc(sizeof(double) * 3 * (size_t)D);
        double *pc = (double *)malloc(sizeof(double) * (size_t)Dout);
        double *dpc = (double *)malloc(sizeof(double) * 3 * (size_t)Dout);
        double *A = (double *)malloc(sizeof(double) * (size_t)nlm);
        double *dA = (double *)malloc(sizeof(double) * 3 * (size_t)nlm);
#pragma omp for schedule(dynamic, 4)
        for (int i = 0; i < n_sites; ++i) {
            memset(c, 0, sizeof(double) * (size_t)nmax * nlm);
            for (int64_t k = start[i]; k < start[i + 1]; ++k) {
                int self = (k == start[i]);
                for (int s = 0; s < ns; ++s) {
                    if (!mask[k + (int64_t)s * P]) continue;
                    double R[ORC_MAX_ALPHA];
                    if (self) {
                        radial_eval(h, s, tb + s, 0.0, 1, R, NULL);
                        for (int n = 0; n < h->alpha_max[s]; ++n)
                            c[(size_t)(noff[s] + n) * nlm] += R[n] * 0.5 / sqrt(M_PI);
                        continue;
                    }
                    double r = rjs[k];
                    if (r >= h->rcut_hard[s]) continue;
                    double u[3] = {sin(thetas[k]) * cos(phis[k]), sin(thetas[k]) * sin(phis[k]),
                                   cos(thetas[k])};
                    radial_eval(h, s, tb + s, r, 0, R, NULL);
                    angular_eval(h, s, r, u, A, NULL);
                    for (int n = 0; n < h->alpha_max[s]; ++n)
                        for (int kk = 0; kk < nlm; ++kk) c[(size_t)(noff[s] + n) * nlm + kk] += R[n] * A[kk];
                }
            }
            /* power spectrum */
            int cnt = 0;
            double nrm2 = 0.0;
            for (int n = 0; n < nmax; ++n)
                for (int np = n; np < nmax; ++np) {
                    double mult = (n == np) ? 1.0 : M_SQRT2;
                    for (int l = 0; l <= L; ++l) {
                        double acc = 0.0;
                        for (int kk = l * l; kk < (l + 1) * (l + 1); ++kk)
                            acc += c[(size_t)n * nlm + kk] * c[(size_t)np * nlm + kk];
                        p[cnt] = mult * acc;
                        nrm2 += p[cnt] * p[cnt];
                        ++cnt;
                    }
                }
            if (cmp) {
                /* P p in the order the entries are given, and its norm */
                memset(pc, 0, sizeof(double) * (size_t)Dout);
                for (int e = 0; e < h->n_compress; ++e)
                    pc[h->compress_P_i[e] - 1] += h->compress_P_el[e] * p[h->compress_P_j[e] - 1];
                nrm2 = 0.0;
                for (int d = 0; d < Dout; ++d) nrm2 += pc[d] * pc[d];
            }
            const double *pv = cmp ? pc : p;
            double nrm = sqrt(nrm2);
            double *q = soap + (size_t)i * Dout;
            for (int d = 0; d < Dout; ++d) q[d] = nrm > 0.0 ? pv[d] / nrm : 0.0;
            if (!soap_cart_der) continue;
            /* derivatives: one pair at a time (non-self), self slot = -sum */
            double *self_der = soap_cart_der + (size_t)start[i] * Dout * 3;
            memset(self_der, 0, sizeof(double) * 3 * (size_t)Dout);
            for (int64_t k = start[i] + 1; k < start[i + 1]; ++k) {
                double *out = soap_cart_der + (size_t)k * Dout * 3;
                memset(dc, 0, sizeof(double) * 3 * (size_t)nmax * nlm);
                int any = 0;
                double r = rjs[k];
                double u[3] = {sin(thetas[k]) * cos(phis[k]), sin(thetas[k]) * sin(phis[k]),
                               cos(thetas[k])};
                for (int s = 0; s < ns; ++s) {
                    if (!mask[k + (int64_t)s * P] || r >= h->rcut_hard[s]) continue;
                    double R[ORC_MAX_ALPHA], dR[ORC_MAX_ALPHA];
                    radial_eval(h, s, tb + s, r, 0, R, dR);
                    angular_eval(h, s, r, u, A, dA);
                    for (int n = 0; n < h->alpha_max[s]; ++n)
                        for (int kk = 0; kk < nlm; ++kk)
                            for (int x = 0; x < 3; ++x)
                                dc[((size_t)(noff[s] + n) * nlm + kk) * 3 + x] +=
                                    dR[n] * u[x] * A[kk] + R[n] * dA[3 * kk + x];
                    any = 1;
                }
                if (!any || nrm == 0.0) {
                    memset(out, 0, sizeof(double) * 3 * (size_t)Dout);
                    continue;
                }
                cnt = 0;
                double qdp[3] = {0.0, 0.0, 0.0};
                for (int n = 0; n < nmax; ++n)
                    for (int np = n; np < nmax; ++np) {
                        double mult = (n == np) ? 1.0 : M_SQRT2;
                        for (int l = 0; l <= L; ++l) {
                            double acc[3] = {0.0, 0.0, 0.0};
                            for (int kk = l * l; kk < (l + 1) * (l + 1); ++kk) {
                                double cn = c[(size_t)n * nlm + kk], cnp = c[(size_t)np * nlm + kk];
                                const double *dn = dc + ((size_t)n * nlm + kk) * 3;
                                const double *dnp = dc + ((size_t)np * nlm + kk) * 3;
                                for (int x = 0; x < 3; ++x) acc[x] += dn[x] * cnp + cn * dnp[x];
                            }
                            for (int x = 0; x < 3; ++x) {
                                dp[3 * cnt + x] = mult * acc[x];
                                if (!cmp) qdp[x] += q[cnt] * dp[3 * cnt + x];
                            }
                            ++cnt;
                        }
                    }
                const double *dpv = dp;
                if (cmp) {
                    memset(dpc, 0, sizeof(double) * 3 * (size_t)Dout);
                    for (int e = 0; e < h->n_compress; ++e)
                        for (int x = 0; x < 3; ++x)
                            dpc[3 * (h->compress_P_i[e] - 1) + x] +=
                                h->compress_P_el[e] * dp[3 * (h->compress_P_j[e] - 1) + x];
                    for (int d = 0; d < Dout; ++d)
                        for (int x = 0; x < 3; ++x) qdp[x] += q[d] * dpc[3 * d + x];
                    dpv = dpc;
                }
                for (int d = 0; d < Dout; ++d)
                    for (int x = 0; x < 3; ++x) {
                        double v = (dpv[3 * d + x] - q[d] * qdp[x]) / nrm;
                        out[3 * d + x] = v;
                        self_der[3 * d + x] -= v;
                    }
            }
        }
        free(c);
        free(dc);
        free(p);
        free(dp);
        free(pc);
        free(dpc);
        free(A);
        free(dA);
    }
    free(start);
    free(tb);
    return 0;
}
