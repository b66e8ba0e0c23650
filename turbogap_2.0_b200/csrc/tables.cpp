// Host-side set-up of the descriptor tables (compiled by the host C++ compiler; uses
// binary128 where the poly3 basis is ill-conditioned).
//
// The poly3 radial basis of soap_turbo (basis keyword, src/gap/read_gap.f90:274-284) is
// phi_a(x) = sqrt(2a+5) (1-x)^(a+2), a = 1..alpha_max, on x = r / rcut_hard in [0, 1],
// orthonormalised with W = S^{-1/2}, S_ab = sqrt((2a+5)(2b+5)) / (a+b+5). lambda_min(S) is
// ~6e-13 for alpha_max = 8, so W is computed here in binary128 (coupled Newton-Schulz
// iteration) and the orthonormal functions are tabulated at Gauss-Legendre nodes; kernels
// then integrate each neighbor's smeared density against the table, which keeps FP64 and
// FP32 evaluations well conditioned.
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <string>
#include <vector>

#include "tgap_internal.h"

namespace tgap {

typedef __float128 f128;

static f128 sqrt128(f128 x)
{
    if (x <= 0) return 0;
    f128 y = (f128)std::sqrt((double)x);
    for (int i = 0; i < 4; ++i) y = 0.5Q * (y + x / y);
    return y;
}

static void matmul128(int n, const f128 *A, const f128 *B, f128 *C)
{
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            f128 s = 0;
            for (int k = 0; k < n; ++k) s += A[i * n + k] * B[k * n + j];
            C[i * n + j] = s;
        }
}

// W = S^{-1/2} by the coupled Newton-Schulz iteration on S / c (c >= lambda_max):
// Y -> (S/c)^{1/2}, Z -> (S/c)^{-1/2}; W = Z / sqrt(c).
static void inv_sqrt_newton_schulz(int n, const f128 *S, f128 *W)
{
    std::vector<f128> Y(n * n), Z(n * n), T(n * n), U(n * n), V(n * n);
    f128 c = 0;  // Frobenius norm bounds lambda_max
    for (int i = 0; i < n * n; ++i) c += S[i] * S[i];
    c = sqrt128(c);
    for (int i = 0; i < n * n; ++i) {
        Y[i] = S[i] / c;
        Z[i] = (i / n == i % n) ? 1 : 0;
    }
    for (int it = 0; it < 400; ++it) {
        matmul128(n, Z.data(), Y.data(), T.data());
        f128 dev = 0;
        for (int i = 0; i < n * n; ++i) {
            f128 id = (i / n == i % n) ? 1 : 0;
            f128 d = T[i] - id;
            dev += d * d;
            T[i] = 0.5Q * (3 * id - T[i]);
        }
        matmul128(n, Y.data(), T.data(), U.data());
        matmul128(n, T.data(), Z.data(), V.data());
        Y.swap(U);
        Z.swap(V);
        if (dev < (f128)1e-60Q) break;
    }
    f128 s = 1 / sqrt128(c);
    for (int i = 0; i < n * n; ++i) W[i] = Z[i] * s;
}

void poly3_orthonormaliser(int am, double *W)
{
    std::vector<f128> S(am * am), Wq(am * am);
    for (int a = 1; a <= am; ++a)
        for (int b = 1; b <= am; ++b)
            S[(a - 1) * am + b - 1] = sqrt128((f128)((2 * a + 5) * (2 * b + 5))) / (f128)(a + b + 5);
    inv_sqrt_newton_schulz(am, S.data(), Wq.data());
    for (int i = 0; i < am * am; ++i) W[i] = (double)Wq[i];
}

// Gauss-Legendre rule on [-1, 1] (Newton iteration in binary128 from the Tricomi guess).
static void gauss_legendre128(int n, double *t, double *w)
{
    const double pi = 3.14159265358979323846;
    for (int i = 0; i < n; ++i) {
        f128 z = (f128)std::cos(pi * (4.0 * i + 3.0) / (4.0 * n + 2.0));
        f128 dp = 1;
        for (int it = 0; it < 60; ++it) {
            f128 p0 = 1, p1 = z;
            for (int k = 2; k <= n; ++k) {
                f128 p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            if (n == 1) { p1 = z; p0 = 1; }
            dp = n * (z * p1 - p0) / (z * z - 1);
            f128 dz = p1 / dp;
            z -= dz;
            f128 adz = dz < 0 ? -dz : dz;
            if (adz < (f128)1e-32Q) break;
        }
        t[n - 1 - i] = (double)z;
        w[n - 1 - i] = (double)(2 / ((1 - z * z) * dp * dp));
    }
}

static int up4(int v) { return (v + 3) / 4 * 4; }
static int clamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

int make_soap_params(const tgap_soap_hypers *h, SoapParams *p, std::string *why)
{
    std::memset(p, 0, sizeof(*p));
    if (!h || h->n_species < 1 || h->n_species > kMaxSpecies) {
        *why = "n_species must be in 1.." + std::to_string(kMaxSpecies);
        return TGAP_ERR_HYPERS;
    }
    if (h->l_max < 0 || h->l_max > kMaxL) {
        *why = "l_max must be in 0.." + std::to_string(kMaxL);
        return TGAP_ERR_HYPERS;
    }
    if (h->radial_enhancement < 0 || h->radial_enhancement > 2) {
        *why = "radial_enhancement must be 0, 1 or 2";
        return TGAP_ERR_HYPERS;
    }
    p->n_species = h->n_species;
    p->l_max = h->l_max;
    p->radial_enhancement = h->radial_enhancement;
    int nmax = 0, nodes = 0, tq_total = 0;
    for (int s = 0; s < h->n_species; ++s) {
        int am = h->alpha_max[s];
        if (am < 1 || am > kMaxAlpha) {
            *why = "alpha_max must be in 1.." + std::to_string(kMaxAlpha);
            return TGAP_ERR_HYPERS;
        }
        double rc = h->rcut_hard[s], rs = h->rcut_soft[s];
        if (!(rc > 0) || !(rs > 0) || rs > rc || !(h->atom_sigma_r[s] > 0) ||
            !(h->atom_sigma_t[s] > 0) || h->atom_sigma_r_scaling[s] < 0 ||
            h->atom_sigma_t_scaling[s] < 0 || !(h->nf[s] > 0) || h->amplitude_scaling[s] < 0) {
            *why = "invalid radial/angular settings for species " + std::to_string(s + 1);
            return TGAP_ERR_HYPERS;
        }
        p->alpha_max[s] = am;
        p->n_off[s] = nmax;
        nmax += am;
        p->rcut_hard[s] = rc;
        p->rcut_soft[s] = rs;
        p->nf[s] = h->nf[s];
        p->global_scaling[s] = h->global_scaling[s];
        p->sigma_r[s] = h->atom_sigma_r[s];
        p->sigma_r_scaling[s] = h->atom_sigma_r_scaling[s];
        p->sigma_t[s] = h->atom_sigma_t[s];
        p->sigma_t_scaling[s] = h->atom_sigma_t_scaling[s];
        p->amplitude_scaling[s] = h->amplitude_scaling[s];
        p->central_weight[s] = h->central_weight[s];
        if (rc > p->rcut_max) p->rcut_max = rc;
        // node-count rule (shared with the oracle): ~4.5 nodes per Gaussian width
        double xs = rs / rc, sig0 = h->atom_sigma_r[s] / rc;
        int n_in = up4(clamp((int)std::ceil(4.5 * xs / sig0), 24, 128));
        int n_buf = 0;
        if (xs < 1.0) {
            double sf = (1.0 - xs) / h->nf[s];
            double sc = sig0 * sf / std::sqrt(sig0 * sig0 + sf * sf);
            n_buf = up4(clamp((int)std::ceil(4.5 * (1.0 - xs) / sc), 16, 64));
        }
        p->n_nodes[s] = n_in + n_buf;
        p->node_off[s] = nodes;
        p->tq_off[s] = tq_total;
        tq_total += (n_in + n_buf) * am;
        if (am > p->max_alpha) p->max_alpha = am;
        nodes += n_in + n_buf;
        if (n_in + n_buf > kMaxNodes) {
            *why = "too many quadrature nodes";
            return TGAP_ERR_HYPERS;
        }
    }
    if (nmax > kMaxNmax) {
        *why = "sum of alpha_max must be <= " + std::to_string(kMaxNmax);
        return TGAP_ERR_HYPERS;
    }
    p->n_max = nmax;
    p->dim = nmax * (nmax + 1) / 2 * (h->l_max + 1);
    p->dim_out = p->dim;
    p->cmp_row = p->cmp_rcol = p->cmp_col = p->cmp_crow = nullptr;
    p->cmp_rval = p->cmp_cval = nullptr;
    p->cmp_rval32 = p->cmp_cval32 = nullptr;
    for (int s = 0; s < h->n_species; ++s) p->tab_scale[s] = (double)kTabIntervals / p->rcut_hard[s];
    p->am_pad = up4(p->max_alpha);
    return TGAP_OK;
}

int build_soap_tables(const SoapParams &p, SoapTables *t)
{
    int total_nodes = 0, tq_len = 0;
    for (int s = 0; s < p.n_species; ++s) {
        total_nodes += p.n_nodes[s];
        tq_len += p.n_nodes[s] * p.alpha_max[s];
    }
    t->xq.assign(total_nodes, 0.0);
    t->tq.assign(tq_len, 0.0);
    t->central.assign(p.n_max, 0.0);
    int tq_off = 0;
    for (int s = 0; s < p.n_species; ++s) {
        const int am = p.alpha_max[s];
        std::vector<double> Wd(am * am);
        // W in binary128 (rounded copy kept for reference; the table uses the full value)
        std::vector<f128> S(am * am), W(am * am);
        for (int a = 1; a <= am; ++a)
            for (int b = 1; b <= am; ++b)
                S[(a - 1) * am + b - 1] = sqrt128((f128)((2 * a + 5) * (2 * b + 5))) / (f128)(a + b + 5);
        inv_sqrt_newton_schulz(am, S.data(), W.data());
        const double rc = p.rcut_hard[s];
        const double xs = p.rcut_soft[s] / rc;
        const double sig0 = p.sigma_r[s] / rc;
        int n_in = 0, n_buf = 0;
        {
            n_in = up4(clamp((int)std::ceil(4.5 * xs / sig0), 24, 128));
            n_buf = p.n_nodes[s] - n_in;
        }
        const double sf = (1.0 - xs) / p.nf[s];
        std::vector<double> gt(128), gw(128);
        for (int part = 0; part < 2; ++part) {
            int m = part == 0 ? n_in : n_buf;
            if (m <= 0) continue;
            double lo = part == 0 ? 0.0 : xs, hi = part == 0 ? xs : 1.0;
            gauss_legendre128(m, gt.data(), gw.data());
            for (int i = 0; i < m; ++i) {
                int q = (part == 0 ? i : n_in + i);
                double x = lo + (hi - lo) * (gt[i] + 1.0) * 0.5;
                double wx = gw[i] * (hi - lo) * 0.5;
                double filt = part == 0 ? 1.0 : std::exp(-(x - xs) * (x - xs) / (2.0 * sf * sf));
                t->xq[p.node_off[s] + q] = x;
                f128 om = 1 - (f128)x;
                for (int n = 0; n < am; ++n) {
                    f128 acc = 0, pw = om * om;
                    for (int a = 1; a <= am; ++a) {
                        pw *= om;
                        acc += W[n * am + a - 1] * sqrt128((f128)(2 * a + 5)) * pw;
                    }
                    t->tq[tq_off + q * am + n] = (double)(acc * (f128)wx * (f128)filt);
                }
            }
        }
        // central-atom coefficients: R_n(0) * global_scaling * central_weight * Y_00
        double sig = sig0, A = 1.0 / sig;  // (1 + 2x^3 - 3x^2)^a = 1 at x = 0
        if (p.radial_enhancement == 1) A *= std::sqrt(2.0 / M_PI) * sig;
        if (p.radial_enhancement == 2) A *= sig * sig;
        for (int n = 0; n < am; ++n) {
            double acc = 0.0;
            for (int q = 0; q < p.n_nodes[s]; ++q) {
                double u = t->xq[p.node_off[s] + q];
                acc += t->tq[tq_off + q * am + n] * std::exp(-u * u / (2.0 * sig * sig));
            }
            t->central[p.n_off[s] + n] =
                p.global_scaling[s] * p.central_weight[s] * A * acc * 0.28209479177387814;
        }
        tq_off += p.n_nodes[s] * am;
    }
    return TGAP_OK;
}

}  // namespace tgap

extern "C" int tgap_debug_poly3_w(int alpha_max, double *W)
{
    if (alpha_max < 1 || alpha_max > tgap::kMaxAlpha || !W) return TGAP_ERR_ARGUMENT;
    tgap::poly3_orthonormaliser(alpha_max, W);
    return TGAP_OK;
}
