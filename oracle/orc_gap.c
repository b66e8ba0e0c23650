/*
 * ORACLE — test infrastructure only (see tgap_oracle.h).
 *
 * Restatement of the GAP prediction layer and of the dynamics arithmetic:
 *   get_soap_energy_and_forces   src/gap/gap.f90:39-244
 *   get_gap_soap                 src/gap/gap_interface.f90:41-433 (subset, renumber, scatter)
 *   local_property_predict       src/gap/local_properties.f90:46-147
 *   get_2b_energy_and_forces     src/gap/gap.f90:329-460
 *   get_core_pot_energy_and_forces src/gap/gap.f90:552-686 (spline, spline_der: src/utils/splines.f90:33-156)
 *   get_3b_energy_and_forces     src/gap/gap.f90:756-1015 (cov_pp, cov_pp_der: :1022-1081)
 *   velocity_verlet              src/md/md_utils.f90:486-532
 *   monte_carlo_move             src/mc/mc_utils.f90:172-180 (+ min(1,p) of :255)
 */
#include "tgap_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static double ipow(double x, int n)
{
    double r = 1.0;
    for (int i = 0; i < n; ++i) r *= x;
    return r;
}

void orc_get_soap_energy_and_forces(int n_soap, int n_sites, int n_sparse, const double *soap,
                                    const double *soap_der, const double *alphas, double delta,
                                    double zeta0, double e0, const double *Qs,
                                    const int *n_neigh, const int *neighbors_list,
                                    const double *xyz, int do_forces, int n_sites0,
                                    double *energies, double *forces, double *virial)
{
    /* gap.f90:99-105: integer zeta if within 1e-5 */
    int is_int = fabs(zeta0 - (double)(int)zeta0) < 1.0e-5;
    int zi = (int)zeta0;
    double zeta = is_int ? (double)zi : zeta0;
    double *K = (double *)malloc(sizeof(double) * (size_t)n_sites * (size_t)n_sparse);
    /* gap.f90:123 K = soap^T Qs; K(i,s) stored K[i*n_sparse + s] */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n_sites; ++i)
        for (int s = 0; s < n_sparse; ++s) {
            const double *a = soap + (size_t)i * n_soap, *b = Qs + (size_t)s * n_soap;
            double acc = 0.0;
            for (int d = 0; d < n_soap; ++d) acc += a[d] * b[d];
            K[(size_t)i * n_sparse + s] = acc;
        }
    /* gap.f90:128-135 */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n_sites; ++i) {
        double e = 0.0;
        for (int s = 0; s < n_sparse; ++s) {
            double k = K[(size_t)i * n_sparse + s];
            e += (is_int ? ipow(k, zi) : pow(k, zeta)) * alphas[s];
        }
        energies[i] = delta * delta * e + e0;
    }
    if (!do_forces) {
        free(K);
        return;
    }
    /* gap.f90:153-171 Qss = -zeta delta^2 (K^(zeta-1) o alpha) Qs^T */
    double *Qss = (double *)malloc(sizeof(double) * (size_t)n_sites * (size_t)n_soap);
    double pref = -zeta * delta * delta;
#pragma omp parallel
    {
        double *kd = (double *)malloc(sizeof(double) * (size_t)n_sparse);
#pragma omp for schedule(static)
        for (int i = 0; i < n_sites; ++i) {
            for (int s = 0; s < n_sparse; ++s) {
                double k = K[(size_t)i * n_sparse + s];
                kd[s] = (is_int ? ipow(k, zi - 1) : pow(k, zeta - 1.0)) * alphas[s];
            }
            double *out = Qss + (size_t)i * n_soap;
            for (int d = 0; d < n_soap; ++d) out[d] = 0.0;
            for (int s = 0; s < n_sparse; ++s) {
                double w = pref * kd[s];
                const double *b = Qs + (size_t)s * n_soap;
                for (int d = 0; d < n_soap; ++d) out[d] += w * b[d];
            }
        }
        free(kd);
    }
    /* gap.f90:187-209 pair loop */
    for (int x = 0; x < 9; ++x) virial[x] = 0.0;
    for (int x = 0; x < 3 * n_sites0; ++x) forces[x] = 0.0;
    int64_t l = 0;
    for (int i = 0; i < n_sites; ++i) {
        const double *qs = Qss + (size_t)i * n_soap;
        for (int j = 0; j < n_neigh[i]; ++j, ++l) {
            int j2 = (neighbors_list[l] - 1) % n_sites0;
            double f[3];
            for (int k = 0; k < 3; ++k) {
                double acc = 0.0;
                const double *der = soap_der + (size_t)l * n_soap * 3;
                for (int d = 0; d < n_soap; ++d) acc += qs[d] * der[3 * d + k];
                f[k] = acc;
                forces[3 * j2 + k] += f[k];
            }
            const double *r = xyz + 3 * l;
            for (int k1 = 0; k1 < 3; ++k1)
                for (int k2 = 0; k2 < 3; ++k2)
                    virial[k1 + 3 * k2] += 0.5 * (f[k1] * r[k2] + f[k2] * r[k1]);
        }
    }
    free(Qss);
    free(K);
}

void orc_local_property_predict(int n_soap, int n_sites, int n_sparse, const double *soap, const double *Qs,
                                 const double *alphas, double V0, double delta, double zeta, int do_derivatives,
                                 const double *soap_cart_der, const int *n_neigh, double *V, double *V_der)
{
    /* local_properties.f90:77: integer zeta when nint(zeta) is within 1e-10 (not gap.f90's 1e-5) */
    const int zi = (int)lround(zeta);
    const int is_int = fabs((double)zi - zeta) < 1.0e-10;
    double *K = (double *)malloc(sizeof(double) * ((size_t)n_sites * (size_t)n_sparse + 1));
    /* :73-76 K = soap^T Qs */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n_sites; ++i)
        for (int s = 0; s < n_sparse; ++s) {
            const double *a = soap + (size_t)i * n_soap, *b = Qs + (size_t)s * n_soap;
            double acc = 0.0;
            for (int d = 0; d < n_soap; ++d) acc += a[d] * b[d];
            K[(size_t)i * n_sparse + s] = acc;
        }
    /* :110-122 V = delta^2 K^zeta alphas + V0, clipped at zero */
    for (int i = 0; i < n_sites; ++i) {
        double v = 0.0;
        for (int s = 0; s < n_sparse; ++s) {
            const double k = K[(size_t)i * n_sparse + s];
            v += (is_int ? ipow(k, zi) : pow(k, zeta)) * alphas[s];
        }
        v = delta * delta * v + V0;
        V[i] = v < 0.0 ? 0.0 : v;
    }
    if (do_derivatives) {
        /* :82-107, :124-142 Qss = delta^2 (zeta K^(zeta-1) o alphas) Qs^T; V_der(:, j) = Qss(i, :) .
         * soap_cart_der(:, :, j), zero for the pairs of a site whose V was clipped */
        double *qs = (double *)malloc(sizeof(double) * (size_t)n_soap);
        int64_t j = 0;
        for (int i = 0; i < n_sites; ++i) {
            for (int d = 0; d < n_soap; ++d) qs[d] = 0.0;
            for (int s = 0; s < n_sparse; ++s) {
                const double k = K[(size_t)i * n_sparse + s];
                const double kd = (is_int ? (double)zi * ipow(k, zi - 1) : zeta * pow(k, zeta - 1.0)) * alphas[s];
                const double w = delta * delta * kd;
                const double *b = Qs + (size_t)s * n_soap;
                for (int d = 0; d < n_soap; ++d) qs[d] += w * b[d];
            }
            for (int n = 0; n < n_neigh[i]; ++n, ++j)
                for (int c = 0; c < 3; ++c) {
                    double acc = 0.0;
                    if (V[i] != 0.0) {
                        const double *der = soap_cart_der + (size_t)j * n_soap * 3;
                        for (int d = 0; d < n_soap; ++d) acc += qs[d] * der[3 * d + c];
                    }
                    V_der[3 * j + c] = acc;
                }
        }
        free(qs);
    }
    free(K);
}

/* species pair test of gap.f90:381-386 */
static int pair_matches(int si, int sj, int sp1, int sp2)
{
    return (si == sp1 && sj == sp2) || (si == sp2 && sj == sp1);
}

static void virial_add_sym(double *virial, const double *f, const double *r)
{
    for (int k1 = 0; k1 < 3; ++k1)
        for (int k2 = 0; k2 < 3; ++k2) virial[k1 + 3 * k2] -= 0.5 * (f[k1] * r[k2] + f[k2] * r[k1]);
}

void orc_get_2b_energy_and_forces(int n_sites, const double *rjs, const double *xyz, int n_sparse,
                                  const double *alphas, const double *cutoff, double rcut, double buffer,
                                  double delta, double sigma, double e0, const double *Qs, const int *n_neigh,
                                  int do_forces, const int *species, const int *neighbor_species, int sp1, int sp2,
                                  int n_sites0, double *energies, double *forces, double *virial)
{
    const double pi = acos(-1.0);
    /* :374-402 energies */
    for (int i = 0; i < n_sites; ++i) energies[i] = e0;
    int64_t k = 0;
    for (int i = 0; i < n_sites; ++i) {
        if (species[i] != sp1 && species[i] != sp2) {
            k += n_neigh[i];
            continue;
        }
        ++k;
        for (int j = 1; j < n_neigh[i]; ++j, ++k) {
            if (!pair_matches(species[i], neighbor_species[k], sp1, sp2)) continue;
            const double r = rjs[k];
            if (!(r < rcut)) continue;
            const double fcut = r < rcut - buffer ? 1.0 : (cos(pi * (r - rcut + buffer) / buffer) + 1.0) / 2.0;
            for (int s = 0; s < n_sparse; ++s)
                energies[i] += delta * delta * alphas[s] * cutoff[s] * fcut *
                               exp(-0.5 * (r - Qs[s]) * (r - Qs[s]) / (sigma * sigma));
        }
    }
    if (!do_forces) return;
    /* :405-445 forces on the site, then half of the pair virial */
    for (int x = 0; x < 3 * n_sites0; ++x) forces[x] = 0.0;
    for (int x = 0; x < 9; ++x) virial[x] = 0.0;
    k = 0;
    for (int i = 0; i < n_sites; ++i) {
        if (species[i] != sp1 && species[i] != sp2) {
            k += n_neigh[i];
            continue;
        }
        ++k;
        for (int j = 1; j < n_neigh[i]; ++j, ++k) {
            if (!pair_matches(species[i], neighbor_species[k], sp1, sp2)) continue;
            const double r = rjs[k];
            if (!(r < rcut)) continue;
            double fcut, dfcut;
            if (r < rcut - buffer) {
                fcut = 1.0;
                dfcut = 0.0;
            } else {
                fcut = (cos(pi * (r - rcut + buffer) / buffer) + 1.0) / 2.0;
                dfcut = pi / 2.0 / buffer * sin(pi * (r - rcut + buffer) / buffer);
            }
            for (int s = 0; s < n_sparse; ++s) {
                double f[3];
                const double g = -2.0 * delta * delta * alphas[s] * cutoff[s] *
                                 exp(-0.5 * (r - Qs[s]) * (r - Qs[s]) / (sigma * sigma));
                const double h = (r - Qs[s]) / (sigma * sigma) * fcut + dfcut;
                for (int c = 0; c < 3; ++c) f[c] = g * xyz[3 * k + c] / r * h;
                for (int c = 0; c < 3; ++c) forces[3 * i + c] += f[c];
                virial_add_sym(virial, f, xyz + 3 * k);
            }
        }
    }
    for (int x = 0; x < 9; ++x) virial[x] *= 0.5;
}

/* splines.f90:33-105 (one point) */
static double spline_at(int n, const double *x, const double *y, const double *y2, double yp1, double ypn,
                        double r)
{
    if (r < x[0]) return y[0] + (r - x[0]) * yp1;
    if (r > x[n - 1]) return y[n - 1] + (r - x[n - 1]) * ypn;
    int j = 0;
    while (j < n - 2 && !(r < x[j + 1])) ++j;
    const double h = x[j + 1] - x[j], h26 = h * h / 6.0;
    const double A = (x[j + 1] - r) / h, B = 1.0 - A;
    const double C = (A * A * A - A) * h26, D = (B * B * B - B) * h26;
    return A * y[j] + B * y[j + 1] + C * y2[j] + D * y2[j + 1];
}

/* splines.f90:107-156 (one point) */
static double spline_der_at(int n, const double *x, const double *y, const double *y2, double yp1, double ypn,
                            double r)
{
    if (r < x[0]) return yp1;
    if (r > x[n - 1]) return ypn;
    int j = 0;
    while (j < n - 2 && !(r < x[j + 1])) ++j;
    const double h = x[j + 1] - x[j], h6 = h / 6.0;
    const double A = (x[j + 1] - r) / h, B = 1.0 - A;
    const double dAdx = -1.0 / h, dBdx = -dAdx;
    const double dCdx = (1.0 - 3.0 * A * A) * h6, dDdx = (3.0 * B * B - 1.0) * h6;
    return dAdx * y[j] + dBdx * y[j + 1] + dCdx * y2[j] + dDdx * y2[j + 1];
}

void orc_get_core_pot_energy_and_forces(int n_sparse, int n_sites, int n_sites0, const double *rjs,
                                        const double *xyz, const double *x, const double *V, double yp1,
                                        double ypn, const double *dVdx2, const int *n_neigh, int do_forces,
                                        const int *species, const int *neighbor_species, int sp1, int sp2,
                                        double *energies, double *forces, double *virial)
{
    double rcut = x[0];
    for (int s = 1; s < n_sparse; ++s) rcut = x[s] > rcut ? x[s] : rcut; /* :593 maxval(x) */
    for (int i = 0; i < n_sites; ++i) energies[i] = 0.0;
    int64_t k = 0;
    for (int i = 0; i < n_sites; ++i) {
        if (species[i] != sp1 && species[i] != sp2) {
            k += n_neigh[i];
            continue;
        }
        ++k;
        for (int j = 1; j < n_neigh[i]; ++j, ++k) {
            if (!pair_matches(species[i], neighbor_species[k], sp1, sp2)) continue;
            if (rjs[k] < rcut) energies[i] += 0.5 * spline_at(n_sparse, x, V, dVdx2, yp1, ypn, rjs[k]);
        }
    }
    if (!do_forces) return;
    for (int q = 0; q < 3 * n_sites0; ++q) forces[q] = 0.0;
    for (int q = 0; q < 9; ++q) virial[q] = 0.0;
    k = 0;
    for (int i = 0; i < n_sites; ++i) {
        if (species[i] != sp1 && species[i] != sp2) {
            k += n_neigh[i];
            continue;
        }
        ++k;
        for (int j = 1; j < n_neigh[i]; ++j, ++k) {
            if (!pair_matches(species[i], neighbor_species[k], sp1, sp2)) continue;
            if (!(rjs[k] < rcut)) continue;
            const double dv = spline_der_at(n_sparse, x, V, dVdx2, yp1, ypn, rjs[k]);
            double f[3];
            for (int c = 0; c < 3; ++c) f[c] = dv * xyz[3 * k + c] / rjs[k];
            for (int c = 0; c < 3; ++c) forces[3 * i + c] += f[c];
            virial_add_sym(virial, f, xyz + 3 * k);
        }
    }
    for (int q = 0; q < 9; ++q) virial[q] *= 0.5;
}

/* cov_pp / cov_pp_der (gap.f90:1022-1081) for d = 3, q = 1: j = 3 */
static double cov_pp31(double r)
{
    if (r >= 1.0) return 0.0;
    if (r <= 0.0) return 1.0;
    return pow(1.0 - r, 4) * (4.0 * r + 1.0);
}

static double cov_pp31_der(double r) /* includes the 1/r factor */
{
    if (r >= 1.0 || r <= 0.0) return 0.0;
    return (-4.0 * pow(1.0 - r, 3) * (4.0 * r + 1.0) + pow(1.0 - r, 4) * 4.0) / r;
}

void orc_get_3b_energy_and_forces(int n_sites0, int n_sites, const double *rjs, const double *xyz, int n_sparse,
                                  const double *alphas, const double *cutoff, double rcut, double buffer,
                                  double delta, const double *sigma, double e0, const double *Qs,
                                  const int *n_neigh, const int *neighbors_list, int do_forces, int kernel_pol,
                                  const int *species, const int *neighbor_species, int sp0, int sp1, int sp2,
                                  double *energies, double *forces, double *virial)
{
    const double pi = acos(-1.0);
    double *pref = (double *)malloc(sizeof(double) * (size_t)n_sparse);
    double *rr = (double *)malloc(sizeof(double) * (size_t)n_sparse);
    double *kern = (double *)malloc(sizeof(double) * (size_t)n_sparse);
    double *kder = (double *)malloc(sizeof(double) * (size_t)n_sparse);
    double *drdq = (double *)malloc(sizeof(double) * 3 * (size_t)n_sparse);
    for (int s = 0; s < n_sparse; ++s) pref[s] = 2.0 * delta * delta * alphas[s] * cutoff[s]; /* :829 */
    for (int i = 0; i < n_sites; ++i) energies[i] = e0;
    if (do_forces) {
        for (int x = 0; x < 3 * n_sites0; ++x) forces[x] = 0.0;
        for (int x = 0; x < 9; ++x) virial[x] = 0.0;
    }
    int64_t k = 0;
    for (int i = 0; i < n_sites; ++i) {
        if (species[i] != sp0) {
            k += n_neigh[i];
            continue;
        }
        const int i3 = (neighbors_list[k] - 1) % n_sites0;
        ++k;
        for (int j = 1; j < n_neigh[i]; ++j, ++k) {
            const double r12 = rjs[k];
            if ((neighbor_species[k] != sp1 && neighbor_species[k] != sp2) || r12 > rcut) continue;
            const int j3 = (neighbors_list[k] - 1) % n_sites0;
            const double *x12 = xyz + 3 * k;
            double x12r[3];
            for (int c = 0; c < 3; ++c) x12r[c] = x12[c] / r12;
            int64_t k2 = k;
            for (int j2 = j + 1; j2 < n_neigh[i]; ++j2) {
                ++k2;
                const double r13 = rjs[k2];
                const int ok = ((neighbor_species[k] == sp1 && neighbor_species[k2] == sp2) ||
                                (neighbor_species[k] == sp2 && neighbor_species[k2] == sp1)) &&
                               r13 < rcut;
                if (!ok) continue;
                const int k3 = (neighbors_list[k2] - 1) % n_sites0;
                const double *x13 = xyz + 3 * k2;
                double x13r[3], x23[3], x23r[3];
                for (int c = 0; c < 3; ++c) {
                    x13r[c] = x13[c] / r13;
                    x23[c] = x13[c] - x12[c];
                }
                const double r23 = sqrt(x23[0] * x23[0] + x23[1] * x23[1] + x23[2] * x23[2]);
                for (int c = 0; c < 3; ++c) x23r[c] = x23[c] / r23;
                if (!(r12 < rcut && r13 < rcut)) continue;
                double fcut12, fcut13, dfcut12[3], dfcut13[3];
                if (r12 < rcut - buffer) {
                    fcut12 = 1.0;
                    dfcut12[0] = dfcut12[1] = dfcut12[2] = 0.0;
                } else {
                    fcut12 = (cos(pi * (r12 - rcut + buffer) / buffer) + 1.0) / 2.0;
                    for (int c = 0; c < 3; ++c)
                        dfcut12[c] = sin(pi * (r12 - rcut + buffer) / buffer) / 2.0 * pi / buffer * x12r[c];
                }
                if (r13 < rcut - buffer) {
                    fcut13 = 1.0;
                    dfcut13[0] = dfcut13[1] = dfcut13[2] = 0.0;
                } else {
                    fcut13 = (cos(pi * (r13 - rcut + buffer) / buffer) + 1.0) / 2.0;
                    for (int c = 0; c < 3; ++c)
                        dfcut13[c] = sin(pi * (r13 - rcut + buffer) / buffer) / 2.0 * pi / buffer * x13r[c];
                }
                const double fcut = fcut12 * fcut13;
                double dfcut[3];
                for (int c = 0; c < 3; ++c) dfcut[c] = fcut12 * dfcut13[c] + fcut13 * dfcut12[c];
                const double q[3] = {r12 + r13, (r12 - r13) * (r12 - r13), r23};
                for (int s = 0; s < n_sparse; ++s) {
                    double a = 0.0;
                    for (int c = 0; c < 3; ++c) {
                        const double dq = q[c] - Qs[s + (size_t)c * n_sparse];
                        a += dq * dq / (sigma[c] * sigma[c]);
                        drdq[3 * s + c] = dq / (sigma[c] * sigma[c]);
                    }
                    rr[s] = sqrt(a);
                    kern[s] = kernel_pol ? pref[s] * cov_pp31(rr[s]) : pref[s] * exp(-0.5 * rr[s] * rr[s]);
                    if (kernel_pol) kder[s] = pref[s] * cov_pp31_der(rr[s]);
                }
                double ksum = 0.0;
                for (int s = 0; s < n_sparse; ++s) ksum += kern[s];
                energies[i] += fcut * ksum;
                if (!do_forces) continue;
                double f1[3], f2[3], f3[3];
                for (int l = 0; l < 3; ++l) {
                    double s1 = 0.0, s2 = 0.0, s3 = 0.0;
                    for (int s = 0; s < n_sparse; ++s) {
                        const double *d = drdq + 3 * s;
                        const double dx1 = d[0] * (x12r[l] + x13r[l]) + d[1] * 2.0 * (r12 - r13) * (x12r[l] - x13r[l]);
                        const double dx2 = -d[0] * x12r[l] - d[1] * 2.0 * (r12 - r13) * x12r[l] + d[2] * x23r[l];
                        const double dx3 = -d[0] * x13r[l] - d[1] * 2.0 * (r13 - r12) * x13r[l] - d[2] * x23r[l];
                        if (kernel_pol) {
                            s1 += kern[s] * dfcut[l] - kder[s] * fcut * dx1;
                            s2 += -kern[s] * fcut13 * dfcut12[l] - kder[s] * fcut * dx2;
                            s3 += -kern[s] * fcut12 * dfcut13[l] - kder[s] * fcut * dx3;
                        } else {
                            s1 += kern[s] * (dfcut[l] + fcut * dx1);
                            s2 += kern[s] * (-fcut13 * dfcut12[l] + fcut * dx2);
                            s3 += kern[s] * (-fcut12 * dfcut13[l] + fcut * dx3);
                        }
                    }
                    f1[l] = -s1;
                    f2[l] = -s2;
                    f3[l] = -s3;
                }
                for (int c = 0; c < 3; ++c) {
                    forces[3 * i3 + c] += f1[c];
                    forces[3 * j3 + c] += f2[c];
                    forces[3 * k3 + c] += f3[c];
                }
                for (int a1 = 0; a1 < 3; ++a1)
                    for (int a2 = 0; a2 < 3; ++a2) {
                        virial[a1 + 3 * a2] += 0.5 * (f2[a1] * x12[a2] + f2[a2] * x12[a1]);
                        virial[a1 + 3 * a2] += 0.5 * (f3[a1] * x13[a2] + f3[a2] * x13[a1]);
                    }
            }
        }
    }
    free(pref);
    free(rr);
    free(kern);
    free(kder);
    free(drdq);
}

int orc_get_gap_soap(const orc_soap_hypers *h, int n_total_sites, int n_sites0,
                     const int *n_neigh0, const int *neighbors_list0, const double *rjs0,
                     const double *thetas0, const double *phis0, const double *xyz0,
                     const int *species_supercell, int central_species, int n_sparse,
                     const double *alphas, const double *Qs, double delta, double zeta,
                     int do_forces, double *energies0, double *forces0, double *virial)
{
    const int ns = h->n_species;
    double rcut_max = 0.0;
    for (int s = 0; s < ns; ++s)
        if (h->rcut_hard[s] > rcut_max) rcut_max = h->rcut_hard[s];
    /* gap_interface.f90:184-212: count kept sites and pairs */
    int n_sites = 0;
    int64_t n_pairs = 0, k = 0;
    unsigned char *seen = (unsigned char *)calloc((size_t)n_total_sites, 1);
    for (int i = 0; i < n_sites0; ++i) {
        int sp_i = species_supercell[(neighbors_list0[k] - 1) % n_total_sites];
        if (sp_i == central_species || central_species == 0) {
            ++n_sites;
            for (int j = 0; j < n_neigh0[i]; ++j, ++k) {
                int j2 = (neighbors_list0[k] - 1) % n_total_sites;
                if (rjs0[k] < rcut_max && species_supercell[j2] > 0) {
                    ++n_pairs;
                    seen[j2] = 1;
                }
            }
        } else {
            k += n_neigh0[i];
        }
    }
    int n_all = 0;
    for (int i = 0; i < n_total_sites; ++i) n_all += seen[i];
    /* gap_interface.f90:215-289: build the subset and renumber */
    int *n_neigh = (int *)malloc(sizeof(int) * (size_t)(n_sites > 0 ? n_sites : 1));
    int *nl = (int *)malloc(sizeof(int) * (size_t)(n_pairs > 0 ? n_pairs : 1));
    double *rjs = (double *)malloc(sizeof(double) * (size_t)(n_pairs > 0 ? n_pairs : 1));
    double *th = (double *)malloc(sizeof(double) * (size_t)(n_pairs > 0 ? n_pairs : 1));
    double *ph = (double *)malloc(sizeof(double) * (size_t)(n_pairs > 0 ? n_pairs : 1));
    double *xyz = (double *)malloc(sizeof(double) * 3 * (size_t)(n_pairs > 0 ? n_pairs : 1));
    unsigned char *mask = (unsigned char *)calloc((size_t)(n_pairs > 0 ? n_pairs : 1) * ns, 1);
    int *in_to_out = (int *)calloc((size_t)(n_all > 0 ? n_all : 1), sizeof(int));
    int *out_to_in = (int *)calloc((size_t)n_total_sites, sizeof(int));
    int i2 = 0;
    k = 0;
    for (int i = 0; i < n_sites0; ++i) {
        int j = (neighbors_list0[k] - 1) % n_total_sites;
        int sp_i = species_supercell[j];
        if (sp_i == central_species || central_species == 0) {
            in_to_out[i2] = j + 1;
            out_to_in[j] = i2 + 1;
            ++i2;
        }
        k += n_neigh0[i];
    }
    k = 0;
    i2 = 0;
    int i4 = 0;
    int64_t k2 = 0;
    for (int i = 0; i < n_sites0; ++i) {
        int sp_i = species_supercell[(neighbors_list0[k] - 1) % n_total_sites];
        if (sp_i == central_species || central_species == 0) {
            ++i2;
            int jj = 0;
            for (int j = 1; j <= n_neigh0[i]; ++j, ++k) {
                int j3 = (neighbors_list0[k] - 1) % n_total_sites;
                if (rjs0[k] < rcut_max && species_supercell[j3] > 0) {
                    ++jj;
                    rjs[k2] = rjs0[k];
                    ph[k2] = phis0[k];
                    th[k2] = thetas0[k];
                    xyz[3 * k2] = xyz0[3 * k];
                    xyz[3 * k2 + 1] = xyz0[3 * k + 1];
                    xyz[3 * k2 + 2] = xyz0[3 * k + 2];
                    mask[k2 + (int64_t)(species_supercell[j3] - 1) * n_pairs] = 1;
                    if (j > 1 && out_to_in[j3] == 0) {
                        ++i4;
                        in_to_out[n_sites + i4 - 1] = j3 + 1;
                        out_to_in[j3] = n_sites + i4;
                        nl[k2] = out_to_in[j3];
                    } else if (j > 1) {
                        nl[k2] = out_to_in[j3];
                    } else {
                        nl[k2] = i2;
                    }
                    ++k2;
                }
            }
            n_neigh[i2 - 1] = jj;
        } else {
            k += n_neigh0[i];
        }
    }
    int D = orc_soap_dim(h);
    int rc = 0;
    double *soap = (double *)calloc((size_t)D * (size_t)(n_sites > 0 ? n_sites : 1), sizeof(double));
    double *der = NULL;
    if (do_forces) der = (double *)calloc((size_t)D * 3 * (size_t)(n_pairs > 0 ? n_pairs : 1), sizeof(double));
    for (int x = 0; x < 9; ++x) virial[x] = 0.0;
    if (n_sites > 0) {
        rc = orc_get_soap(h, n_sites, n_neigh, (int)n_pairs, mask, rjs, th, ph, soap, der);
        if (rc == 0) {
            double *en = (double *)calloc((size_t)n_sites, sizeof(double));
            double *fo = (double *)calloc((size_t)3 * (size_t)n_all, sizeof(double));
            orc_get_soap_energy_and_forces(D, n_sites, n_sparse, soap, der, alphas, delta, zeta, 0.0,
                                           Qs, n_neigh, nl, xyz, do_forces, n_all, en, fo, virial);
            for (int i = 0; i < n_sites; ++i) energies0[in_to_out[i] - 1] = en[i];
            if (do_forces)
                for (int i = 0; i < n_all; ++i)
                    for (int x = 0; x < 3; ++x) forces0[3 * (in_to_out[i] - 1) + x] = fo[3 * i + x];
            free(en);
            free(fo);
        }
    }
    free(soap);
    free(der);
    free(seen);
    free(n_neigh);
    free(nl);
    free(rjs);
    free(th);
    free(ph);
    free(xyz);
    free(mask);
    free(in_to_out);
    free(out_to_in);
    return rc;
}

void orc_velocity_verlet(int n_sites, double *positions, double *positions_prev,
                         double *velocities, const double *forces, double *forces_prev,
                         const double *masses, double dt, double *dt_prev, int first_step)
{
    if (!first_step)
        for (int i = 0; i < n_sites; ++i)
            for (int j = 0; j < 3; ++j)
                velocities[3 * i + j] = velocities[3 * i + j] +
                                        0.5 * (forces[3 * i + j] + forces_prev[3 * i + j]) /
                                            masses[i] * *dt_prev;
    memcpy(positions_prev, positions, sizeof(double) * 3 * (size_t)n_sites);
    memcpy(forces_prev, forces, sizeof(double) * 3 * (size_t)n_sites);
    for (int i = 0; i < n_sites; ++i)
        for (int j = 0; j < 3; ++j)
            positions[3 * i + j] = positions[3 * i + j] + velocities[3 * i + j] * dt +
                                   0.5 * forces[3 * i + j] / masses[i] * (dt * dt);
    *dt_prev = dt;
}

double orc_mc_move_acceptance(double e_new, double e_prev, double temp)
{
    const double kB = (double)(float)8.617333262e-5;
    double p = exp(-(e_new - e_prev) / (kB * temp));
    return p < 1.0 ? p : 1.0;
}

/* calculate_e0 (src/gap/calculate_gap_soap.f90:135-169): for every site, the loop over
 * j = 1..n_species sets energies_e0(i) = e0(j) when the site's species is species_types(j);
 * species are channel ids here (1..n_species), so the match is species(i) == j. Sites of no
 * listed species keep the value they had (zero after reset, calculation.f90:234-235). */
void orc_calculate_e0(int n_sites, const int *species, int n_species, const double *e0, double *energies_e0)
{
    for (int i = 0; i < n_sites; ++i)
        for (int j = 1; j <= n_species; ++j)
            if (species[i] == j) energies_e0[i] = e0[j - 1];
}
