/*
 * ORACLE — test infrastructure only (see tgap_oracle.h).
 *
 * Restatement of the TurboGAP neighbor-list builder:
 *   build_neighbors_list          src/neighbors/neighbors_interface.f90:144-524
 *   get_distance                  src/neighbors/neighbors_interface.f90:547-643
 *   number_of_unit_cells_...      src/neighbors/neighbors_interface.f90:655-708
 *   set_supercell                 src/xyz/read_xyz.f90:323-373
 *
 * Floating-point expressions keep the Fortran evaluation order (left to right, no fused
 * multiply-add: build with -ffp-contract=off) so that the pair list is reproduced bit for
 * bit. Real MODULO follows gfortran (fmod, then add P when the signs differ).
 */
#include "tgap_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static double f_modulo(double a, double p)
{
    double r = fmod(a, p);
    if (r != 0.0 && ((r < 0.0) != (p < 0.0))) r = r + p;
    return r;
}

static int i_modulo(int a, int m)
{
    int r = a % m;
    if (r != 0 && ((r < 0) != (m < 0))) r += m;
    return r;
}

static double dot3(const double *x, const double *y)
{
    double s = 0.0;
    s = s + x[0] * y[0];
    s = s + x[1] * y[1];
    s = s + x[2] * y[2];
    return s;
}

static int is_orthorhombic(const double a[3], const double b[3], const double c[3])
{
    const double d_tol = 1.0e-6;
    return fabs(a[1]) < d_tol && fabs(a[2]) < d_tol && fabs(b[0]) < d_tol &&
           fabs(b[2]) < d_tol && fabs(c[0]) < d_tol && fabs(c[1]) < d_tol;
}

/* neighbors_interface.f90:582-614: inverse of the lattice Gram matrix (cofactor form). */
static void gram_inverse(const double a[3], const double b[3], const double c[3], double inv[3][3])
{
    double m[3][3];
    m[0][0] = dot3(a, a);
    m[0][1] = dot3(a, b);
    m[0][2] = dot3(a, c);
    m[1][0] = m[0][1];
    m[1][1] = dot3(b, b);
    m[1][2] = dot3(b, c);
    m[2][0] = m[0][2];
    m[2][1] = m[1][2];
    m[2][2] = dot3(c, c);
    double md = -(m[0][2] * m[0][2] * m[1][1]) + 2.0 * m[0][1] * m[0][2] * m[1][2] -
                m[0][0] * (m[1][2] * m[1][2]) - m[0][1] * m[0][1] * m[2][2] +
                m[0][0] * m[1][1] * m[2][2];
    inv[0][0] = m[1][1] * m[2][2] - m[1][2] * m[1][2];
    inv[0][1] = m[0][2] * m[1][2] - m[0][1] * m[2][2];
    inv[0][2] = m[0][1] * m[1][2] - m[0][2] * m[1][1];
    inv[1][0] = inv[0][1];
    inv[1][1] = m[0][0] * m[2][2] - m[0][2] * m[0][2];
    inv[1][2] = m[0][1] * m[0][2] - m[0][0] * m[1][2];
    inv[2][0] = inv[0][2];
    inv[2][1] = inv[1][2];
    inv[2][2] = m[0][0] * m[1][1] - m[0][1] * m[0][1];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) inv[i][j] = inv[i][j] / md;
}

void orc_get_distance(const double posi[3], const double posj[3], const double a[3],
                      const double b[3], const double c[3], double dist[3], double *d,
                      int i_shift[3])
{
    if (is_orthorhombic(a, b, c)) {
        /* neighbors_interface.f90:565-581 */
        double L[3] = {a[0], b[1], c[2]};
        for (int i = 0; i < 3; ++i) {
            double raw = posj[i] - posi[i];
            i_shift[i] = (int)floor(raw / L[i]);
        }
        double d2 = 0.0;
        for (int i = 0; i < 3; ++i) {
            dist[i] = f_modulo(posj[i] - posi[i], L[i]);
            if (dist[i] > L[i] / 2.0) dist[i] = dist[i] - L[i];
            d2 = d2 + dist[i] * dist[i];
        }
        *d = sqrt(d2);
        return;
    }
    /* neighbors_interface.f90:582-636: triclinic, 27-image search around nint(...) */
    double inv[3][3];
    gram_inverse(a, b, c, inv);
    double dv[3] = {posj[0] - posi[0], posj[1] - posi[1], posj[2] - posi[2]};
    double v[3] = {-1.0 * dot3(dv, a), -1.0 * dot3(dv, b), -1.0 * dot3(dv, c)};
    double ir[3];
    for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        s = s + inv[i][0] * v[0];
        s = s + inv[i][1] * v[1];
        s = s + inv[i][2] * v[2];
        ir[i] = s;
    }
    int idx[3];
    for (int i = 0; i < 3; ++i) {
        i_shift[i] = (int)floor(-ir[i]);
        idx[i] = (int)lround(ir[i]);
    }
    double res_opt = 1.0e10;
    double best[3] = {dv[0], dv[1], dv[2]};
    for (int i = idx[0] - 1; i <= idx[0] + 1; ++i)
        for (int j = idx[1] - 1; j <= idx[1] + 1; ++j)
            for (int k = idx[2] - 1; k <= idx[2] + 1; ++k) {
                double t[3];
                for (int q = 0; q < 3; ++q)
                    t[q] = dv[q] + (double)i * a[q] + (double)j * b[q] + (double)k * c[q];
                double res = dot3(t, t);
                if (res < res_opt) {
                    res_opt = res;
                    best[0] = t[0];
                    best[1] = t[1];
                    best[2] = t[2];
                }
            }
    dist[0] = best[0];
    dist[1] = best[1];
    dist[2] = best[2];
    *d = sqrt(dot3(dist, dist));
}

static void cross(const double *x, const double *y, double *z)
{
    z[0] = x[1] * y[2] - x[2] * y[1];
    z[1] = x[2] * y[0] - x[0] * y[2];
    z[2] = x[0] * y[1] - x[1] * y[0];
}

void orc_number_of_unit_cells(const double a[3], const double b[3], const double c[3],
                              double rcut, int indices[3])
{
    double axb[3], bxc[3], cxa[3];
    cross(a, b, axb);
    cross(c, a, cxa);
    cross(b, c, bxc);
    double n;
    n = sqrt(dot3(axb, axb));
    for (int i = 0; i < 3; ++i) axb[i] = axb[i] / n;
    n = sqrt(dot3(cxa, cxa));
    for (int i = 0; i < 3; ++i) cxa[i] = cxa[i] / n;
    n = sqrt(dot3(bxc, bxc));
    for (int i = 0; i < 3; ++i) bxc[i] = bxc[i] / n;
    double m[3][3];
    m[0][0] = dot3(axb, a);
    m[0][1] = dot3(axb, b);
    m[0][2] = dot3(axb, c);
    m[1][0] = dot3(cxa, a);
    m[1][1] = dot3(cxa, b);
    m[1][2] = dot3(cxa, c);
    m[2][0] = dot3(bxc, a);
    m[2][1] = dot3(bxc, b);
    m[2][2] = dot3(bxc, c);
    double md = -m[0][2] * m[1][1] * m[2][0] + m[0][1] * m[1][2] * m[2][0] +
                m[0][2] * m[1][0] * m[2][1] - m[0][0] * m[1][2] * m[2][1] -
                m[0][1] * m[1][0] * m[2][2] + m[0][0] * m[1][1] * m[2][2];
    double inv[3][3];
    inv[0][0] = m[1][1] * m[2][2] - m[1][2] * m[2][1];
    inv[0][1] = m[0][2] * m[2][1] - m[0][1] * m[2][2];
    inv[0][2] = m[0][1] * m[1][2] - m[0][2] * m[1][1];
    inv[1][0] = m[1][2] * m[2][0] - m[1][0] * m[2][2];
    inv[1][1] = m[0][0] * m[2][2] - m[0][2] * m[2][0];
    inv[1][2] = m[0][2] * m[1][0] - m[0][0] * m[1][2];
    inv[2][0] = m[1][0] * m[2][1] - m[1][1] * m[2][0];
    inv[2][1] = m[0][1] * m[2][0] - m[0][0] * m[2][1];
    inv[2][2] = m[0][0] * m[1][1] - m[0][1] * m[1][0];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) inv[i][j] = inv[i][j] / md;
    double v = 2.0 * rcut;
    for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        s = s + inv[i][0] * v;
        s = s + inv[i][1] * v;
        s = s + inv[i][2] * v;
        double ir = fabs(s);
        indices[i] = (int)ir;
        if (ir > (double)indices[i]) indices[i] = indices[i] + 1;
    }
}

void orc_set_supercell(int n_sites, const double *pos, const int *species, const int indices[3],
                       double a[3], double b[3], double c[3], double *pos_sc, int *species_sc)
{
    int counter = 0;
    for (int i2 = 1; i2 <= indices[0]; ++i2)
        for (int j2 = 1; j2 <= indices[1]; ++j2)
            for (int k2 = 1; k2 <= indices[2]; ++k2)
                for (int i = 0; i < n_sites; ++i) {
                    for (int q = 0; q < 3; ++q)
                        pos_sc[3 * counter + q] = pos[3 * i + q] + (double)(i2 - 1) * a[q] +
                                                  (double)(j2 - 1) * b[q] +
                                                  (double)(k2 - 1) * c[q];
                    if (species_sc) species_sc[counter] = species[i];
                    ++counter;
                }
    for (int q = 0; q < 3; ++q) {
        a[q] = (double)indices[0] * a[q];
        b[q] = (double)indices[1] * b[q];
        c[q] = (double)indices[2] * c[q];
    }
}

/* Position of atom i relative to the box corner, via the MIC from the box centre
 * (neighbors_interface.f90:311-318). */
static void cell_frac_pos(const double *pos, const double a[3], const double b[3],
                          const double c[3], double out[3])
{
    double centre[3] = {a[0] / 2.0, b[1] / 2.0, c[2] / 2.0};
    double dist[3], d;
    int sh[3];
    orc_get_distance(centre, pos, a, b, c, dist, &d, sh);
    out[0] = dist[0] + centre[0];
    out[1] = dist[1] + centre[1];
    out[2] = dist[2] + centre[2];
}

int64_t orc_build_neighbors(int n_sites, int n_sites_supercell, const double *positions,
                            double a[3], double b[3], double c[3], int box_small,
                            double rcut_max, const int *species_supercell, int *n_neigh,
                            int *neighbors_list, double *rjs, double *xyz, double *thetas,
                            double *phis, int *neighbor_species)
{
    const double d_tol = 1.0e-6;
    int square = is_orthorhombic(a, b, c);
    if (square) {
        /* neighbors_interface.f90:216-225 snaps near-zero off-diagonals to 0 */
        (void)d_tol;
        a[1] = a[2] = b[0] = b[2] = c[0] = c[1] = 0.0;
    }
    const double tol = 1.0e-10;
    int64_t n_pairs = 0;
    int fill = neighbors_list != NULL;

    if (square && !box_small) {
        int mx = (int)(a[0] / rcut_max);
        int my = (int)(b[1] / rcut_max);
        int mz = (int)(c[2] / rcut_max);
        int ncell = mx * my * mz;
        int *head = (int *)calloc((size_t)ncell, sizeof(int));
        int *this_list = (int *)calloc((size_t)n_sites + 1, sizeof(int));
        for (int i = 1; i <= n_sites; ++i) {
            double p[3];
            cell_frac_pos(positions + 3 * (i - 1), a, b, c, p);
            int j = 1 + i_modulo((int)(p[0] / (a[0] + tol) * mx), mx) +
                    i_modulo((int)(p[1] / (b[1] + tol) * my), my) * mx +
                    i_modulo((int)(p[2] / (c[2] + tol) * mz), mz) * my * mx;
            this_list[i] = head[j - 1];
            head[j - 1] = i;
        }
        for (int i = 1; i <= n_sites; ++i) {
            int nn = 1;
            if (fill) neighbors_list[n_pairs] = i;
            ++n_pairs;
            double p[3];
            cell_frac_pos(positions + 3 * (i - 1), a, b, c, p);
            int i2 = 1 + (int)(p[0] / (a[0] + tol) * mx);
            int j2 = 1 + (int)(p[1] / (b[1] + tol) * my);
            int k2 = 1 + (int)(p[2] / (c[2] + tol) * mz);
            for (int k3 = k2 - 1; k3 <= k2 + 1; ++k3) {
                if (mz == 1 && k3 != 1) continue;
                if (mz == 2 && k2 == 1 && k3 == 0) continue;
                if (mz == 2 && k2 == 2 && k3 == 3) continue;
                for (int j3 = j2 - 1; j3 <= j2 + 1; ++j3) {
                    if (my == 1 && j3 != 1) continue;
                    if (my == 2 && j2 == 1 && j3 == 0) continue;
                    if (my == 2 && j2 == 2 && j3 == 3) continue;
                    for (int i3 = i2 - 1; i3 <= i2 + 1; ++i3) {
                        if (mx == 1 && i3 != 1) continue;
                        if (mx == 2 && i2 == 1 && i3 == 0) continue;
                        if (mx == 2 && i2 == 2 && i3 == 3) continue;
                        int j = 1 + i_modulo(i3 - 1, mx) + i_modulo(j3 - 1, my) * mx +
                                i_modulo(k3 - 1, mz) * mx * my;
                        int k = head[j - 1];
                        while (k != 0) {
                            if (k != i) {
                                double dist[3], d;
                                int sh[3];
                                orc_get_distance(positions + 3 * (i - 1), positions + 3 * (k - 1),
                                                 a, b, c, dist, &d, sh);
                                if (d < rcut_max) {
                                    if (fill) neighbors_list[n_pairs] = k;
                                    ++n_pairs;
                                    ++nn;
                                }
                            }
                            k = this_list[k];
                        }
                    }
                }
            }
            if (fill) n_neigh[i - 1] = nn;
        }
        free(head);
        free(this_list);
    } else {
        for (int i = 1; i <= n_sites; ++i) {
            int nn = 1;
            if (fill) neighbors_list[n_pairs] = i;
            ++n_pairs;
            for (int j = 1; j <= n_sites_supercell; ++j) {
                if (j == i) continue;
                double dist[3], d;
                int sh[3];
                orc_get_distance(positions + 3 * (i - 1), positions + 3 * (j - 1), a, b, c, dist,
                                 &d, sh);
                if (d < rcut_max) {
                    if (fill) neighbors_list[n_pairs] = j;
                    ++n_pairs;
                    ++nn;
                }
            }
            if (fill) n_neigh[i - 1] = nn;
        }
    }
    if (fill)
        orc_neighbor_geometry(n_sites, positions, a, b, c, n_neigh, neighbors_list,
                              species_supercell, rjs, xyz, thetas, phis, neighbor_species);
    return n_pairs;
}

void orc_neighbor_geometry(int n_sites, const double *positions, const double a[3],
                           const double b[3], const double c[3], const int *n_neigh,
                           const int *neighbors_list, const int *species_supercell,
                           double *rjs, double *xyz, double *thetas, double *phis,
                           int *neighbor_species)
{
    /* neighbors_interface.f90:467-510 */
    int64_t *start = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n_sites + 1));
    start[0] = 0;
    for (int i = 0; i < n_sites; ++i) start[i + 1] = start[i] + n_neigh[i];
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= n_sites; ++i) {
        for (int64_t k2 = start[i - 1]; k2 < start[i]; ++k2) {
            int j = neighbors_list[k2];
            if (k2 == start[i - 1]) {
                rjs[k2] = 0.0;
                xyz[3 * k2] = xyz[3 * k2 + 1] = xyz[3 * k2 + 2] = 0.0;
                thetas[k2] = 0.0;
                phis[k2] = 0.0;
                if (neighbor_species) neighbor_species[k2] = species_supercell[i - 1];
            } else {
                double dist[3], d;
                int sh[3];
                orc_get_distance(positions + 3 * (i - 1), positions + 3 * (j - 1), a, b, c, dist,
                                 &d, sh);
                rjs[k2] = d;
                xyz[3 * k2] = dist[0];
                xyz[3 * k2 + 1] = dist[1];
                xyz[3 * k2 + 2] = dist[2];
                if (fabs(dist[2]) >= d)
                    thetas[k2] = dist[2] > 0.0 ? 0.0 : acos(-1.0);
                else
                    thetas[k2] = acos(dist[2] / d);
                phis[k2] = atan2(dist[1], dist[0]);
                if (neighbor_species) neighbor_species[k2] = species_supercell[j - 1];
            }
        }
    }
    free(start);
}
