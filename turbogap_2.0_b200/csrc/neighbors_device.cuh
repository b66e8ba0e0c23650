// Minimum-image geometry on the device, shared by the neighbor build (neighbors.cu), the Monte
// Carlo trial geometry (mc.cu) and the per-step pair geometry of the descriptor forward.
// get_distance (src/neighbors/neighbors_interface.f90:547-643) is reproduced operation by
// operation with every product and sum rounded separately (__dmul_rn / __dadd_rn: no FMA
// contraction whatever the translation unit's flags), so the accept test d < rcut and the pair
// vectors carry the reference's bits.
#pragma once

#include "neighbors.h"

namespace tgap {

__device__ __forceinline__ double f_modulo(double a, double p)
{
    // fmod(a, p) is exact and equals a when |a| < p: skip the call on that (common) path
    double r = fabs(a) < p ? a : fmod(a, p);
    if (r != 0.0 && ((r < 0.0) != (p < 0.0))) r = __dadd_rn(r, p);
    return r;
}

__device__ __forceinline__ int i_modulo(int a, int m)
{
    int r = a % m;
    if (r != 0 && ((r < 0) != (m < 0))) r += m;
    return r;
}

__device__ __forceinline__ double dot3(const double *x, const double *y)
{
    double s = 0.0;
    s = __dadd_rn(s, __dmul_rn(x[0], y[0]));
    s = __dadd_rn(s, __dmul_rn(x[1], y[1]));
    s = __dadd_rn(s, __dmul_rn(x[2], y[2]));
    return s;
}

__device__ __forceinline__ void get_distance_dev(const double *pi, const double *pj, const StructDesc &S,
                                 double dist[3], double *d)
{
    if (S.ortho) {
        const double L[3] = {S.a[0], S.b[1], S.c[2]};
        double d2 = 0.0;
        for (int i = 0; i < 3; ++i) {
            dist[i] = f_modulo(__dsub_rn(pj[i], pi[i]), L[i]);
            if (dist[i] > L[i] / 2.0) dist[i] = __dsub_rn(dist[i], L[i]);
            d2 = __dadd_rn(d2, __dmul_rn(dist[i], dist[i]));
        }
        *d = sqrt(d2);
        return;
    }
    double dv[3] = {__dsub_rn(pj[0], pi[0]), __dsub_rn(pj[1], pi[1]), __dsub_rn(pj[2], pi[2])};
    double v[3] = {-1.0 * dot3(dv, S.a), -1.0 * dot3(dv, S.b), -1.0 * dot3(dv, S.c)};
    int idx[3];
    for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        s = __dadd_rn(s, __dmul_rn(S.inv[3 * i + 0], v[0]));
        s = __dadd_rn(s, __dmul_rn(S.inv[3 * i + 1], v[1]));
        s = __dadd_rn(s, __dmul_rn(S.inv[3 * i + 2], v[2]));
        idx[i] = (int)llround(s);
    }
    double res_opt = 1.0e10;
    double best[3] = {dv[0], dv[1], dv[2]};
    for (int i = idx[0] - 1; i <= idx[0] + 1; ++i)
        for (int j = idx[1] - 1; j <= idx[1] + 1; ++j)
            for (int k = idx[2] - 1; k <= idx[2] + 1; ++k) {
                double t[3];
                for (int q = 0; q < 3; ++q) {
                    double u = __dadd_rn(dv[q], __dmul_rn((double)i, S.a[q]));
                    u = __dadd_rn(u, __dmul_rn((double)j, S.b[q]));
                    t[q] = __dadd_rn(u, __dmul_rn((double)k, S.c[q]));
                }
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

// Position of supercell atom j (1-based within structure S) from the primitive positions, with
// the replication arithmetic of set_supercell (read_xyz.f90:331-345: replicas a -> b -> c outer,
// atoms inner; no contraction).
__device__ __forceinline__ void sc_position(const StructDesc &S, const double *pos, int j, double out[3])
{
    const int a = (j - 1) % S.n, r = (j - 1) / S.n;
    const int k2 = r % S.rep[2], j2 = (r / S.rep[2]) % S.rep[1], i2 = r / (S.rep[2] * S.rep[1]);
    const double *p = pos + 3 * (size_t)(S.atom_off + a);
    for (int q = 0; q < 3; ++q) {
        double v = __dadd_rn(p[q], __dmul_rn((double)i2, S.pa[q]));
        v = __dadd_rn(v, __dmul_rn((double)j2, S.pb[q]));
        v = __dadd_rn(v, __dmul_rn((double)k2, S.pc[q]));
        out[q] = v;
    }
}

}  // namespace tgap
