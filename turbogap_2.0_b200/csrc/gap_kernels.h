// GAP kernel contraction launchers (gap.cu: FP64; gemm_tc.cu: bf16x3 tensor cores).
#pragma once

#include <cuda_bf16.h>

#include "tgap_internal.h"

namespace tgap {

// One soap_turbo GAP model resident on the device.
struct DeviceModel {
    int n_sparse = 0, dim = 0;
    int dim_pad = 0, m_pad = 0;  // padded sizes of the bf16 operands (multiples of 64 / 128)
    double delta = 1.0, zeta = 4.0;
    // integer-zeta test: |zeta - z| < zeta_tol with z = trunc(zeta) (gap.f90:99-105, 1e-5) or, for
    // local properties, z = nint(zeta) and 1e-10 (local_properties.f90:76-77)
    double zeta_tol = 1.0e-5;
    bool zeta_nint = false;
    DevBuf Qs;        // double [n_sparse][dim]  (row = sparse point; Fortran Qs(dim, n_sparse))
    DevBuf QsT;       // double [dim][n_sparse]
    DevBuf alphas;    // double [n_sparse]
    DevBuf alphas32;  // float  [m_pad] (zero padded)
    DevBuf Q_hi, Q_lo;    // bf16 [m_pad][dim_pad]
    DevBuf QT_hi, QT_lo;  // bf16 [dim_pad][m_pad]
};

struct GapWork {
    DevBuf e_part;    // energy partials
    DevBuf G;         // FP64: [M][n_sparse]
    DevBuf g;         // dE/dq: double [M][dim] (FP64) or float [M][dim_pad] (mixed)
    DevBuf G_hi, G_lo;  // mixed: bf16 [m_rows_pad][m_pad]
};

int dgemm_nt(tgap_context *ctx, int M, int N, int K, const double *A, int lda, const double *B,
             int ldb, double *C, int ldc, double alpha);
int transpose_f64(tgap_context *ctx, int R, int C, const double *in, double *out);

// Energies (delta^2 sum alpha K^zeta + e0) added into d_energies[sites[row]] and/or written to
// d_e_rows; when do_forces, w->g = dE/dq (double, [n_rows][dim]).
int gap_energy_grad_f64(tgap_context *ctx, const DeviceModel &m, const double *d_q, int q_ld,
                        int n_rows, double e0, int do_forces, GapWork *w, const int *d_sites,
                        double *d_e_rows, double *d_energies);

// Mixed path: q given as bf16 hi/lo [rows_pad][dim_pad]; w->g = dE/dq (float [n_rows][dim_pad]).
// d_skip (fused kernel only): a device flag that, when set at run time, makes the launch a no-op.
// g_cleared: the caller zeroed rows [0, n_rows) of w->g (sized [rows_pad][dim_pad]) already.
// d_skip_tiles: optional device flags per 128-row tile; the fused kernel leaves the energies (and
// dE/dq) of a flagged tile's rows untouched (the unfused path computes every tile).
int gap_energy_grad_mixed(tgap_context *ctx, const DeviceModel &m, const __nv_bfloat16 *q_hi,
                          const __nv_bfloat16 *q_lo, int n_rows, double e0, int do_forces,
                          GapWork *w, const int *d_sites, double *d_e_rows, double *d_energies,
                          const int *d_skip = nullptr, bool g_cleared = false,
                          const int *d_skip_tiles = nullptr);
int model_upload_mixed(tgap_context *ctx, DeviceModel *m);

// Local properties (local_properties.f90:46-147): V clipped at zero, and per-pair derivatives
// V_der(:, j) = g_i . der(:, :, j) (zero for clipped sites) from a materialised soap_cart_der.
int clip_nonneg(tgap_context *ctx, int n, double *d_v);
int local_property_pairs(tgap_context *ctx, int n_sites, const int64_t *d_start, const double *d_g, int D,
                         const double *d_der, const double *d_V, double *d_V_der);

int pair_forces_from_der(tgap_context *ctx, int n_sites, const int64_t *d_start, const int *d_nl,
                         int n_sites0, const double *d_g, int D, const double *d_der,
                         const double *d_xyz, double *d_forces, double *d_virial);

}  // namespace tgap
