// Launchers of the descriptor kernels (soap.cu).
#pragma once

#include <cuda_bf16.h>

#include "tgap_internal.h"

namespace tgap {

// Outputs of the forward pass for n_rows sites (element type double or float by precision).
struct SoapOut {
    void *c = nullptr;     // [n_rows][n_max][nlm] expansion coefficients
    void *q = nullptr;     // [n_rows][q_ld] normalised descriptor (columns >= dim are zero)
    void *norm = nullptr;  // [n_rows] |p|
    int q_ld = 0;
    __nv_bfloat16 *q_hi = nullptr;  // optional bf16 split of q for the tensor-core GEMM
    __nv_bfloat16 *q_lo = nullptr;
    float *g_clear = nullptr;  // optional: row r of this [n_rows][q_ld] FP32 accumulator is zeroed
};

int upload_ylm_constants();
int soap_forward(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites,
                 int n_rows, int precision, SoapOut &o);
int soap_backward(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites,
                  int n_rows, int precision, const SoapOut &o, const void *d_g, int g_ld,
                  int g_is_double, const int *site_struct, double *d_forces, double *d_virial);
// Per-precision instantiations of the warp kernels (soap_fwd_f32.cu, soap_fwd_f64.cu,
// soap_bwd_f32.cu, soap_bwd_f64.cu) and of their compressed-descriptor forms (the *_cmp.cu files,
// for a model whose ds.p.cmp_row is set; the uncompressed kernels carry no compression code).
#define TGAP_SOAP_FWD_DECL(name)                                                                          \
    int name(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites, int n_rows, \
             SoapOut &o);
TGAP_SOAP_FWD_DECL(soap_fwd_f32)
TGAP_SOAP_FWD_DECL(soap_fwd_f64)
TGAP_SOAP_FWD_DECL(soap_fwd_f32_cmp)
TGAP_SOAP_FWD_DECL(soap_fwd_f64_cmp)
#undef TGAP_SOAP_FWD_DECL
int soap_bwd_f32(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites, int n_rows,
                 const SoapOut &o, const void *d_g, int g_ld, int g_is_double, const int *site_struct,
                 double *d_forces, double *d_virial);
int soap_bwd_f32_cmp(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites, int n_rows,
                     const SoapOut &o, const void *d_g, int g_ld, int g_is_double, const int *site_struct,
                     double *d_forces, double *d_virial);
int soap_bwd_f64(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites, int n_rows,
                 const SoapOut &o, const void *d_g, int g_ld, const int *site_struct, double *d_forces,
                 double *d_virial);
int soap_bwd_f64_cmp(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites, int n_rows,
                     const SoapOut &o, const void *d_g, int g_ld, const int *site_struct, double *d_forces,
                     double *d_virial);
int soap_cart_der(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites,
                  int n_rows, const SoapOut &o, double *d_der);
// SOAP compression of n_sites normalised uncompressed rows q (and, with der, their per-pair
// derivatives [pair][dim][3]); P by rows in ds.p (CSR). Writes q_c [site][dim_out] and
// der_c [pair][dim_out][3].
int soap_compress_rows(tgap_context *ctx, const DeviceSoap &ds, int n_sites, const int64_t *d_start,
                       const double *d_q, const double *d_der, double *d_qc, double *d_derc);

}  // namespace tgap
