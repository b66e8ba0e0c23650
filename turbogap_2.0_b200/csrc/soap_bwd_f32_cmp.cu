// FP32 (mixed path) instantiations of the SOAP adjoint for compressed descriptors (dE/dp = P^T dE/d(P p)).
#include "soap_warp.cuh"

namespace tgap {

int soap_bwd_f32_cmp(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites, int n_rows,
                     const SoapOut &o, const void *d_g, int g_ld, int g_is_double, const int *site_struct,
                     double *d_forces, double *d_virial)
{
    if (g_is_double)
        return launch_bwd<float, double, true>(ctx, ds, pv, d_sites, n_rows, o, d_g, g_ld, site_struct, d_forces,
                                               d_virial);
    return launch_bwd<float, float, true>(ctx, ds, pv, d_sites, n_rows, o, d_g, g_ld, site_struct, d_forces,
                                          d_virial);
}

}  // namespace tgap
