// FP64 (plain path) instantiations of the SOAP adjoint for compressed descriptors (dE/dp = P^T dE/d(P p)).
#include "soap_warp.cuh"

namespace tgap {

int soap_bwd_f64_cmp(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites, int n_rows,
                     const SoapOut &o, const void *d_g, int g_ld, const int *site_struct, double *d_forces,
                     double *d_virial)
{
    return launch_bwd<double, double, true>(ctx, ds, pv, d_sites, n_rows, o, d_g, g_ld, site_struct, d_forces,
                                            d_virial);
}

}  // namespace tgap
