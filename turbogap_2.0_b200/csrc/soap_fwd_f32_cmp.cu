// FP32 (mixed path) instantiations of the SOAP forward for compressed descriptors (q = P p / |P p|).
#include "soap_warp.cuh"

namespace tgap {

int soap_fwd_f32_cmp(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites, int n_rows,
                     SoapOut &o)
{
    if (o.q_hi) return launch_fwd<float, true, true>(ctx, ds, pv, d_sites, n_rows, o);
    return launch_fwd<float, false, true>(ctx, ds, pv, d_sites, n_rows, o);
}

}  // namespace tgap
