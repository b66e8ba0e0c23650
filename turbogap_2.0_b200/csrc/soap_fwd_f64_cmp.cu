// FP64 (plain path) instantiations of the SOAP forward for compressed descriptors (q = P p / |P p|).
#include "soap_warp.cuh"

namespace tgap {

int soap_fwd_f64_cmp(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites, int n_rows,
                     SoapOut &o)
{
    return launch_fwd<double, false, true>(ctx, ds, pv, d_sites, n_rows, o);
}

}  // namespace tgap
