// FP64 (plain path) instantiations of the warp-per-site SOAP forward expansion + power spectrum kernels.
#include "soap_warp.cuh"

namespace tgap {

int soap_fwd_f64(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites, int n_rows,
                 SoapOut &o)
{
    return launch_fwd<double, false, false>(ctx, ds, pv, d_sites, n_rows, o);
}

}  // namespace tgap
