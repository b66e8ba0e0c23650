// FP32 (mixed path) instantiations of the warp-per-site SOAP forward expansion + power spectrum kernels.
#include "soap_warp.cuh"

namespace tgap {

int soap_fwd_f32(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites, int n_rows,
                 SoapOut &o)
{
    if (o.q_hi) return launch_fwd<float, true, false>(ctx, ds, pv, d_sites, n_rows, o);
    return launch_fwd<float, false, false>(ctx, ds, pv, d_sites, n_rows, o);
}

}  // namespace tgap
