"""GPU test of tgap_soap_energies_noalloc, the energies-only entry point for callers that cannot
allocate device memory themselves (for example a Fortran driver working only on device arrays
it was handed, or a code whose memory pool was sized at start-up). Its scratch is a fixed
array inside the library, so the test checks that two calls in a row, sharing that array,
both reproduce the energies of the ordinary allocating entry point
tgap_get_soap_energy_and_forces, and that sizes beyond the array are refused.

The file is named to be collected last, so a run that stops at the first failure has already
run every other test; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E_TOL = 1e-10  # eV / atom, the FP64 energy bar of the parity tests


def _bind(native):
    f = native.lib().tgap_soap_energies_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                  C.c_double, C.c_void_p, C.c_void_p]
    return f


def _inputs(seed, n_sites=300, n_sparse=150, dim=324):
    rng = np.random.default_rng(seed)
    q = np.abs(rng.normal(size=(n_sites, dim))) + 0.05
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    Qs = q[rng.choice(n_sites, n_sparse)] + 0.01 * rng.normal(size=(n_sparse, dim))
    Qs /= np.linalg.norm(Qs, axis=1, keepdims=True)
    alphas = rng.normal(0.0, 1e-3, n_sparse)
    return q, Qs, alphas


@pytest.mark.parametrize("zeta,delta", [(4.0, 1.0), (2.5, 0.7), (4.0, 1.3)])
def test_noalloc_energies_match_allocating_entry_twice(tg, zeta, delta):
    """zeta = 4 takes the integer-power path of the GEMM epilogue, 2.5 the real power (the
    integer test of gap.f90:99-105 fails); delta scales every energy by delta^2."""
    import torch
    from turbogap_b200 import native
    noalloc = _bind(native)
    q, Qs, alphas = _inputs(3)
    n_sites, dim = q.shape
    ctx = tg.Context(0)
    ones = np.ones(n_sites, np.int32)
    e_ref, _, _ = ctx.get_soap_energy_and_forces(q, None, alphas, delta, zeta, -0.25, Qs, ones,
                                                 np.arange(1, n_sites + 1), np.zeros((n_sites, 3)),
                                                 do_forces=False)
    ctx.close()
    dq = torch.from_numpy(q).cuda()
    dQ = torch.from_numpy(Qs).cuda()
    da = torch.from_numpy(alphas).cuda()
    de = torch.empty(n_sites, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        de.fill_(float("nan"))  # the call must overwrite every output
        st = noalloc(C.c_void_p(stream), dim, n_sites, len(alphas), C.c_void_p(dq.data_ptr()),
                     C.c_void_p(da.data_ptr()), delta, zeta, -0.25, C.c_void_p(dQ.data_ptr()),
                     C.c_void_p(de.data_ptr()))
        assert st == 0, f"call {call}: status {st}"
        torch.cuda.synchronize()
        e = de.cpu().numpy()
        assert np.all(np.isfinite(e))
        assert np.max(np.abs(e - e_ref)) < E_TOL, f"call {call}"


def test_noalloc_rejects_sizes_beyond_its_scratch(tg):
    import torch
    from turbogap_b200 import native
    noalloc = _bind(native)
    buf = torch.zeros(64, dtype=torch.float64, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    # 2^20 + 1 sites x 1 tile of sparse points exceeds the 2^20 partials; refused before any launch
    st = noalloc(None, 8, (1 << 20) + 1, 64, p, p, 1.0, 4.0, 0.0, p, p)
    assert st == 3  # TGAP_ERR_CAPACITY
    assert b"exceeds" in native.lib().tgap_last_error(None)  # the calling thread's context-free message
    assert noalloc(None, 8, 0, 64, p, p, 1.0, 4.0, 0.0, p, p) == 1  # TGAP_ERR_ARGUMENT
