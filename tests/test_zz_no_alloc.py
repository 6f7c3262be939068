"""dmfted_lanc_tridiag_noalloc, the tridiagonalisation entry point for callers
that cannot allocate device memory when they call it (their device memory is
owned by their own pool, or the call sits in a loop where cudaMalloc must not
run).  The caller passes every vector as a device pointer; the library uses a
fixed scratch array of its own.

Checks, through the C-ABI:
  - the entry point is the first work on a fresh context (only the tables of
    set_bath exist), so no buffer an earlier call allocated can hide an
    allocation of its own;
  - the device's free memory is the same before and after a call (the first
    call may also load the library's kernel code under lazy module loading,
    which is the driver's memory, so the check runs on the later calls);
  - two calls in a row reproduce the allocating entry point dmfted_lanc_tridiag
    on the same start vector within the tolerances of tests/test_gpu_parity.py
    (first 20 alpha/beta to 1e-10, the continued fraction G(iwn) to 1e-8) and
    agree with each other bit for bit;
  - an nlanc beyond the fixed scratch is refused with DMFTED_ERR_ARG."""
import numpy as np
import pytest

import dmfted
import oracle as O

pytestmark = pytest.mark.gpu


def test_no_alloc_tridiag_matches_allocating_entry_point():
    import torch
    m = O.seeded_model(3, nbath=7, u=2.0, beta=100.0)
    hi = O.build_sector(m.ns, 4, 4)
    hj = O.build_sector(m.ns, 5, 4)
    e0, psi, _ = O.lanczos_gs(m, hi)
    n2, vv = O.gf_vvinit(True, 1, hi, hj, psi)
    v = np.ascontiguousarray(vv.real)
    nlanc = 200
    dim = v.size
    dev = torch.device("cuda", 0)
    d_v = torch.tensor(v, dtype=torch.float64, device=dev)
    d_work = torch.empty(2 * dim, dtype=torch.float64, device=dev)
    d_a = torch.zeros(nlanc, dtype=torch.float64, device=dev)
    d_b = torch.zeros(nlanc, dtype=torch.float64, device=dev)
    d_n = torch.zeros(1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()

    p = dmfted.default_params(nbath=7, uloc=[2.0], beta=100.0, lmats=16, lreal=0)
    s = dmfted.EDSolver(p)
    s.set_bath(m.bath_array())
    isec = s.sector_index(5, 4)
    L = dmfted.lib()

    def call():
        dmfted._ck(L.dmfted_lanc_tridiag_noalloc(s.ctx, isec, d_v.data_ptr(), nlanc,
                                                 d_work.data_ptr(), d_a.data_ptr(),
                                                 d_b.data_ptr(), d_n.data_ptr()))
        torch.cuda.synchronize()
        return d_a.cpu().numpy().copy(), d_b.cpu().numpy().copy(), int(d_n.item())

    outs = [call()]
    for _ in range(2):
        free0 = torch.cuda.mem_get_info(dev)[0]
        outs.append(call())
        assert torch.cuda.mem_get_info(dev)[0] == free0

    # the allocating entry point on the same start vector
    a_ref, b_ref, n_ref = s.lanc_tridiag(isec, v, nlanc)
    wm = O.matsubara(100.0, 1024)

    def cf(a, b):
        g = np.zeros(1024, complex)
        O.add_to_lanczos_gf(1.0, e0, e0, 1.0, False, 100.0, a, b, 1, wm, np.zeros(0), 0.01, g,
                            np.zeros(0, complex))
        return g

    g_ref = cf(a_ref, b_ref)
    for a, b, n in outs:
        assert n == n_ref
        assert np.allclose(a[:20], a_ref[:20], rtol=0, atol=1e-10)
        assert np.allclose(b[:20], b_ref[:20], rtol=0, atol=1e-10)
        assert np.abs(cf(a, b) - g_ref).max() <= 1e-8
    # the fixed scratch keeps the previous call's contents; results do not
    # depend on them
    for a, b, _ in outs[1:]:
        assert np.array_equal(outs[0][0], a) and np.array_equal(outs[0][1], b)

    with pytest.raises(dmfted.DmftedError) as err:
        dmfted._ck(L.dmfted_lanc_tridiag_noalloc(s.ctx, isec, d_v.data_ptr(), 5000,
                                                 d_work.data_ptr(), d_a.data_ptr(),
                                                 d_b.data_ptr(), d_n.data_ptr()))
    assert err.value.code == dmfted.ERR_ARG
    s.close()
