"""Several solver contexts in one process: contexts of different Ns (and so
different class tables) used alternately must give the results each gives
alone.  Every context keeps its own tables; nothing Ns-dependent may live in
process-wide device state."""
import numpy as np
import pytest

import dmfted
import oracle as O

pytestmark = pytest.mark.gpu


def params_for(m, **kw):
    return dmfted.default_params(norb=m.norb, nbath=m.nbath, nspin=m.nspin, uloc=list(m.uloc),
                                 ust=m.ust, jh=m.jh, beta=m.beta, lmats=64, lreal=0, **kw)


def test_interleaved_contexts_of_different_ns():
    big = O.seeded_model(31, nbath=9, u=3.0)          # Ns = 10
    small = O.seeded_model(32, norb=2, nbath=2, u=2.0, ust=1.0, jh=0.5)  # Ns = 6
    a = dmfted.EDSolver(params_for(big))
    ia = a.sector_index(5, 5)
    a.ed_solve(big.bath_array(), sectors=[ia])
    e_a, g_a = a.egs(), a.ed_get_gimp_matsubara()
    # a second context with another Ns, created and solved in between,
    # finite temperature so that the batched kernels run too
    b = dmfted.EDSolver(params_for(small, lanc_nstates_total=8))
    b.ed_solve(small.bath_array())
    e_b = b.egs()
    b.close()
    # the first context again: the bath upload rebuilds its hopping tables
    a.ed_solve(big.bath_array(), sectors=[ia])
    assert a.egs() == e_a
    assert np.array_equal(a.ed_get_gimp_matsubara(), g_a)
    hm = O.build_sector(big.ns, 5, 5)
    e0, _, _ = O.lanczos_gs(big, hm)
    assert abs(a.egs() - e0) <= 1e-10 * abs(e0)
    # and a fresh small context after the big one agrees with the first
    b2 = dmfted.EDSolver(params_for(small, lanc_nstates_total=8))
    b2.ed_solve(small.bath_array())
    assert abs(b2.egs() - e_b) <= 1e-12 * abs(e_b)
    b2.close()
    a.close()


def test_bath_updates_with_and_without_zero_couplings():
    # the hopping tables depend on which couplings are non-zero: a bath with a
    # zero V_k removes those hops, the next bath without one restores them
    m = O.seeded_model(33, nbath=7, u=2.0)
    s = dmfted.EDSolver(params_for(m))
    isec = s.sector_index(4, 4)
    hm = O.build_sector(m.ns, 4, 4)
    for zero in (None, 2, None, 5, 5, None):
        mk = O.seeded_model(33, nbath=7, u=2.0)
        if zero is not None:
            mk.v[:, :, zero] = 0.0
        s.ed_solve(mk.bath_array(), sectors=[isec])
        e0, _, _ = O.lanczos_gs(mk, hm)
        assert abs(s.egs() - e0) <= 1e-10 * abs(e0), zero
    s.close()
