"""Local energies of the solve (local_energy_impurity, ED_OBSERVABLES.f90:
454-635) against the oracle's restatement: ed_get_eimp = [Epot, Eint,
Ehartree, Eknot] and ed_get_doubles = [Dust, Dund, Dse, Dph], within 1e-9.
Cases: one orbital at T=0; two orbitals at finite temperature with
inter-orbital Hloc hopping and Jhflag on (Jx = Jp = 0, so H has no
spin-exchange or pair-hopping term while Dse and Dph are still measured);
three degenerate orbitals at T=0, where several ground states share a
sector."""
import numpy as np
import pytest

import dmfted
import oracle as O
from test_oracle import degenerate_models

pytestmark = pytest.mark.gpu


def solver(m, **kw):
    ul = list(m.uloc) + [0.0] * (3 - len(m.uloc))
    p = dmfted.default_params(norb=m.norb, nbath=m.nbath, nspin=m.nspin, uloc=ul, ust=m.ust,
                              jh=m.jh, jx=m.jx, jp=m.jp, xmu=m.xmu, beta=m.beta,
                              hfmode=int(m.hfmode), jhflag=int(m.jhflag), lreal=0, **kw)
    return dmfted.EDSolver(p, hloc=m.hloc)


def check(s, ref):
    assert np.allclose(s.ed_get_eimp(), ref["obs"]["eimp"], rtol=0, atol=1e-9), (
        s.ed_get_eimp(), ref["obs"]["eimp"])
    assert np.allclose(s.ed_get_doubles(), ref["obs"]["doubles"], rtol=0, atol=1e-9), (
        s.ed_get_doubles(), ref["obs"]["doubles"])


@pytest.mark.parametrize("precision", [dmfted.FP64, dmfted.MIXED])
def test_local_energies_single_orbital_t0(precision):
    m = O.seeded_model(1, nbath=7, u=2.0, beta=100.0)
    s = solver(m, lmats=64, precision=precision)
    s.ed_solve(m.bath_array(), sectors=[s.sector_index(4, 4)])
    ref = O.solve_t0(m, sectors=[(4, 4)], lmats=64)
    check(s, ref)
    s.close()


def test_local_energies_two_orbitals_finite_t():
    rng = np.random.default_rng(31)
    norb, nbath = 2, 2
    e1 = rng.uniform(-1.5, 1.5, (norb, nbath))
    v1 = 0.4 + rng.uniform(-0.1, 0.1, (norb, nbath))
    e = np.stack([e1, e1 + rng.uniform(-0.2, 0.2, (norb, nbath))])
    v = np.stack([v1, v1 + rng.uniform(-0.05, 0.05, (norb, nbath))])
    hloc = np.zeros((2, 2, norb, norb), complex)
    for s_ in range(2):
        hloc[s_, s_] = [[0.1, 0.15], [0.15, -0.05]]
    m = O.Model(norb=norb, nbath=nbath, nspin=2, uloc=(3.0, 3.0, 0.0), ust=2.0, jh=0.5,
                jhflag=True, beta=30.0, e=e, v=v, hloc=hloc)
    s = solver(m, lmats=64, lanc_nstates_total=12)
    s.ed_solve(m.bath_array())
    ref = O.solve_finite_t(m, lmats=64, nstates_total=12, nthreads=4)
    assert abs(s.ed_get_doubles()[2]) > 1e-6  # Dse is measured
    check(s, ref)
    s.close()


def test_local_energies_degenerate_three_orbitals():
    m = O.Model(norb=3, nbath=1, nspin=1, uloc=(3.0, 3.0, 3.0), ust=2.0, jh=0.5,
                beta=100.0, e=np.zeros((1, 3, 1)), v=np.full((1, 3, 1), 0.5))
    s = solver(m, lmats=32)
    s.ed_solve(m.bath_array())
    ref = O.solve_t0(m, lmats=32, nthreads=4)
    check(s, ref)
    m2, nkeep, _ = degenerate_models()[0]
    s2 = solver(m2, lmats=32)
    s2.ed_solve(m2.bath_array())
    ref2 = O.solve_t0(m2, lmats=32, nthreads=4)
    assert ref2["zeta"] == nkeep
    check(s2, ref2)
    s.close()
    s2.close()
