"""Finite-temperature solve (lanc_nstates_total > 1) against the oracle:
the kept eigenspace (energies, sectors, Z), the Boltzmann-weighted
observables and G(iwn) (1e-8), on a spin-split two-orbital model and a
one-orbital model.  The spin splitting keeps symmetry multiplets from
straddling the list boundary, where the reference's own choice between
equal energies depends on rounding."""
import numpy as np
import pytest

import dmfted
import oracle as O

pytestmark = pytest.mark.gpu


def split_model(seed, norb, nbath, beta, u=3.0, ust=0.0, jh=0.0):
    rng = np.random.default_rng(seed)
    e1 = rng.uniform(-1.5, 1.5, (norb, nbath))
    v1 = 0.4 + rng.uniform(-0.1, 0.1, (norb, nbath))
    e = np.stack([e1, e1 + rng.uniform(-0.2, 0.2, (norb, nbath))])
    v = np.stack([v1, v1 + rng.uniform(-0.05, 0.05, (norb, nbath))])
    ul = [u] * norb + [0.0] * (3 - norb)
    return O.Model(norb=norb, nbath=nbath, nspin=2, uloc=tuple(ul), ust=ust, jh=jh, beta=beta,
                   e=e, v=v)


@pytest.mark.parametrize("norb,nbath,total", [(1, 4, 8), (2, 2, 16)])
def test_finite_t_solve_matches_oracle(norb, nbath, total):
    m = split_model(5 + norb, norb, nbath, beta=50.0, ust=2.0 if norb > 1 else 0.0,
                    jh=0.5 if norb > 1 else 0.0)
    ul = list(m.uloc)
    p = dmfted.default_params(norb=norb, nbath=nbath, nspin=2, uloc=ul, ust=m.ust, jh=m.jh,
                              beta=m.beta, lmats=512, lreal=0, lanc_nstates_total=total)
    s = dmfted.EDSolver(p)
    s.ed_solve(m.bath_array())
    ref = O.solve_finite_t(m, lmats=512, nstates_total=total, nthreads=4)
    e, secs, z = s.eigenspace()
    re = np.array([x[0] for x in ref["states"]])
    rs = np.array([x[1] for x in ref["states"]])
    assert len(e) == len(re)
    assert np.array_equal(secs, rs)
    assert np.allclose(e, re, rtol=0, atol=1e-10 * max(1.0, np.abs(re).max()))
    assert abs(z - ref["zeta"]) <= 1e-10 * ref["zeta"]
    ob = s.observables()
    for k in ("dens", "dens_up", "dens_dw", "docc", "magz"):
        assert np.allclose(ob[k], ref["obs"][k], rtol=0, atol=1e-9), k
    gm = s.ed_get_gimp_matsubara()
    for ispin in range(2):
        for a in range(norb):
            dg = np.abs(gm[ispin, ispin, a, a] - ref["gmats"][ispin, a]).max()
            assert dg <= 1e-8, (ispin, a, dg)
    s.close()


def test_finite_t_second_solve_adapts_state_count():
    # ed_analysis grows lanc_nstates_total / trims between solves; a second
    # solve on the same context must still agree with a fresh oracle run
    # given the adapted parameters
    m = split_model(11, 1, 4, beta=20.0)
    p = dmfted.default_params(nbath=4, nspin=2, uloc=list(m.uloc), beta=m.beta, lmats=128,
                              lreal=0, lanc_nstates_total=4)
    s = dmfted.EDSolver(p)
    s.ed_solve(m.bath_array())
    n1 = len(s.eigenspace()[0])
    s.ed_solve(m.bath_array())
    e2, _, _ = s.eigenspace()
    assert len(e2) >= n1
    assert np.all(np.diff(e2) >= -1e-12)
    s.close()


def test_finite_t_three_orbitals_with_spin_exchange():
    """Norb = 3 (the largest orbital count) with the Jhflag spin-exchange and
    pair-hopping terms (Jx = Jp = 0.4) at finite temperature on a spin-split
    bath: the kept eigenspace, Z, the observables and G(iwn) of every spin and
    orbital against the oracle (1e-10, 1e-9, 1e-8)."""
    import dataclasses
    m = split_model(41, 3, 1, beta=30.0, ust=2.0, jh=0.4)
    m = dataclasses.replace(m, jx=0.4, jp=0.4, jhflag=True)
    p = dmfted.default_params(norb=3, nbath=1, nspin=2, uloc=list(m.uloc), ust=m.ust, jh=m.jh,
                              jx=m.jx, jp=m.jp, jhflag=1, beta=m.beta, lmats=256, lreal=0,
                              lanc_nstates_total=12)
    s = dmfted.EDSolver(p)
    s.ed_solve(m.bath_array())
    ref = O.solve_finite_t(m, lmats=256, nstates_total=12, nthreads=4)
    e, secs, z = s.eigenspace()
    re = np.array([x[0] for x in ref["states"]])
    assert len(e) == len(re)
    assert np.array_equal(secs, np.array([x[1] for x in ref["states"]]))
    assert np.allclose(e, re, rtol=0, atol=1e-10 * max(1.0, np.abs(re).max()))
    assert abs(z - ref["zeta"]) <= 1e-10 * ref["zeta"]
    ob = s.observables()
    for k in ("dens", "docc", "magz"):
        assert np.allclose(ob[k], ref["obs"][k], rtol=0, atol=1e-9), k
    gm = s.ed_get_gimp_matsubara()
    for ispin in range(2):
        for a in range(3):
            assert np.abs(gm[ispin, ispin, a, a] - ref["gmats"][ispin, a]).max() <= 1e-8
    s.close()
