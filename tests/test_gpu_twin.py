"""ed_twin: the sectors with nup < ndw are not diagonalised; every state of a
sector with nup != ndw enters the state list together with a twin entry of
the same energy in the spin-flipped sector, whose vector the library builds
from the state's (ED_DIAG.f90:111-123, ED_EIGENSPACE.f90:157-213,399-430,
ED_SETUP.f90:429-438,1098-1161).  On spin-symmetric models the solve with
twins equals the oracle's restatement of the twin list (ED_EIGENSPACE.f90
insertion, popping and the twin vector's permutation): finite-T lists, the
two-orbital finite-T workload against its fixture, and degenerate and
single-orbital T=0 scans."""
import os

import numpy as np
import pytest

import dmfted
import oracle as O
from test_oracle import degenerate_models

pytestmark = pytest.mark.gpu


def multiset(e, secs, e0):
    return sorted((round(float(x - e0), 8), int(s)) for x, s in zip(e, secs))


def _check_list(s, ref, nspin, norb, ns):
    en, secs, zeta = s.eigenspace()
    re = [x[0] for x in ref["states"]]
    assert multiset(en, secs, re[0]) == multiset(re, [x[1] for x in ref["states"]], re[0])
    assert abs(zeta - ref["zeta"]) <= 1e-10 * ref["zeta"]
    g = s.ed_get_gimp_matsubara()
    for ispin in range(nspin):
        for a in range(norb):
            assert np.abs(g[ispin, ispin, a, a] - ref["gmats"][ispin, a]).max() <= 1e-8
    ob = s.observables()
    for k in ("dens", "docc", "magz"):
        assert np.allclose(ob[k], ref["obs"][k], atol=1e-9), k


@pytest.mark.parametrize("total", [8, 12])
def test_twin_finite_t_matches_oracle(total):
    # the capped list with twin pairs can hold one state more than the cap
    # (a pair inserted at cap - 1); the oracle restates that list
    rng = np.random.default_rng(41)
    e = rng.uniform(-1.5, 1.5, (1, 2, 2))
    v = 0.4 + rng.uniform(-0.1, 0.1, (1, 2, 2))
    m = O.Model(norb=2, nbath=2, nspin=1, uloc=(3.0, 3.0, 0.0), ust=2.0, jh=0.5, beta=20.0,
                e=e, v=v)
    p = dmfted.default_params(norb=2, nbath=2, uloc=[3.0, 3.0], ust=2.0, jh=0.5, beta=20.0,
                              lmats=128, lreal=0, lanc_nstates_total=total, ed_twin=1)
    s = dmfted.EDSolver(p)
    s.ed_solve(m.bath_array())
    ref = O.solve_finite_t(m, lmats=128, nstates_total=total, nthreads=4, twin=True)
    _check_list(s, ref, 1, 2, m.ns)
    s.close()


def test_twin_finite_t_matches_fixture():
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "config_pins.npz"))
    if "cfg4t_e" not in z:
        pytest.fail("cfg4t_e missing from config_pins.npz (run tests/golden/make_config_pins.py)")
    rng = np.random.default_rng(4)
    e = rng.uniform(-1.5, 1.5, size=(2, 4))
    v = 0.4 + rng.uniform(-0.1, 0.1, size=(2, 4))
    bath = np.concatenate([e.reshape(-1), e.reshape(-1), v.reshape(-1), v.reshape(-1)])
    p = dmfted.default_params(norb=2, nbath=4, nspin=2, uloc=[3.0, 3.0], ust=2.0, jh=0.5,
                              beta=50.0, lmats=4096, lreal=0, lanc_nstates_total=16, ed_twin=1)
    s = dmfted.EDSolver(p)
    s.ed_solve(bath)
    ref = dict(states=list(zip(z["cfg4t_e"], z["cfg4t_sector"])), zeta=float(z["cfg4t_zeta"]),
               gmats=z["cfg4t_gmats"], obs={k: z["cfg4t_" + k] for k in ("dens", "docc", "magz")})
    _check_list(s, ref, 2, 2, 10)
    s.close()


@pytest.mark.parametrize("which", ["degenerate", "single"])
def test_twin_t0_scan_matches_oracle(which):
    if which == "degenerate":
        m = degenerate_models()[0][0]
    else:
        m = O.seeded_model(5, nbath=3, u=2.0)
    ul = list(m.uloc) + [0.0] * (3 - len(m.uloc))
    out = []
    for twin in (0, 1):
        p = dmfted.default_params(norb=m.norb, nbath=m.nbath, nspin=m.nspin, uloc=ul, ust=m.ust,
                                  jh=m.jh, beta=m.beta, lmats=128, lreal=0, ed_twin=twin)
        s = dmfted.EDSolver(p)
        s.ed_solve(m.bath_array())
        e, secs, zeta = s.eigenspace()
        out.append((e, secs, zeta, s.ed_get_gimp_matsubara(), s.observables()))
        s.close()
    ref = O.solve_t0(m, lmats=128, nthreads=4)
    rsec = [a * (m.ns + 1) + b + 1 for _, a, b in ref["states"]]
    for e, secs, zeta, g, ob in out:
        assert zeta == ref["zeta"]
        assert multiset(e, secs, ref["egs"]) == multiset([x[0] for x in ref["states"]], rsec,
                                                         ref["egs"])
        assert np.abs(g[0, 0, 0, 0] - ref["gmats"][0, 0]).max() <= 1e-8
        assert np.allclose(ob["docc"], ref["obs"]["docc"], atol=1e-9)
