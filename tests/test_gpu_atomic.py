"""The empty bath (Nbath = 0: the isolated impurity, every sector of dimension
one or a few states) through the whole solve.

Checks:
  - one orbital, U=2, half filling, HFMODE, T=0 over all sectors: the
    doublet (1,0), (0,1) is kept (Z = 2) at E0 = -U/4, <n> = 1, docc = 0, and
    G(iwn) is the atomic limit (1/(iwn - U/2) + 1/(iwn + U/2))/2 within 1e-12,
    in FP64 and in the mixed form;
  - two orbitals with inter-orbital Hloc hopping (Ust, Jh), T=0 over all
    sectors: energies, Z, <n>, docc and G(iwn) equal the oracle's solve
    within 1e-10 / 1e-9 / 1e-8."""
import numpy as np
import pytest

import dmfted
import oracle as O

pytestmark = pytest.mark.gpu

LM = 128


def solver(m, **kw):
    ul = list(m.uloc) + [0.0] * (3 - len(m.uloc))
    p = dmfted.default_params(norb=m.norb, nbath=m.nbath, nspin=m.nspin, uloc=ul, ust=m.ust,
                              jh=m.jh, xmu=m.xmu, beta=m.beta, hfmode=int(m.hfmode), lmats=LM,
                              lreal=0, **kw)
    return dmfted.EDSolver(p, hloc=m.hloc)


@pytest.mark.parametrize("precision", [dmfted.FP64, dmfted.MIXED])
def test_single_orbital_atom(precision):
    u, beta = 2.0, 100.0
    m = O.Model(norb=1, nbath=0, nspin=1, uloc=(u, 0.0, 0.0), beta=beta,
                e=np.zeros((1, 1, 0)), v=np.zeros((1, 1, 0)))
    s = solver(m, precision=precision)
    s.ed_solve(np.zeros(0))
    assert abs(s.egs() - (-u / 4)) <= 1e-14
    e, _, z = s.eigenspace()
    assert len(e) == 2 and z == 2.0
    ob = s.observables()
    assert abs(ob["dens"][0] - 1.0) <= 1e-14 and abs(ob["docc"][0]) <= 1e-14
    wm = O.matsubara(beta, LM)
    g = s.ed_get_gimp_matsubara()[0, 0, 0, 0]
    ref = 0.5 * (1.0 / (1j * wm - u / 2) + 1.0 / (1j * wm + u / 2))
    assert np.abs(g - ref).max() <= 1e-12
    s.close()


def test_two_orbital_atom_matches_oracle():
    hloc = np.zeros((1, 1, 2, 2), complex)
    hloc[0, 0] = [[0.2, 0.15], [0.15, -0.1]]
    m = O.Model(norb=2, nbath=0, nspin=1, uloc=(3.0, 3.0, 0.0), ust=2.0, jh=0.5, beta=100.0,
                e=np.zeros((1, 2, 0)), v=np.zeros((1, 2, 0)), hloc=hloc)
    s = solver(m)
    s.ed_solve(np.zeros(0))
    ref = O.solve_t0(m, lmats=LM)
    assert abs(s.egs() - ref["egs"]) <= 1e-10 * max(1.0, abs(ref["egs"]))
    e, _, z = s.eigenspace()
    assert len(e) == int(round(ref["zeta"])) and abs(z - ref["zeta"]) <= 1e-12
    ob = s.observables()
    for k in ("dens", "docc"):
        assert np.allclose(ob[k], ref["obs"][k], rtol=0, atol=1e-9), k
    g = s.ed_get_gimp_matsubara()
    for a in range(2):
        assert np.abs(g[0, 0, a, a] - ref["gmats"][0, a]).max() <= 1e-8
    s.close()


@pytest.mark.parametrize("nspin", [1, 2])
def test_single_orbital_atom_finite_temperature(nspin):
    """beta = 2, all four states kept (lanc_nstates_total = 4): Z over the
    kept states, relative to the ground doublet's weight, is
    2 + 2 e^{-beta U/2}; <n> = 1 and docc = e^{-beta U/2}/Z; at half filling
    G(iwn) is the same atomic limit at any temperature; the chains have
    length one (jdim = 1)."""
    u, beta = 2.0, 2.0
    m = O.Model(norb=1, nbath=0, nspin=nspin, uloc=(u, 0.0, 0.0), beta=beta,
                e=np.zeros((nspin, 1, 0)), v=np.zeros((nspin, 1, 0)))
    s = solver(m, lanc_nstates_total=4)
    s.ed_solve(np.zeros(0))
    e, _, z = s.eigenspace()
    assert len(e) == 4
    # weights relative to the ground state (E = -U/4): two states at +U/4
    assert abs(z - (2.0 + 2.0 * np.exp(-beta * u / 2))) <= 1e-12 * z
    ob = s.observables()
    assert abs(ob["dens"][0] - 1.0) <= 1e-13
    assert abs(ob["docc"][0] - np.exp(-beta * u / 2) / z) <= 1e-13
    wm = O.matsubara(beta, LM)
    g = s.ed_get_gimp_matsubara()
    ref = 0.5 * (1.0 / (1j * wm - u / 2) + 1.0 / (1j * wm + u / 2))
    for i in range(nspin):
        assert np.abs(g[i, i, 0, 0] - ref).max() <= 1e-12
    s.close()
