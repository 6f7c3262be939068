"""Ragged frequency grids through the whole solve.

  - Lmats = 0 with Lreal = 64: the real-axis G and Sigma alone; G against
    the oracle's solve within 2e-2 of max|G| (the bar of the parity tests for
    G(w + i eps) from independent chains, whose tails differ: near a pole the
    function at eps = 0.01 magnifies them), Sigma finite;
  - Lmats = 1: the solve, the printed self-energy and the observables file,
    whose zimp and simp (get_szr reads Sigma at two Matsubara points) are
    those of a zero self-energy: 1 and 0."""
import numpy as np
import pytest

import dmfted
import oracle as O

pytestmark = pytest.mark.gpu


def solver(m, **kw):
    ul = list(m.uloc) + [0.0] * (3 - len(m.uloc))
    p = dmfted.default_params(norb=m.norb, nbath=m.nbath, nspin=m.nspin, uloc=ul, ust=m.ust,
                              jh=m.jh, xmu=m.xmu, beta=m.beta, hfmode=int(m.hfmode), **kw)
    return dmfted.EDSolver(p, hloc=m.hloc)


def test_real_axis_only():
    m = O.seeded_model(4, nbath=5, u=2.0, beta=100.0)
    s = solver(m, lmats=0, lreal=64, precision=dmfted.FP64)
    s.ed_solve(m.bath_array(), sectors=[s.sector_index(3, 3)])
    ref = O.solve_t0(m, sectors=[(3, 3)], lmats=1, lreal=64)
    gr = s.ed_get_gimp_real()[0, 0, 0, 0]
    assert gr.shape == (64,)
    assert np.abs(gr - ref["greal"][0, 0]).max() <= 2e-2 * np.abs(ref["greal"][0, 0]).max()
    sr = s.ed_get_sigma_real()[0, 0, 0, 0]
    assert np.all(np.isfinite(sr))
    s.close()


def test_single_matsubara_point(tmp_path):
    m = O.seeded_model(4, nbath=5, u=2.0, beta=100.0)
    s = solver(m, lmats=1, lreal=0)
    for it in range(2):
        s.ed_solve(m.bath_array(), sectors=[s.sector_index(3, 3)])
        s.write_observables(str(tmp_path), "", legend=(it == 0))
    s.print_impSigma(str(tmp_path), "")
    lines = (tmp_path / "observables_all.ed").read_text().splitlines()
    assert len(lines) == 2
    vals = np.array(lines[1].split(), dtype=float)
    assert vals[-2] == 1.0 and vals[-1] == 0.0  # zimp, simp of the one-point grid
    a = np.loadtxt(tmp_path / "impSigma_l11_s1_iw.ed").reshape(-1, 3)
    assert a.shape == (1, 3)
    assert np.isclose(a[0, 2] + 1j * a[0, 1], s.ed_get_sigma_matsubara()[0, 0, 0, 0, 0],
                      rtol=0, atol=0)
    s.close()


@pytest.mark.parametrize("precision", [dmfted.FP64, dmfted.MIXED])
def test_doped_polarised_scan_t0(precision):
    """xmu = 0.7, HFMODE off, a spin-split bath (Nspin = 2), T = 0 over all
    sectors: the ground state lies away from half filling and is magnetised;
    E0, Z, n_up, n_dw, magz and G(iwn) of both spins against the oracle's
    solve (1e-10, 1e-9, 1e-8)."""
    rng = np.random.default_rng(21)
    e = rng.uniform(-1.0, 1.0, (1, 1, 4))
    v = 0.5 + rng.uniform(-0.1, 0.1, (1, 1, 4))
    e = np.concatenate([e - 0.15, e + 0.15])
    v = np.concatenate([v, v * 1.05])
    m = O.Model(norb=1, nbath=4, nspin=2, uloc=(2.5, 0.0, 0.0), xmu=0.7, hfmode=False,
                beta=100.0, e=e, v=v)
    s = solver(m, lmats=128, lreal=0, precision=precision)
    s.ed_solve(m.bath_array())
    ref = O.solve_t0(m, lmats=128, nthreads=4)
    assert abs(s.egs() - ref["egs"]) <= 1e-10 * abs(ref["egs"])
    _, _, z = s.eigenspace()
    assert abs(z - ref["zeta"]) <= 1e-12
    ob = s.observables()
    for k in ("dens_up", "dens_dw", "magz"):
        assert np.allclose(ob[k], ref["obs"][k], rtol=0, atol=1e-9), k
    assert abs(ob["magz"][0]) > 1e-3 and abs(ob["dens"][0] - 1.0) > 1e-3
    g = s.ed_get_gimp_matsubara()
    for i in range(2):
        assert np.abs(g[i, i, 0, 0] - ref["gmats"][i, 0]).max() <= 1e-8
    s.close()
