"""The printed outputs (ED_IO print_impG / print_impSigma / print_impG0 /
read_impSigma, ED_OBSERVABLES write_legend / write_observables /
write_energy_info / write_energy) through the C-ABI, on solved contexts.

Checks:
  - the Green's-function files hold one line per point with the abscissa,
    Im f, Re f (the columns of SciFortran's splot), and read back bit for bit
    into the arrays ed_get_* returns; the abscissae are the reference grids
    wm = pi/beta (2n-1) and wr = linspace(wini, wfin, Lreal);
  - print_impG0 writes G0and under the impG_... names, as the reference does;
  - read_impSigma into a fresh context gives ed_get_sigma_* bit for bit, and a
    missing or short file is an error that leaves the context unchanged;
  - observables_info.ed / energy_info.ed equal the oracle's restatement of
    the Fortran formats character for character; every observables_all
    record equals the oracle's record of the solve's own values (dens, docc,
    dens_up, dens_dw, magz, s2tot, egs, sz2, n2, zimp, simp), and those values
    agree with the oracle's solve within 1e-9 (s2tot, sz2, n2 included; at
    finite temperature for the first solve, before ed_analysis grows the
    state list);
  - zimp and simp of a solve come from the previous solve's Sigma (1 and 0 on
    the first), as get_szr runs before the Green's functions in ed_solve;
  - energy_last holds ed_get_eimp / ed_get_doubles in write_energy's order."""
import numpy as np
import pytest

import dmfted
import oracle as O

pytestmark = pytest.mark.gpu

LM, LR = 64, 48


def solver(m, **kw):
    ul = list(m.uloc) + [0.0] * (3 - len(m.uloc))
    p = dmfted.default_params(norb=m.norb, nbath=m.nbath, nspin=m.nspin, uloc=ul, ust=m.ust,
                              jh=m.jh, xmu=m.xmu, beta=m.beta, hfmode=int(m.hfmode),
                              lmats=LM, lreal=LR, **kw)
    return dmfted.EDSolver(p, hloc=m.hloc)


def read3(path):
    a = np.loadtxt(path)
    assert a.ndim == 2 and a.shape[1] == 3, a.shape
    return a[:, 0], a[:, 2] + 1j * a[:, 1]


def two_orbital_model():
    rng = np.random.default_rng(5)
    e = rng.uniform(-1.0, 1.0, (2, 2, 2))
    v = 0.4 + rng.uniform(-0.1, 0.1, (2, 2, 2))
    e[1] = e[0] + 0.1
    return O.Model(norb=2, nbath=2, nspin=2, uloc=(3.0, 3.0, 0.0), ust=2.0, jh=0.5, beta=40.0,
                   e=e, v=v)


def test_green_function_files_round_trip(tmp_path):
    m = O.seeded_model(1, nbath=5, u=2.0, beta=60.0)
    s = solver(m)
    s.ed_solve(m.bath_array(), sectors=[s.sector_index(3, 3)])
    wm = O.matsubara(m.beta, LM)
    wr = O.realaxis(-5.0, 5.0, LR)
    d = str(tmp_path)
    s.print_impG(d, "_x")
    s.print_impSigma(d, "_x")
    for name, mats, real in (("impG", s.ed_get_gimp_matsubara(), s.ed_get_gimp_real()),
                             ("impSigma", s.ed_get_sigma_matsubara(), s.ed_get_sigma_real())):
        x, y = read3(tmp_path / f"{name}_l11_s1_iw_x.ed")
        assert np.array_equal(y, mats[0, 0, 0, 0])
        assert np.allclose(x, wm, rtol=1e-15, atol=0)
        x, y = read3(tmp_path / f"{name}_l11_s1_realw_x.ed")
        assert np.array_equal(y, real[0, 0, 0, 0])
        assert np.allclose(x, wr, rtol=0, atol=1e-13)  # linspace: a few ulp apart
    # G0and under the impG names
    s.print_impG0(d, "_x")
    _, y = read3(tmp_path / "impG_l11_s1_iw_x.ed")
    assert np.array_equal(y, s.ed_get_g0imp_matsubara()[0, 0, 0, 0])
    _, y = read3(tmp_path / "impG_l11_s1_realw_x.ed")
    g0r = s.ed_get_g0imp_real()[0, 0, 0, 0]
    assert np.array_equal(y, g0r)
    # G0and = 1/(z + xmu - Delta(z)) on the real axis
    z = wr + 1j * 0.01
    ref = 1.0 / (z + m.xmu - O.delta_bath(m.e[0, 0], m.v[0, 0], z))
    assert np.abs(g0r - ref).max() <= 1e-12 * np.abs(ref).max()
    s.close()


def test_read_impsigma(tmp_path):
    m = two_orbital_model()
    s = solver(m, lanc_nstates_total=8)
    s.ed_solve(m.bath_array())
    d = str(tmp_path)
    s.print_impSigma(d, "")
    fresh = solver(m, lanc_nstates_total=8)
    with pytest.raises(dmfted.DmftedError):
        fresh.ed_get_sigma_matsubara()  # nothing solved or read yet
    fresh.read_impSigma(d, "")
    assert np.array_equal(fresh.ed_get_sigma_matsubara(), s.ed_get_sigma_matsubara())
    assert np.array_equal(fresh.ed_get_sigma_real(), s.ed_get_sigma_real())
    # a short file: an error, the context's self-energy unchanged
    lines = (tmp_path / "impSigma_l22_s2_realw.ed").read_text().splitlines()
    (tmp_path / "impSigma_l22_s2_realw.ed").write_text("\n".join(lines[:-1]) + "\n")
    with pytest.raises(dmfted.DmftedError):
        fresh.read_impSigma(d, "")
    assert np.array_equal(fresh.ed_get_sigma_matsubara(), s.ed_get_sigma_matsubara())
    with pytest.raises(dmfted.DmftedError):
        fresh.read_impSigma(str(tmp_path / "missing"), "")
    s.close()
    fresh.close()


@pytest.mark.parametrize("case", ["one_orbital_t0", "two_orbitals_finite_t"])
def test_observable_and_energy_files(tmp_path, case):
    if case == "one_orbital_t0":
        m = O.seeded_model(2, nbath=5, u=2.0, beta=60.0)
        s = solver(m)
        sectors = [s.sector_index(3, 3)]
        ref = O.solve_t0(m, sectors=[(3, 3)], lmats=LM, lreal=LR)
    else:
        m = two_orbital_model()
        s = solver(m, lanc_nstates_total=8)
        sectors = None
        ref = O.solve_finite_t(m, lmats=LM, lreal=LR, nstates_total=8, nthreads=4)
    d = str(tmp_path)
    no, ns = m.norb, m.nspin
    records = []
    prev_sigma = None
    for it in range(2):
        s.ed_solve(m.bath_array(), sectors=sectors)
        s.write_observables(d, "", legend=(it == 0))
        s.write_energy(d, "")
        ob = s.observables()
        if prev_sigma is None:
            zimp, simp = np.ones((ns, no)), np.zeros((ns, no))
        else:
            zs = [[O.szr(prev_sigma[i, i, a, a, :2], m.beta) for a in range(no)] for i in range(ns)]
            zimp = np.array([[z[0] for z in row] for row in zs])
            simp = np.array([[z[1] for z in row] for row in zs])
        prev_sigma = s.ed_get_sigma_matsubara()
        records.append((ob, zimp, simp))
    info = (tmp_path / "observables_info.ed").read_text()
    assert info == O.observables_legend_text(no, ns)
    lines = (tmp_path / "observables_all.ed").read_text().splitlines(keepends=True)
    assert len(lines) == 2
    for it, (line, (ob, zimp, simp)) in enumerate(zip(lines, records)):
        vals = np.array(line.split(), dtype=float)
        nso = 5 * no + 2 + 2 * no * no
        s2tot, egs = vals[5 * no], vals[5 * no + 1]
        sz2 = vals[5 * no + 2:5 * no + 2 + no * no].reshape(no, no)
        n2 = vals[5 * no + 2 + no * no:nso].reshape(no, no)
        want = O.observables_record_text(ob["dens"], ob["docc"], ob["dens_up"], ob["dens_dw"],
                                         ob["magz"], s2tot, s.egs(), sz2, n2, zimp, simp)
        assert line == want
        if it > 0 and case != "one_orbital_t0":
            continue  # ed_analysis has grown the state list: not the oracle's solve
        # the values against the oracle's solve (F15.9: 5e-10 of rounding)
        assert abs(egs - ref["egs" if "egs" in ref else "e0"]) <= 1e-9
        assert abs(s2tot - ref["obs"]["s2tot"]) <= 1e-9
        assert np.allclose(sz2, ref["obs"]["sz2"], rtol=0, atol=1e-9)
        assert np.allclose(n2, ref["obs"]["n2"], rtol=0, atol=1e-9)
    assert (tmp_path / "observables_last.ed").read_text() == lines[-1]
    pl = (tmp_path / "parameters_last.ed").read_text()
    want = "".join(O.f15_9(x) for x in [m.xmu, m.beta, *m.uloc[:no], m.ust, m.jh, 0.0, 0.0])
    assert pl == want + "\n"
    info_e, last_e = O.energy_texts(s.ed_get_eimp(), s.ed_get_doubles())
    assert (tmp_path / "energy_info.ed").read_text() == info_e
    assert (tmp_path / "energy_last.ed").read_text() == last_e
    s.close()
