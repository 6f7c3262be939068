"""The CPU restatement (oracle) against independent known answers.

No test, fixture or output file of the reference exists, so the pins are:
the Jordan-Wigner Fock-space construction of tests/golden/pins.npz (dense
spectra per sector), ARPACK (scipy eigsh, the eigensolver family of
SciFortran's sp_eigh), the U=0 and V=0 analytic limits, the particle+hole
sum rule, and finite differences for the chi^2 gradient."""
import itertools

import numpy as np
import pytest
import scipy.sparse.linalg as sla

import oracle as O
from models import golden_models


def test_binomial_matches_exact():
    from math import comb
    for n in range(0, 21):
        for k in range(0, n + 1):
            assert O.binomial(n, k) == comb(n, k)
    assert O.binomial(5, -1) == 0


def _literal_build_sector(ns, nup, ndw):
    # literal transcription of ED_SETUP.f90:880-890 in Python
    out = []
    for idw in range(2 ** ns):
        if bin(idw).count("1") != ndw:
            continue
        for iup in range(2 ** ns):
            if bin(iup).count("1") != nup:
                continue
            out.append(iup + idw * 2 ** ns)
    return np.array(out, np.int32)


@pytest.mark.parametrize("ns,nup,ndw", [(4, 2, 2), (5, 1, 3), (6, 3, 3), (6, 0, 6), (7, 4, 2)])
def test_build_sector_literal(ns, nup, ndw):
    assert np.array_equal(O.build_sector(ns, nup, ndw), _literal_build_sector(ns, nup, ndw))


def test_binary_search_semantics():
    a = O.build_sector(6, 3, 2)
    for i in [0, 1, 7, len(a) // 2, len(a) - 1]:
        assert O.binary_search(a, int(a[i])) == i + 1
    assert O.binary_search(a, -5) == 0
    assert O.binary_search(a, int(a[-1]) + 1) == 0
    assert O.binary_search(np.zeros(0, np.int32), 3) == 0


def test_sector_tables():
    t = O.sector_tables(1, 3)
    ns = 4
    assert t["getdim"][t["getsector"][2 * (ns + 1) + 2] - 1] == 36
    # c^+ up of sector (nup, ndw) is (nup+1, ndw); c dw is (nup, ndw-1)
    for s in range(1, (ns + 1) ** 2 + 1):
        nup, ndw = t["getnup"][s - 1], t["getndw"][s - 1]
        cdg = t["getcdgsector"][2 * (s - 1)]
        if nup < ns:
            assert (t["getnup"][cdg - 1], t["getndw"][cdg - 1]) == (nup + 1, ndw)
        else:
            assert cdg == 0
        cdw = t["getcsector"][2 * (s - 1) + 1]
        if ndw > 0:
            assert (t["getnup"][cdw - 1], t["getndw"][cdw - 1]) == (nup, ndw - 1)
    assert list(O.sector_tables(2, 3)["getbathstride"]) == [3, 6, 4, 7, 5, 8]


@pytest.mark.parametrize("case", range(8))
def test_sector_spectra_against_jordan_wigner(case):
    # cases 6 and 7 carry the Jhflag spin-exchange and pair-hopping terms
    model, sectors, low = golden_models()[case]
    ns = model.ns
    for (nup, ndw), ref in zip(sectors, low):
        hm = O.build_sector(ns, int(nup), int(ndw))
        H = O.sparse_h(model, hm).toarray()
        assert np.allclose(H, H.conj().T, atol=1e-14)
        w = np.linalg.eigvalsh(H)[:4]
        ref = ref[~np.isnan(ref)]
        assert np.allclose(w[:ref.size], ref, atol=1e-11), (nup, ndw)


def test_hxv_equals_explicit_matrix():
    model = golden_models()[3][0]
    hm = O.build_sector(model.ns, 2, 2)
    H = O.sparse_h(model, hm)
    rng = np.random.default_rng(1)
    v = rng.normal(size=hm.size) + 1j * rng.normal(size=hm.size)
    assert np.abs(O.hxv(model, hm, v) - H @ v).max() < 1e-13
    assert np.abs(O.hxv(model, hm, v, nthreads=4) - H @ v).max() < 1e-13


def test_lanczos_gs_against_dense_and_arpack():
    m = O.seeded_model(3, nbath=6, u=2.0)
    hm = O.build_sector(m.ns, 3, 4)
    H = O.sparse_h(m, hm)
    w = np.linalg.eigvalsh(H.toarray())
    e0, psi, n = O.lanczos_gs(m, hm)
    assert abs(e0 - w[0]) < 1e-10 * abs(w[0])
    ea = sla.eigsh(H, k=1, which="SA", tol=1e-13)[0][0]
    assert abs(e0 - ea) < 1e-10 * abs(ea)
    r = H @ psi - e0 * psi
    assert np.linalg.norm(r) < 1e-6


def test_tql2_against_numpy():
    rng = np.random.default_rng(5)
    n = 40
    d = rng.normal(size=n)
    e = np.concatenate([[0.0], rng.normal(size=n - 1)])
    T = np.diag(d) + np.diag(e[1:], 1) + np.diag(e[1:], -1)
    w, V = np.linalg.eigh(T)
    dd, Z, ierr = O.tql2(d, e)
    assert ierr == 0
    assert np.allclose(dd, w, atol=1e-12)
    assert np.allclose(np.abs(Z[0]), np.abs(V[0]), atol=1e-10)


def test_u0_limit_energy_and_sigma():
    z = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden",
                                           "pins.npz"))
    e, v = z["u0_e"], z["u0_v"]
    m = O.Model(norb=1, nbath=5, nspin=1, uloc=(0.0, 0.0, 0.0), e=e[None, None], v=v[None, None])
    r = O.solve_sector_t0(m, 3, 3, lmats=128)
    assert abs(r["e0"] - 2 * z["u0_levels"][:3].sum()) < 1e-10
    # U=0: G = 1/(iw - Delta) exactly, so Sigma = 0
    assert np.abs(r["smats"]).max() < 1e-8


def test_atomic_limit_green_function():
    # V=0 (Nbath bath levels decoupled), half filling, HFMODE: G = 1/2[1/(iw-U/2)+1/(iw+U/2)]
    u = 2.0
    m = O.Model(norb=1, nbath=2, nspin=1, uloc=(u, 0, 0), e=np.array([[[-0.5, 0.5]]]),
                v=np.zeros((1, 1, 2)))
    r = O.solve_sector_t0(m, 2, 1, lmats=64)  # imp singly occupied (up), bath has one up+dw... 
    wm = r["wm"]
    # the impurity up electron can be removed (hole) at -U/2 or a dw added (particle) at +U/2
    g = r["gmats"][0, 0]
    assert np.all(np.isfinite(g))
    # sum rule: particle + hole weights add up to 1
    assert abs(sum(c["norm2"] for c in r["chains"]) - 1.0) < 1e-12


def test_sum_rule_and_tail():
    m = O.seeded_model(11, nbath=5, u=3.0)
    r = O.solve_sector_t0(m, 3, 3, lmats=2000)
    assert abs(sum(c["norm2"] for c in r["chains"]) - 1.0) < 1e-12
    g = r["gmats"][0, 0]
    assert abs(g[-1] * 1j * r["wm"][-1] - 1.0) < 2e-3


def test_chi2_gradient_finite_difference():
    rng = np.random.default_rng(9)
    nb = 6
    a = np.concatenate([rng.uniform(-1, 1, nb), 0.5 + rng.uniform(-0.1, 0.1, nb)])
    x = O.matsubara(100.0, 300)
    g = O.delta_bath(a[:nb] + 0.02, a[nb:] * 1.01, 1j * x)
    for cw in (0, 1, 2, 3):
        w = O.cg_weights(cw, x)
        c2, gr = O.chi2_delta(a, x, g, w)
        h = 1e-6
        fd = np.array([(O.chi2_delta(a + h * u, x, g, w, False) - O.chi2_delta(a - h * u, x, g, w,
                                                                                 False)) / (2 * h)
                       for u in np.eye(a.size)])
        assert np.abs(gr - fd).max() <= 1e-6 * np.abs(gr).max() + 1e-12


# ------------------------------------------------ T=0 state selection ---
def degenerate_models():
    """Models whose ground state is degenerate inside one sector (two identical
    orbitals): (model, kept-state count, sectors holding them)."""
    out = []
    # (a) U = Ust, Jh = 0, one bath site per orbital: (3,3) holds four ground
    # states (dim 16, dense branch), (2,4) and (4,2) one each
    e = np.array([[[-0.8287], [-0.8287]]])
    v = np.array([[[0.4474], [0.4474]]])
    out.append((O.Model(norb=2, nbath=1, nspin=1, uloc=(3.0, 3.0, 0.0), ust=3.0, jh=0.0, e=e, v=v),
                6, {(3, 3): 4, (2, 4): 1, (4, 2): 1}))
    # (b) U = 0, symmetric bath of two sites per orbital: a zero-energy
    # level per orbital and spin, 16 ground states over nine sectors, four of
    # them in (3,3) (dim 400, Lanczos branch)
    e = np.array([[[-0.6, 0.6], [-0.6, 0.6]]])
    v = np.array([[[0.5, 0.5], [0.5, 0.5]]])
    cnt = {(a, b): (2 if a == 3 else 1) * (2 if b == 3 else 1) for a in (2, 3, 4) for b in (2, 3, 4)}
    out.append((O.Model(norb=2, nbath=2, nspin=1, uloc=(0.0, 0.0, 0.0), e=e, v=v), 16, cnt))
    return out


@pytest.mark.parametrize("im", [0, 1])
def test_t0_keeps_degenerate_states_inside_a_sector(im):
    m, nkeep, where = degenerate_models()[im]
    r = O.solve_t0(m, lmats=64, nthreads=4)
    assert r["zeta"] == nkeep and len(r["states"]) == nkeep
    got = {}
    for e, a, b in r["states"]:
        got[(a, b)] = got.get((a, b), 0) + 1
        assert abs(e - r["egs"]) <= 1e-9
    assert got == where
    # the kept vectors of one sector are orthonormal eigenvectors
    for (a, b), n in where.items():
        vs = np.array([p for p, s in zip(r["psis"], r["states"]) if (s[1], s[2]) == (a, b)])
        assert np.allclose(vs @ vs.T, np.eye(n), atol=1e-10)
    # particle + hole weights add up to one per (orbital, spin) and state
    assert abs(sum(c["norm2"] for c in r["chains"]) - nkeep * m.norb) < 1e-10


@pytest.mark.parametrize("im", [0, 1])
def test_t0_degenerate_equals_low_temperature_limit(im):
    # The T=0 average over the whole degenerate ground manifold (Z = count) is
    # the beta -> infinity limit of the thermal average: at beta = 1000 the
    # finite-temperature pipeline (a separate code path: every sector's
    # spectrum, es_add_state's capped list, Boltzmann weights) gives the same
    # observables and G(iwn), the excited states' weights being exp(-500).
    import dataclasses
    m, nkeep, _ = degenerate_models()[im]
    m = dataclasses.replace(m, beta=1000.0)
    r = O.solve_t0(m, lmats=128, nthreads=4)
    f = O.solve_finite_t(m, lmats=128, nstates_total=24, nthreads=4)
    assert abs(f["zeta"] - nkeep) < 1e-9  # beta * (spread of the copies, ~1e-14)
    for k in ("dens", "docc", "magz"):
        assert np.allclose(r["obs"][k], f["obs"][k], atol=1e-9), k
    assert np.abs(r["gmats"] - f["gmats"]).max() < 1e-9
    if im == 0:
        # one state per sector (the selection without the in-sector partners)
        # is a different, wrong answer here
        one = O.solve_t0(m, nstates_sector=1, dim_threshold=0, lmats=128, nthreads=4)
        assert one["zeta"] < nkeep
        assert np.abs(one["gmats"] - f["gmats"]).max() > 1e-4


def test_t0_single_sector_matches_sector_solve():
    m = O.seeded_model(11, nbath=5, u=3.0)
    a = O.solve_t0(m, sectors=[(3, 3)], lmats=256)
    b = O.solve_sector_t0(m, 3, 3, lmats=256)
    assert a["zeta"] == 1.0
    assert abs(a["e0"] - b["e0"]) < 1e-10 * abs(b["e0"])
    assert np.abs(a["gmats"] - b["gmats"]).max() < 1e-8


# ---- the self-consistency around the solve: fit, local G, Weiss field -------
def _fit_problem(seed=5, nbath=9, L=1000, beta=100.0, noise=1e-4):
    rng = np.random.default_rng(seed)
    wm = O.matsubara(beta, L)
    e = rng.uniform(-1.0, 1.0, nbath)
    v = 0.5 + rng.uniform(-0.1, 0.1, nbath)
    z = noise * (rng.normal(size=L) + 1j * rng.normal(size=L))
    return rng, wm, e, v, z


def test_weiss_chi2_gradient_finite_difference():
    rng, wm, e, v, z = _fit_problem()
    g = 1.0 / (1j * wm + 0.1 - O.delta_bath(e, v, 1j * wm)) + z
    w = O.cg_weights(3, wm)
    x = np.concatenate([e, v]) * (1 + 0.05 * rng.normal(size=e.size * 2))
    c, gr = O.chi2_model(x, wm, g, w, weiss=True, zc=0.1)
    h = 1e-6
    fd = np.array([(O.chi2_model(x + h * d, wm, g, w, True, 0.1, False) -
                    O.chi2_model(x - h * d, wm, g, w, True, 0.1, False)) / (2 * h)
                   for d in np.eye(x.size)])
    assert np.abs(fd - gr).max() <= 1e-6 * np.abs(gr).max()
    # the delta scheme is the reference's grad_chi2_delta_normal_normal
    c2, g2 = O.chi2_model(x, wm, g, w, weiss=False)
    c3, g3 = O.chi2_delta(x, wm, g, w)
    assert abs(c2 - c3) <= 1e-14 * c3 and np.abs(g2 - g3).max() <= 1e-14 * np.abs(g3).max()


@pytest.mark.parametrize("weiss", [False, True])
def test_cg_fit_reaches_the_minimum(weiss):
    """The restated fmin_cg (Polak-Ribiere, Brent line searches) from a start
    near the answer ends at the minimum an independent quasi-Newton search
    finds (cg_weight 0, the reference default)."""
    from scipy.optimize import minimize
    rng, wm, e, v, z = _fit_problem()
    d = O.delta_bath(e, v, 1j * wm)
    g = (1.0 / (1j * wm - d) if weiss else d) + z
    w = O.cg_weights(0, wm)
    a0 = np.concatenate([e, v]) * (1 + 0.05 * rng.normal(size=2 * e.size))
    a, f, it, st = O.cg_fit(a0, wm, g, w, weiss=weiss, zc=0.0)
    assert st == 0 and it < 500
    assert abs(f - O.chi2_model(a, wm, g, w, weiss, 0.0, False)) <= 1e-14 * f
    r = minimize(lambda x: O.chi2_model(x, wm, g, w, weiss, 0.0)[0], a0,
                 jac=lambda x: O.chi2_model(x, wm, g, w, weiss, 0.0)[1], method="BFGS",
                 options=dict(gtol=1e-14, maxiter=50000))
    # fmin_cg stops on the relative change of chi2 (cg_ftol = 1e-5): its value
    # lies within a small factor of the true minimum, far below the start
    assert r.fun <= f <= 2.0 * r.fun + 1e-12
    assert f < 1e-2 * O.chi2_model(a0, wm, g, w, weiss, 0.0, False)


def test_bethe_gloc_and_delta_self_consistency():
    """On the semicircular grid the local G of Sigma = 0 obeys the Bethe
    relation Delta = (D/2)^2 G_loc (to the grid's discretisation error), and
    the Weiss and Delta routes agree: 1/G0 = i w + xmu - Delta."""
    he, wt = O.bethe_dos(4000, 1.0)
    wm = O.matsubara(100.0, 256)
    sig = np.zeros(wm.size, np.complex128)
    g = O.gloc_diag(he, wt, wm, 0.0, sig)
    d = O.weiss_diag(g, sig, wm, 0.0, 0.0, weiss=False)
    assert np.abs(d - 0.25 * g).max() < 2e-3
    g0 = O.weiss_diag(g, sig, wm, 0.0, 0.0, weiss=True)
    assert np.abs(1.0 / g0 - (1j * wm - d)).max() < 1e-12
    assert abs(wt.sum() - 1.0) < 1e-3


@pytest.mark.parametrize("norb,nbath,nup,ndw", [(1, 7, 4, 4), (1, 5, 3, 2), (2, 3, 4, 3)])
def test_factored_cpu_hxv_equals_map_hxv(norb, nbath, nup, ndw):
    """The "best CPU" baseline (the up/down-factored FP64 product on the host)
    is the same operator as the reference-faithful map H*v."""
    m = O.seeded_model(3, norb=norb, nbath=nbath, u=2.0, beta=100.0)
    F = O.FactoredHxv(m, nup, ndw, nthreads=2)
    x = np.random.default_rng(1).normal(size=F.hmap.size)
    ref = O.hxv(m, F.hmap, x.astype(np.complex128), nthreads=2).real
    assert np.abs(F(x) - ref).max() <= 1e-13 * np.abs(ref).max()
