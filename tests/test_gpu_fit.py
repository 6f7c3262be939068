"""The self-consistency around the solve on the device against the oracle:
the bath fit (ed_chi2_fitgf / fmin_cg restated), the local Green's function on
a density-of-states grid (dmft_gloc_matsubara) and the Weiss field or
hybridisation (dmft_weiss / dmft_delta), and one whole iteration of the
Bethe-lattice DMFT loop (drivers/ed_hm_bethe.f90:53-88).

Bars: the lattice sums and the Weiss field within 1e-12 relative (the same
sums in the same order); a fit that converges within cg_niter ends at the
oracle's point: chi2 within 1e-6 relative, parameters within 1e-5 (both
minimisers take the same steps up to the rounding of the frequency sums).
On a flat landscape the rounding of the frequency sums alone sends two
conjugate-gradient paths apart (both stop by the reference's test a few parts
in 1e3 apart in chi2); the loop test holds that case to 2e-2."""
import numpy as np
import pytest

import dmfted
import oracle as O
from dmfted import bethe

pytestmark = pytest.mark.gpu


def fit_problem(seed=5, nbath=9, L=1000, beta=100.0, noise=1e-4, weiss=False):
    rng = np.random.default_rng(seed)
    wm = O.matsubara(beta, L)
    e = rng.uniform(-1.0, 1.0, nbath)
    v = 0.5 + rng.uniform(-0.1, 0.1, nbath)
    d = O.delta_bath(e, v, 1j * wm)
    g = (1.0 / (1j * wm + 0.2 - d) if weiss else d) + noise * (
        rng.normal(size=L) + 1j * rng.normal(size=L))
    a0 = np.concatenate([e, v]) * (1 + 0.05 * rng.normal(size=2 * nbath))
    return wm, g, a0


@pytest.fixture(scope="module")
def ctx():
    with dmfted.EDSolver(dmfted.default_params(nbath=9, beta=100.0, lmats=1000, lreal=0)) as s:
        yield s


@pytest.mark.parametrize("weiss", [False, True])
def test_cg_fit_matches_oracle(ctx, weiss):
    wm, g, a0 = fit_problem(weiss=weiss)
    w = O.cg_weights(0, wm)
    scheme = dmfted.CG_WEISS if weiss else dmfted.CG_DELTA
    a, c2, it = ctx.cg_fit_batch(a0, wm, g, w, scheme=scheme, zc=0.2)
    ar, fr, itr, st = O.cg_fit(a0, wm, g, w, weiss=weiss, zc=0.2)
    assert st == 0 and itr < 500
    assert abs(c2[0] - fr) <= 1e-6 * fr, (c2[0], fr)
    assert np.abs(a[0] - ar).max() <= 1e-5 * np.abs(ar).max()
    assert abs(int(it[0]) - itr) <= 2
    # the returned chi2 is the chi2 of the returned point
    assert abs(c2[0] - O.chi2_model(a[0], wm, g, w, weiss, 0.2, False)) <= 1e-12 * c2[0]


def test_cg_fit_batch_of_starts(ctx):
    """Many start points at once (one CTA each): every fit equals the same fit
    run alone, and each ends below its start."""
    wm, g, a0 = fit_problem()
    w = O.cg_weights(0, wm)
    rng = np.random.default_rng(11)
    starts = a0[None, :] * (1 + 0.03 * rng.normal(size=(64, a0.size)))
    a, c2, it = ctx.cg_fit_batch(starts, wm, g, w, scheme=dmfted.CG_DELTA)
    for b in (0, 17, 63):
        a1, c1, _ = ctx.cg_fit_batch(starts[b], wm, g, w, scheme=dmfted.CG_DELTA)
        assert np.array_equal(a1[0], a[b]) and c1[0] == c2[b]
    c0 = np.array([O.chi2_model(s, wm, g, w, False, 0.0, False) for s in starts])
    assert np.all(c2 < c0)


def test_gloc_and_weiss_match_oracle():
    p = dmfted.default_params(norb=2, nbath=3, nspin=2, beta=50.0, lmats=512, lreal=0, xmu=0.3)
    hloc = np.zeros((2, 2, 2, 2), np.complex128, order="F")
    hloc[0, 0, 1, 1] = hloc[1, 1, 1, 1] = 0.25
    with dmfted.EDSolver(p, hloc=hloc) as s:
        rng = np.random.default_rng(2)
        sig = np.zeros((2, 2, 2, 2, 512), np.complex128, order="F")
        for i in range(2):
            for a in range(2):
                sig[i, i, a, a] = rng.normal(size=512) * 0.3 + 1j * (-np.abs(rng.normal(size=512)))
        he = np.stack([np.linspace(-1, 1, 300), np.linspace(-2, 2, 300)])
        wt = np.full(300, 1.0 / 300)
        gl = s.gloc_matsubara_diag(he, wt, sig)
        wm = O.matsubara(50.0, 512)
        for i in range(2):
            for a in range(2):
                ref = O.gloc_diag(he[a], wt, wm, 0.3, sig[i, i, a, a])
                assert np.abs(gl[i, i, a, a] - ref).max() <= 1e-12 * np.abs(ref).max()
                for weiss in (True, False):
                    out = s.get_weiss(gl, sig, dmfted.CG_WEISS if weiss else dmfted.CG_DELTA)
                    r2 = O.weiss_diag(ref, sig[i, i, a, a], wm, 0.3, hloc[i, i, a, a].real, weiss)
                    assert np.abs(out[i, i, a, a] - r2).max() <= 1e-12 * np.abs(r2).max()
        assert np.abs(gl[0, 0, 0, 1]).max() == 0.0 and np.abs(gl[0, 1, 0, 0]).max() == 0.0


def test_gloc_real_axis_matches_oracle():
    p = dmfted.default_params(norb=1, nbath=3, nspin=1, beta=50.0, lmats=64, lreal=400, xmu=0.1,
                              wini=-3.0, wfin=3.0, eps=0.05)
    with dmfted.EDSolver(p) as s:
        rng = np.random.default_rng(4)
        sig = np.zeros((1, 1, 1, 1, 400), np.complex128, order="F")
        sig[0, 0, 0, 0] = 0.2 * rng.normal(size=400) - 0.1j * np.abs(rng.normal(size=400))
        he, wt = bethe.bethe_dos(500, 1.0)
        gr = s.gloc_realaxis_diag(he, wt, sig)
        w = np.linspace(-3.0, 3.0, 400)
        z = w + 0.05j + 0.1 - sig[0, 0, 0, 0]
        ref = np.zeros(400, np.complex128)
        for k in range(he.size):
            ref = ref + (1.0 / (z - he[k])) * wt[k]
        assert np.abs(gr[0, 0, 0, 0] - ref).max() <= 1e-12 * np.abs(ref).max()


def test_chi2_fitgf_per_orbital_matches_oracle():
    """ed_chi2_fitgf on a two-orbital bath: each orbital's fit of spin 1 equals
    the oracle's fit of that orbital; the spin-2 parameters stay as they were."""
    p = dmfted.default_params(norb=2, nbath=4, nspin=2, beta=50.0, lmats=800, lreal=0,
                              cg_scheme=dmfted.CG_WEISS, lfit=600, cg_weight=1)
    nb = dmfted.get_bath_dimension(p)
    rng = np.random.default_rng(9)
    bath = np.concatenate([rng.uniform(-1, 1, nb // 2), 0.4 + rng.uniform(-0.1, 0.1, nb // 2)])
    wm = O.matsubara(50.0, 800)
    fg = np.zeros((2, 2, 2, 2, 800), np.complex128, order="F")
    targets = []
    for a in range(2):
        e = rng.uniform(-1, 1, 4)
        v = 0.4 + rng.uniform(-0.1, 0.1, 4)
        t = 1.0 / (1j * wm - O.delta_bath(e, v, 1j * wm))
        fg[0, 0, a, a] = t
        targets.append(t)
    with dmfted.EDSolver(p) as s:
        new, it, c2 = s.ed_chi2_fitgf(fg, bath, ispin=1)
    half = nb // 2
    w = O.cg_weights(1, wm[:600])
    for a in range(2):
        io = np.arange(4) + a * 4
        a0 = np.concatenate([bath[io], bath[half + io]])
        ar, fr, itr, st = O.cg_fit(a0, wm[:600], targets[a][:600], w, weiss=True, zc=0.0)
        assert abs(c2[a] - fr) <= 1e-6 * max(fr, 1e-300) + 1e-14, (a, c2[a], fr)
        got = np.concatenate([new[io], new[half + io]])
        assert np.abs(got - ar).max() <= 1e-5 * np.abs(ar).max()
    spin2 = np.arange(8, 16)
    assert np.array_equal(new[spin2], bath[spin2])
    assert np.array_equal(new[half + spin2], bath[half + spin2])


def test_bethe_dmft_iteration_matches_oracle():
    """One iteration of the Bethe loop at the small configuration (Ns=8, U=2,
    half filling, beta=100, the ground state of sector 4/4): the solve, Sigma, G_loc
    on the 500-point semicircle, the Weiss field and the fitted bath against
    the same chain of oracle steps."""
    m = O.seeded_model(1, norb=1, nbath=7, u=2.0, beta=100.0)
    p = dmfted.default_params(norb=1, nbath=7, uloc=[2.0], beta=100.0, lmats=1024, lreal=0,
                              lanc_nstates_sector=1)
    bath = m.bath_array()
    he, wt = bethe.bethe_dos(500, 1.0)
    with dmfted.EDSolver(p) as s:
        new, weiss, c2 = bethe.dmft_step(s, bath, he, wt, sectors=[s.sector_index(4, 4)])
        smats = s.ed_get_sigma_matsubara()[0, 0, 0, 0]
    ref = O.solve_t0(m, sectors=[(4, 4)], nstates_sector=1, lmats=1024, nthreads=4)
    wm = O.matsubara(100.0, 1024)
    assert np.all(np.abs(smats - ref["smats"][0, 0]) <= 1e-8 * np.maximum(1.0, wm ** 2))
    gl = O.gloc_diag(he, wt, wm, 0.0, ref["smats"][0, 0])
    wr = O.weiss_diag(gl, ref["smats"][0, 0], wm, 0.0, 0.0, weiss=True)
    assert np.abs(weiss[0, 0, 0, 0] - wr).max() <= 1e-7
    # the fit of this target from the model's bath: this landscape is flat
    # near its minimum, where the rounding of the frequency sums already sends
    # the two conjugate-gradient paths apart; both stop by the reference's
    # test, within a per cent of each other and far below the start
    xd = wm[:1000]
    tg = weiss[0, 0, 0, 0, :1000]
    w = O.cg_weights(0, xd)
    ar, fr, itr, st = O.cg_fit(bath, xd, tg, w, weiss=True, zc=0.0)
    assert abs(c2[0][0] - O.chi2_model(new, xd, tg, w, True, 0.0, False)) <= 1e-12 * fr
    assert abs(c2[0][0] - fr) <= 2e-2 * fr, (c2[0][0], fr)
    assert c2[0][0] < 1e-2 * O.chi2_model(bath, xd, tg, w, True, 0.0, False)


def test_bethe_dmft_loop_converges_to_a_self_consistent_solution():
    """The whole loop of drivers/ed_hm_bethe.f90:53-88 (dmft_loop) at the small
    configuration (Ns=8, U=2, half filling, the ground state of sector 4/4):
    it reaches the reference's convergence test (relative change of the Weiss
    field below 1e-5) within the iteration budget, and its fixed point is
    self-consistent: the impurity G equals the local G built from the same
    Sigma to the bath-fit accuracy (Nbath=7).  At the converged bath the
    solve's Sigma and the Weiss field agree with the oracle's chain of steps,
    as in the one-iteration test above."""
    m = O.seeded_model(1, norb=1, nbath=7, u=2.0, beta=100.0)
    p = dmfted.default_params(norb=1, nbath=7, uloc=[2.0], beta=100.0, lmats=1024, lreal=0,
                              lanc_nstates_sector=1)
    he, wt = bethe.bethe_dos(500, 1.0)
    wm = O.matsubara(100.0, 1024)
    with dmfted.EDSolver(p) as s:
        sec = [s.sector_index(4, 4)]
        bath, nit = bethe.dmft_loop(s, m.bath_array(), nloop=80, wmixing=0.5, dmft_error=1e-5,
                                    sectors=sec)
        assert nit < 80, "the loop did not converge"
        s.ed_solve(bath, sectors=sec)
        gimp = s.ed_get_gimp_matsubara()[0, 0, 0, 0]
        smats = s.ed_get_sigma_matsubara()[0, 0, 0, 0]
        gloc = s.gloc_matsubara_diag(he, wt, s.ed_get_sigma_matsubara())[0, 0, 0, 0]
        weiss = s.get_weiss(s.gloc_matsubara_diag(he, wt, s.ed_get_sigma_matsubara()),
                            s.ed_get_sigma_matsubara(), None)[0, 0, 0, 0]
    # self-consistency G_imp = G_loc on the fitted frequencies
    rel = np.abs(gimp[:1000] - gloc[:1000]).max() / np.abs(gloc[:1000]).max()
    assert rel < 5e-3, rel
    # the converged bath through the oracle's steps
    mc = O.seeded_model(1, norb=1, nbath=7, u=2.0, beta=100.0)
    mc.e[0, 0], mc.v[0, 0] = bath[:7], bath[7:]
    ref = O.solve_t0(mc, sectors=[(4, 4)], nstates_sector=1, lmats=1024, nthreads=4)
    assert np.all(np.abs(smats - ref["smats"][0, 0]) <= 1e-8 * np.maximum(1.0, wm ** 2))
    gl = O.gloc_diag(he, wt, wm, 0.0, ref["smats"][0, 0])
    assert np.abs(gloc - gl).max() <= 1e-8
    wr = O.weiss_diag(gl, ref["smats"][0, 0], wm, 0.0, 0.0, weiss=True)
    assert np.abs(weiss - wr).max() <= 1e-7
