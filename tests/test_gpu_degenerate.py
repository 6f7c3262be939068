"""Degenerate eigenvalues inside a sector, against the oracle.

The reference diagonalises Neigen = min(dim, lanc_nstates_sector) eigenpairs
of every sector even at T=0 and keeps every one within gs_threshold of the
ground energy (ED_DIAG.f90:131,202-214); its sp_eigh (ARPACK) and eigh return
degenerate copies.  Models with two or three identical orbitals have ground
states and excited multiplets that are degenerate inside one sector, both in
sectors small enough for the dense branch (dim <= lanc_dim_threshold) and in
Lanczos sectors (batched and grid-wide).  Bars: kept-state count, sectors and
Z exact; energies 1e-10; observables 1e-9; G(iwn) 1e-8."""
import os

import numpy as np
import pytest

import dmfted
import oracle as O
from test_oracle import degenerate_models

pytestmark = pytest.mark.gpu


def _solver(m, env=None, **kw):
    env = env or {}
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        ul = list(m.uloc) + [0.0] * (3 - len(m.uloc))
        p = dmfted.default_params(norb=m.norb, nbath=m.nbath, nspin=m.nspin, uloc=ul, ust=m.ust,
                                  jh=m.jh, xmu=m.xmu, beta=m.beta, hfmode=int(m.hfmode), **kw)
        s = dmfted.EDSolver(p, hloc=m.hloc)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    return s


def _multiset(energies, sectors, e0):
    return sorted((round(float(e - e0), 8), int(s)) for e, s in zip(energies, sectors))


def _check(s, m, ref, lmats):
    e, secs, z = s.eigenspace()
    ns = m.ns
    rsec = [a * (ns + 1) + b + 1 for _, a, b in ref["states"]]
    ren = [x[0] for x in ref["states"]]
    assert len(e) == len(ren)
    assert _multiset(e, secs, ref["egs"]) == _multiset(ren, rsec, ref["egs"])
    assert np.allclose(np.sort(e), np.sort(ren), rtol=0, atol=1e-10 * max(1.0, abs(ref["egs"])))
    assert abs(z - ref["zeta"]) <= 1e-9 * ref["zeta"]
    ob = s.observables()
    for k in ("dens", "dens_up", "dens_dw", "docc", "magz"):
        assert np.allclose(ob[k], ref["obs"][k], rtol=0, atol=1e-9), k
    gm = s.ed_get_gimp_matsubara()
    for ispin in range(m.nspin):
        for a in range(m.norb):
            dg = np.abs(gm[ispin, ispin, a, a] - ref["gmats"][ispin, a]).max()
            assert dg <= 1e-8, (ispin, a, dg)


@pytest.mark.parametrize("im", [0, 1])
@pytest.mark.parametrize("precision", [dmfted.FP64, dmfted.MIXED])
@pytest.mark.parametrize("path", ["batch", "grid"])
def test_t0_degenerate_ground_states_match_oracle(im, precision, path):
    m, nkeep, _ = degenerate_models()[im]
    env = {"DMFTED_BATCH_MAX_DIM": "0"} if path == "grid" else {}
    s = _solver(m, env, lmats=128, lreal=0, precision=precision)
    s.ed_solve(m.bath_array())
    ref = O.solve_t0(m, lmats=128, nthreads=4)
    assert ref["zeta"] == nkeep
    _check(s, m, ref, 128)
    s.close()


def _ft_model():
    # three identical orbitals: threefold multiplets in sectors (4,3), (2,3),
    # (3,4), (3,2) (dim 300, Lanczos branch) and (4,2), (2,4) (dim 225, dense);
    # 14 states end at a gap of the spectrum
    e = np.zeros((1, 3, 1))
    v = np.full((1, 3, 1), 0.5)
    return O.Model(norb=3, nbath=1, nspin=1, uloc=(3.0, 3.0, 3.0), ust=2.0, jh=0.5, beta=10.0,
                   e=e, v=v)


@pytest.mark.parametrize("path", ["batch", "grid"])
def test_finite_t_degenerate_multiplets_match_oracle(path):
    m = _ft_model()
    env = {"DMFTED_BATCH_MAX_DIM": "0"} if path == "grid" else {}
    s = _solver(m, env, lmats=256, lreal=0, lanc_nstates_total=14)
    s.ed_solve(m.bath_array())
    ref = O.solve_finite_t(m, lmats=256, nstates_total=14, nthreads=4)
    ref = dict(ref, states=[(e, (sec - 1) // 7, (sec - 1) % 7) for e, sec in ref["states"]])
    _check(s, m, ref, 256)
    s.close()


def test_dense_branch_threshold_matches_lanczos_branch():
    # the same finite-T solve with every sector on the dense branch
    # (lanc_dim_threshold above the largest sector) and with none on it
    m = _ft_model()
    out = []
    for thr in (1024, 0):
        s = _solver(m, lmats=128, lreal=0, lanc_nstates_total=14, lanc_dim_threshold=thr)
        s.ed_solve(m.bath_array())
        e, secs, z = s.eigenspace()
        out.append((e, secs, z, s.ed_get_gimp_matsubara(), s.observables()))
        s.close()
    (e1, s1, z1, g1, o1), (e2, s2, z2, g2, o2) = out
    assert _multiset(e1, s1, e1[0]) == _multiset(e2, s2, e1[0])
    assert abs(z1 - z2) <= 1e-9 * z1
    assert np.abs(g1 - g2).max() <= 1e-9
    for k in ("dens", "docc"):
        assert np.allclose(o1[k], o2[k], atol=1e-10)


@pytest.mark.parametrize("nup,ndw,neigen", [(3, 3, 6), (2, 2, 6), (1, 1, 36), (3, 3, 1)])
def test_gs_lanczos_entry_point(nup, ndw, neigen):
    # dmfted_gs_lanczos: the sp_eigh / eigh call of one sector, degenerate
    # copies included, against a dense eigh of the oracle's sector H
    m, _, _ = degenerate_models()[1]
    s = _solver(m)
    s.set_bath(m.bath_array())
    isec = s.sector_index(nup, ndw)
    ev, vec = s.gs_lanczos(isec, neigen)
    hm = O.build_sector(m.ns, nup, ndw)
    H = O.sparse_h(m, hm).toarray()
    w = np.linalg.eigvalsh(H)
    k = min(neigen, hm.size)
    assert len(ev) == k
    assert np.allclose(ev, w[:k], rtol=0, atol=1e-10 * max(1.0, abs(w[0])))
    X = vec.T
    assert np.allclose(X.conj().T @ X, np.eye(k), atol=1e-9)
    assert np.linalg.norm(H @ X - X * ev) <= 1e-8 * max(1.0, abs(w[0]))
    s.close()
