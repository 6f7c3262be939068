"""The workload configurations at their full sizes against oracle fixtures
(tests/golden/config_pins.npz, written by tests/golden/make_config_pins.py).

  cfg2  Ns=12, sector 6/6 (dim 853,776), T=0 ground state + G(iwn)
  cfg3  Ns=14, sector 7/7 (dim 11,778,624): one H*v, then the same solve
  cfg4  Norb=2, Ns=10, Nspin=2, beta=50: all 121 sectors, 16 kept states

Both precision forms are held to the FP64 bars: |dE0|/|E0| <= 1e-10,
observables 1e-9, max|dG(iwn)| <= 1e-8; Sigma(iwn) within 1e-8 * max(1, wn^2)
(Sigma = G0^-1 - G^-1 carries the error of G times 1/|G|^2 ~ wn^2 at high
frequency); the H*v
checks within 1e-13 relative; the leading chain coefficients of the FP64
form within 1e-10."""
import os

import numpy as np
import pytest

import dmfted

pytestmark = pytest.mark.gpu

PINS = os.path.join(os.path.dirname(__file__), "golden", "config_pins.npz")
LMATS = 4096


def pins():
    return np.load(PINS)


def need(z, key):
    if key not in z:
        pytest.fail(f"{key} missing from config_pins.npz (run tests/golden/make_config_pins.py)")


def single_orbital_bath(nbath, seed):
    # seeded_model's draws: e ~ U[-1,1], V = 0.5 + U[-0.1,0.1]
    rng = np.random.default_rng(seed)
    e = rng.uniform(-1.0, 1.0, size=(1, nbath))
    v = 0.5 + rng.uniform(-0.1, 0.1, size=(1, nbath))
    return np.concatenate([e.reshape(-1), v.reshape(-1)])


def t0_case(prefix, nbath, seed, nup, precision):
    z = pins()
    need(z, prefix + "_e0")
    p = dmfted.default_params(nbath=nbath, uloc=[3.0], beta=100.0, lmats=LMATS, lreal=0,
                              lanc_nstates_sector=1, precision=precision)
    s = dmfted.EDSolver(p)
    isec = s.sector_index(nup, nup)
    s.ed_solve(single_orbital_bath(nbath, seed), sectors=[isec])
    e0 = float(z[prefix + "_e0"])
    assert abs(s.egs() - e0) <= 1e-10 * abs(e0), (s.egs(), e0)
    ob = s.observables()
    for k in ("dens", "dens_up", "dens_dw", "docc", "magz"):
        assert np.allclose(ob[k], z[prefix + "_" + k], rtol=0, atol=1e-9), k
    g = s.ed_get_gimp_matsubara()[0, 0, 0, 0]
    dg = np.abs(g - z[prefix + "_gmats"]).max()
    assert dg <= 1e-8, dg
    wm = np.pi / 100.0 * (2 * np.arange(1, LMATS + 1) - 1)
    sg = s.ed_get_sigma_matsubara()[0, 0, 0, 0]
    ds = np.abs(sg - z[prefix + "_smats"]) / np.maximum(1.0, wm ** 2)
    assert ds.max() <= 1e-8, ds.max()
    s.close()
    return dg


@pytest.mark.parametrize("precision", [dmfted.FP64, dmfted.MIXED])
def test_cfg2_solve_matches_oracle(precision):
    t0_case("cfg2", 11, 2, 6, precision)


def test_cfg2_chain_coefficients():
    # the particle chain of the solver's ground state through the
    # sp_lanc_tridiag entry point against the oracle's chain
    z = pins()
    need(z, "cfg2_alpha_p")
    p = dmfted.default_params(nbath=11, uloc=[3.0], beta=100.0, lmats=16, lreal=0,
                              lanc_nstates_sector=1)
    s = dmfted.EDSolver(p)
    s.set_bath(single_orbital_bath(11, 2))
    isec = s.sector_index(6, 6)
    ev, vec = s.gs_lanczos(isec, 1)
    assert abs(ev[0] - float(z["cfg2_e0"])) <= 1e-10 * abs(ev[0])
    # c^+_{1,up} |GS> into sector 7/6: the impurity is bit 0 of the up word
    import oracle as O
    hi = O.build_sector(12, 6, 6)
    hj = O.build_sector(12, 7, 6)
    n2, vv = O.gf_vvinit(True, 1, hi, hj, vec[0])
    assert abs(n2 - float(z["cfg2_norm2_p"])) <= 1e-10
    a, b, _ = s.lanc_tridiag(s.sector_index(7, 6), vv / np.sqrt(n2), 200)
    # The ground state's overall sign does not change the chain.  The two
    # ground states differ by their convergence error (~1e-12), which the
    # recurrence amplifies step by step (1e-5 by step 12 here): the leading
    # coefficients are compared, G(iwn) -- which weighs coefficient k less the
    # deeper it is -- at the full length in test_cfg2_solve_matches_oracle.
    assert np.abs(a[:8] - z["cfg2_alpha_p"][:8]).max() <= 1e-10
    assert np.abs(b[:8] - z["cfg2_beta_p"][:8]).max() <= 1e-10
    s.close()


def test_cfg3_hxv_matches_oracle():
    import torch
    z = pins()
    need(z, "cfg3_hv_wHv")
    p = dmfted.default_params(nbath=13, uloc=[3.0], beta=100.0, lmats=16, lreal=0)
    s = dmfted.EDSolver(p)
    s.set_bath(single_orbital_bath(13, 1))
    isec = s.sector_index(7, 7)
    s.setup_hv_sector(isec)
    dim = s.sector_dim(isec)
    rng = np.random.default_rng(123)
    v = rng.uniform(-1.0, 1.0, dim)
    w = rng.uniform(-1.0, 1.0, dim)
    x = torch.from_numpy(v).cuda()
    y = torch.empty_like(x)
    torch.cuda.synchronize()
    dmfted._ck(dmfted.lib().dmfted_hxv_device_f64(s.ctx, x.data_ptr(), y.data_ptr(), 1))
    s.time_hxv(fp32=False, warmup=0, reps=1)  # drains the library stream
    hv = y.cpu().numpy()
    norm = float(z["cfg3_hv_norm"])
    assert abs(np.linalg.norm(hv) - norm) <= 1e-13 * norm
    assert abs(w @ hv - float(z["cfg3_hv_wHv"])) <= 1e-13 * norm * np.linalg.norm(w)
    assert np.abs(hv[z["cfg3_hv_idx"]] - z["cfg3_hv_val"]).max() <= 1e-13 * np.abs(hv).max()
    s.close()


@pytest.mark.parametrize("precision", [dmfted.FP64, dmfted.MIXED])
def test_cfg3_solve_matches_oracle(precision):
    t0_case("cfg3", 13, 1, 7, precision)


@pytest.mark.parametrize("precision", [dmfted.FP64, dmfted.MIXED])
def test_cfg4_finite_t_matches_oracle(precision):
    z = pins()
    need(z, "cfg4_e")
    rng = np.random.default_rng(4)
    e = rng.uniform(-1.5, 1.5, size=(2, 4))
    v = 0.4 + rng.uniform(-0.1, 0.1, size=(2, 4))
    bath = np.concatenate([e.reshape(-1), e.reshape(-1), v.reshape(-1), v.reshape(-1)])
    p = dmfted.default_params(norb=2, nbath=4, nspin=2, uloc=[3.0, 3.0], ust=2.0, jh=0.5,
                              beta=50.0, lmats=LMATS, lreal=0, lanc_nstates_total=16,
                              precision=precision)
    s = dmfted.EDSolver(p)
    s.ed_solve(bath)
    en, secs, zeta = s.eigenspace()
    re, rs = z["cfg4_e"], z["cfg4_sector"]
    assert len(en) == len(re)
    # spin doublets have equal energies: compare (energy, sector) as multisets
    key = lambda E, S: sorted((round(float(x - re[0]), 8), int(y)) for x, y in zip(E, S))
    assert key(en, secs) == key(re, rs)
    assert np.allclose(np.sort(en), np.sort(re), rtol=0, atol=1e-10 * np.abs(re).max())
    assert abs(zeta - float(z["cfg4_zeta"])) <= 1e-10 * float(z["cfg4_zeta"])
    ob = s.observables()
    for k in ("dens", "dens_up", "dens_dw", "docc", "magz"):
        assert np.allclose(ob[k], z["cfg4_" + k], rtol=0, atol=1e-9), k
    g = s.ed_get_gimp_matsubara()
    for ispin in range(2):
        for a in range(2):
            dg = np.abs(g[ispin, ispin, a, a] - z["cfg4_gmats"][ispin, a]).max()
            assert dg <= 1e-8, (ispin, a, dg)
    s.close()
