"""The global-memory H*v (k_hxv_global) that serves sectors whose columns do
not fit in shared memory (DimUp x 16 bytes above 200 KB: Ns >= 16 near half
filling), against the oracle.

Checks:
  - forced on small sectors (DMFTED_HXV_KERNEL=3), the product equals the
    oracle's directMatVec_cc restatement within 1e-13 (FP64) and 2e-6 (FP32),
    for one and two orbitals (inter-orbital Hloc hopping included);
  - a whole T=0 solve through it equals the solve through the default
    kernels (E0 within 1e-12, G(iwn) within 1e-10), FP64 and mixed;
  - on a long-column sector of Ns=16 (8 up electrons: 12,870 rows, 2 down:
    120 columns) it is chosen by itself; beyond the reference's own range
    (its 32-bit Fock index), the product is checked against the spin-flipped
    twin sector on the shared-memory kernels within 1e-13, the ground-state
    energies of the two sectors agree within 1e-10, the FP64 ground state
    meets |H psi - E psi| <= 1e-9, and the mixed one its energy within
    1e-10."""
import numpy as np
import pytest

import dmfted
import oracle as O

pytestmark = pytest.mark.gpu


def solver(m, **kw):
    ul = list(m.uloc) + [0.0] * (3 - len(m.uloc))
    p = dmfted.default_params(norb=m.norb, nbath=m.nbath, nspin=m.nspin, uloc=ul, ust=m.ust,
                              jh=m.jh, xmu=m.xmu, beta=m.beta, hfmode=int(m.hfmode), **kw)
    s = dmfted.EDSolver(p, hloc=m.hloc)
    s.set_bath(m.bath_array())
    return s


def two_orbital_model():
    rng = np.random.default_rng(9)
    e = rng.uniform(-1.0, 1.0, (1, 2, 2))
    v = 0.4 + rng.uniform(-0.1, 0.1, (1, 2, 2))
    hloc = np.zeros((1, 1, 2, 2), complex)
    hloc[0, 0] = [[0.1, 0.2], [0.2, -0.1]]
    return O.Model(norb=2, nbath=2, nspin=1, uloc=(3.0, 3.0, 0.0), ust=2.0, jh=0.5, beta=50.0,
                   e=e, v=v, hloc=hloc)


@pytest.mark.parametrize("case", ["one_orbital", "two_orbitals"])
def test_forced_global_product_matches_oracle(monkeypatch, case):
    import torch
    monkeypatch.setenv("DMFTED_HXV_KERNEL", "3")
    if case == "one_orbital":
        m, nup, ndw = O.seeded_model(3, nbath=7, u=2.0), 4, 3
    else:
        m, nup, ndw = two_orbital_model(), 3, 3
    s = solver(m, lmats=16, lreal=0)
    isec = s.sector_index(nup, ndw)
    s.setup_hv_sector(isec)
    hm = O.build_sector(m.ns, nup, ndw)
    rng = np.random.default_rng(17)
    v = rng.normal(size=hm.size) + 1j * rng.normal(size=hm.size)
    ref = O.hxv(m, hm, v)
    assert np.abs(s.hxv(v) - ref).max() <= 1e-13 * np.abs(ref).max()
    x = torch.tensor(v.real, dtype=torch.float64, device="cuda")
    x32 = x.float()
    y32 = torch.empty_like(x32)
    torch.cuda.synchronize()
    dmfted._ck(dmfted.lib().dmfted_hxv_device_f32(s.ctx, x32.data_ptr(), y32.data_ptr(), 1))
    s.time_hxv(fp32=True, warmup=0, reps=1)  # drains the library stream
    ref_r = O.hxv(m, hm, v.real.astype(complex)).real
    assert np.abs(y32.cpu().double().numpy() - ref_r).max() <= 2e-6 * np.abs(ref_r).max()
    s.close()


@pytest.mark.parametrize("precision", [dmfted.FP64, dmfted.MIXED])
def test_forced_global_solve_matches_default_kernels(monkeypatch, precision):
    m = O.seeded_model(1, nbath=7, u=2.0, beta=100.0)
    out = []
    for kern in ("0", "3"):
        monkeypatch.setenv("DMFTED_HXV_KERNEL", kern)
        s = solver(m, lmats=256, lreal=0, precision=precision, lanc_nstates_sector=1)
        s.ed_solve(m.bath_array(), sectors=[s.sector_index(4, 4)])
        out.append((s.egs(), s.ed_get_gimp_matsubara()))
        s.close()
    assert abs(out[0][0] - out[1][0]) <= 1e-12 * abs(out[0][0])
    assert np.abs(out[0][1] - out[1][1]).max() <= 1e-10


def test_long_column_sector_ns16():
    """Ns=16 lies beyond the reference itself (its Fock index iup + idw*2^Ns
    is a default integer: 2Ns = 32 bits overflow it, and the oracle's int32
    map likewise), so the long-column sector (8 up, 2 down: 12,870 rows, 120
    columns) is checked through the spin-flip symmetry of a one-spin bath:
    H(8,2) = P H(2,8) P^T with P the transpose of the DimUp x DimDw matrix
    (each spin's hop signs depend on its own word only), where (2,8) has
    120-row columns and runs on the shared-memory kernels."""
    m = O.seeded_model(5, nbath=15, u=2.0, beta=100.0)
    s = solver(m, lmats=16, lreal=0)
    a, b = s.sector_index(8, 2), s.sector_index(2, 8)
    dup, ddw = 12870, 120
    assert s.sector_dim(a) == dup * ddw
    rng = np.random.default_rng(3)
    v = rng.normal(size=dup * ddw) + 1j * rng.normal(size=dup * ddw)
    s.setup_hv_sector(a)
    y_long = s.hxv(v)  # element iup + dup*idw
    s.setup_hv_sector(b)
    w = v.reshape(ddw, dup).T.reshape(-1)  # element idw + ddw*iup of the twin
    y_short = s.hxv(w).reshape(dup, ddw).T.reshape(-1)
    assert np.abs(y_long - y_short).max() <= 1e-13 * np.abs(y_short).max()
    # the ground states of the two sectors (the same spectrum)
    e_long, psi, _ = s.lanczos_gs(a)
    e_short, _, _ = s.lanczos_gs(b)
    assert abs(e_long - e_short) <= 1e-10 * abs(e_short)
    s.setup_hv_sector(a)
    assert np.linalg.norm(s.hxv(psi) - e_long * psi) <= 1e-9
    s.close()
    sm = solver(m, lmats=16, lreal=0, precision=dmfted.MIXED)
    e32, _, _ = sm.lanczos_gs(sm.sector_index(8, 2))
    assert abs(e32 - e_long) <= 1e-10 * abs(e_long)
    sm.close()


@pytest.mark.parametrize("precision", [dmfted.FP64, dmfted.MIXED])
def test_ground_state_with_a_capped_basis(monkeypatch, precision):
    """A Krylov basis cut by device memory (here a 120 MB budget: 16 FP64 or
    33 FP32 vectors of the Ns=12 half-filled sector, against the ~130 steps a
    run needs) restarts from its Ritz vector until the stopping test holds:
    the energy equals the uncapped run's within 1e-10 and the vector meets
    |H psi - E psi| <= 1e-9 with the oracle's product."""
    m = O.seeded_model(2, nbath=11, u=3.0)
    res = []
    for budget in (None, "120"):
        if budget:
            monkeypatch.setenv("DMFTED_GS_BASIS_MB", budget)
        s = solver(m, lmats=16, lreal=0, precision=precision)
        isec = s.sector_index(6, 6)
        e0, psi, nit = s.lanczos_gs(isec)
        res.append((e0, psi, nit))
        s.close()
    (e_full, _, n_full), (e_cap, psi, n_cap) = res
    if precision == dmfted.FP64:
        assert n_cap > n_full  # the restarts cost steps (the mixed form restarts anyway)
    assert abs(e_cap - e_full) <= 1e-10 * abs(e_full)
    hm = O.build_sector(m.ns, 6, 6)
    hpsi = O.hxv(m, hm, psi.astype(complex), nthreads=O.lib().or_host_threads()).real
    assert np.linalg.norm(hpsi - e_cap * psi) <= 1e-9
