"""ed_solve_lattice on the GPU solver (one context, sites swapped in): equal to
independent per-site contexts, over two solves so that each site's adaptive
eigenspace sizes (neigen_sector, lanc_nstates_total) are carried separately,
as ed_solve_lattice does with neigen_sectorii / neigen_totalii
(ED_MAIN.f90:419-423,597-611)."""
import numpy as np
import pytest

import dmfted
from dmfted.lattice import LatticeSolver

pytestmark = pytest.mark.gpu


def site_baths(nsites, nbath, seed):
    rng = np.random.default_rng(seed)
    e = rng.uniform(-1, 1, (nsites, nbath))
    v = 0.5 + rng.uniform(-0.1, 0.1, (nsites, nbath))
    return np.concatenate([e, v], axis=1)


@pytest.mark.parametrize("total", [1, 4])
def test_lattice_matches_independent_site_solvers(monkeypatch, total):
    # fixed cluster sizes: a measured choice could differ between contexts and
    # move the results at the rounding level
    monkeypatch.setenv("DMFTED_AUTOTUNE", "0")
    nb, nsites = 5, 3
    kw = dict(nbath=nb, uloc=[2.0], beta=30.0, lmats=128, lreal=0, lanc_nstates_total=total)
    b = site_baths(nsites, nb, 17)
    with dmfted.EDSolver(dmfted.default_params(**kw)) as s:
        st = LatticeSolver(s, nsites)
        lat = [st.solve(b), st.solve(b * 1.02)]
        ne_lat = st.neigen.copy()
    for i in range(nsites):
        with dmfted.EDSolver(dmfted.default_params(**kw)) as s1:
            for it, bb in enumerate((b[i], b[i] * 1.02)):
                s1.ed_solve(bb)
                g = s1.ed_get_gimp_matsubara()
                assert np.array_equal(lat[it]["gmats"][i], g), (i, it)
                assert np.array_equal(lat[it]["smats"][i], s1.ed_get_sigma_matsubara())
                assert lat[it]["egs"][i] == s1.egs()
                assert np.array_equal(lat[it]["dens"][i], s1.observables()["dens"])
            assert np.array_equal(ne_lat[i], s1.get_neigen()[0])


def test_neigen_round_trip_and_checks():
    with dmfted.EDSolver(dmfted.default_params(nbath=3, lanc_nstates_total=4)) as s:
        ne, tot = s.get_neigen()
        assert ne.size == s.nsectors and tot == 4
        s.set_neigen(ne + 2, 6)
        ne2, tot2 = s.get_neigen()
        assert np.array_equal(ne2, ne + 2) and tot2 == 6
        with pytest.raises(dmfted.DmftedError):
            s.set_neigen(np.zeros_like(ne), 6)
        with pytest.raises(dmfted.DmftedError):
            s.set_neigen(ne[:-1], 6)
