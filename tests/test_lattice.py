"""The lattice solve's host logic (dmfted/lattice.py, the counterpart of
ed_solve_lattice / ed_solve_lattice_mpi, ED_MAIN.f90:364-670) on CPU: sites
shared round robin over two gloo ranks, per-site adaptive eigenspace sizes,
and the one all-reduce that gives every rank every site.  The impurity solver
is a stand-in with the EDSolver interface backed by the oracle (T=0 solve of
a small single-orbital bath), so no GPU is involved."""
import os
import socket
import sys
import tempfile
import types

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NB = 3          # bath levels (Ns = 4)
NSITES = 5
LMATS = 64


class OracleSite:
    """EDSolver stand-in: ed_solve runs the oracle's T=0 pipeline on the half-
    filled sector; the eigenspace sizes follow a per-solve rule (the real
    adaptation is ed_analysis's) so that their per-site bookkeeping is seen."""

    def __init__(self):
        self.params = types.SimpleNamespace(nspin=1, norb=1, lmats=LMATS, lreal=0)
        self.nsectors = (NB + 2) ** 2
        self.ne = np.full(self.nsectors, 6, np.int32)
        self.tot = 1
        self.solved = []

    def get_neigen(self):
        return self.ne.copy(), self.tot

    def set_neigen(self, ne, tot):
        self.ne = np.asarray(ne, np.int32).copy()
        self.tot = int(tot)

    def set_hloc(self, h):
        raise AssertionError("no hloc in this test")

    def ed_solve(self, bath, sectors=None):
        import oracle as O
        m = O.Model(norb=1, nbath=NB, nspin=1, uloc=(2.0, 0.0, 0.0), beta=100.0,
                    e=np.asarray(bath[:NB]).reshape(1, 1, NB),
                    v=np.asarray(bath[NB:]).reshape(1, 1, NB))
        self.r = O.solve_sector_t0(m, 2, 2, lmats=LMATS, lreal=0)
        self.solved.append(float(bath[0]))
        self.ne = self.ne + 1 + (int(bath[0] * 1e3) % 3)
        self.tot += 2

    def ed_get_gimp_matsubara(self):
        return self.r["gmats"].reshape(1, 1, 1, 1, LMATS)

    def ed_get_sigma_matsubara(self):
        return self.r["smats"].reshape(1, 1, 1, 1, LMATS)

    def observables(self):
        o = self.r["obs"]
        return dict(dens=np.asarray(o["dens"][:1]), docc=np.asarray(o["docc"][:1]),
                    magz=np.zeros(1))

    def egs(self):
        return self.r["e0"]


def baths():
    rng = np.random.default_rng(11)
    e = rng.uniform(-1, 1, (NSITES, NB))
    v = 0.5 + rng.uniform(-0.1, 0.1, (NSITES, NB))
    return np.concatenate([e, v], axis=1)


def run_two_calls(group=None):
    from dmfted.lattice import LatticeSolver
    site = OracleSite()
    st = LatticeSolver(site, NSITES)
    b = baths()
    r1 = st.solve(b, group=group)
    r2 = st.solve(b * 1.01, group=group)
    return r1, r2, st.neigen.copy(), st.ntotal.copy(), site.solved


def _worker(rank, port, out):
    sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "dmft-ed_b200")]
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=2,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        r1, r2, ne, nt, solved = run_two_calls()
        np.savez(os.path.join(out, f"rank{rank}.npz"), g1=r1["gmats"], g2=r2["gmats"],
                 s2=r2["smats"], d2=r2["dens"], e2=r2["egs"], ne=ne, nt=nt,
                 solved=np.array(solved))
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_lattice_two_gloo_ranks_match_serial():
    import torch.multiprocessing as mp
    serial = run_two_calls()
    with tempfile.TemporaryDirectory() as out:
        mp.spawn(_worker, args=(free_port(), out), nprocs=2, join=True)
        ranks = [np.load(os.path.join(out, f"rank{r}.npz")) for r in range(2)]
    r1, r2, ne, nt, _ = serial
    for z in ranks:
        # every rank holds every site, equal to the serial solve
        assert np.array_equal(z["g1"], r1["gmats"])
        assert np.array_equal(z["g2"], r2["gmats"])
        assert np.array_equal(z["s2"], r2["smats"])
        assert np.array_equal(z["d2"], r2["dens"])
        assert np.array_equal(z["e2"], r2["egs"])
        # per-site eigenspace sizes carried across calls, as serially
        assert np.array_equal(z["ne"], ne) and np.array_equal(z["nt"], nt)
    # round robin: rank 0 solves sites 0, 2, 4 and rank 1 sites 1, 3 (twice)
    b = baths()
    own0 = [b[i, 0] for i in (0, 2, 4)] + [b[i, 0] * 1.01 for i in (0, 2, 4)]
    own1 = [b[i, 0] for i in (1, 3)] + [b[i, 0] * 1.01 for i in (1, 3)]
    assert np.allclose(ranks[0]["solved"], own0) and np.allclose(ranks[1]["solved"], own1)


def test_lattice_sites_keep_their_own_sizes():
    # without the per-site copies every site would inherit the previous
    # site's adapted sizes; with them site i's sizes depend only on its baths
    r1, r2, ne, nt, _ = run_two_calls()
    b = baths()
    for i in range(NSITES):
        expect = 6 + (1 + int(b[i, 0] * 1e3) % 3) + (1 + int(b[i, 0] * 1.01 * 1e3) % 3)
        assert np.all(ne[i] == expect)
        assert nt[i] == 1 + 2 + 2
    assert r1["gmats"].shape == (NSITES, 1, 1, 1, 1, LMATS)


def test_lattice_rejects_wrong_bath_shape():
    from dmfted.lattice import LatticeSolver
    st = LatticeSolver(OracleSite(), NSITES)
    with pytest.raises(ValueError):
        st.solve(baths()[:2])
