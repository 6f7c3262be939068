"""ed_solve_lattice: the impurity problems of the inequivalent sites of a
lattice DMFT, one solve per site, the sites shared over the ranks of a
process group -- the host side of ED_MAIN.f90:364-483 (serial) and
:488-670 (MPI), with torch.distributed standing in for MPI.

As in the reference:
  * site ilat (0-based here) is solved by rank ilat % size, in increasing order
    on each rank (ED_MAIN.f90:597: do ilat = 1+MPI_ID, Nsites, MPI_SIZE);
  * every site keeps its own adaptive eigenspace sizes, neigen_sector(:) and
    lanc_nstates_total, swapped into the single impurity context before its
    solve and read back after it (neigen_sectorii / neigen_totalii,
    :419-423,597-611);
  * each rank fills zero-initialised [Nsites, ...] arrays for its sites and one
    all-reduce (sum) gives every rank the result of every site (:655-670).
    That is the only collective; it moves Nsites x (G, Sigma, observables)
    (64 KB per site at Lmats=4096, Norb=Nspin=1), not vectors.

The solver is one EDSolver per process (one GPU per rank); nothing of the
device path changes.  With no process group, or a group of one, every site
is solved locally.
"""
import numpy as np


def site_owner(ilat, size):
    """The rank that solves site ilat (round robin, ED_MAIN.f90:597)."""
    return ilat % size


class LatticeSolver:
    """Per-site state and the lattice solve over one impurity solver.

    solver: an EDSolver (or an object with its interface: params, nsectors,
    ed_solve, set_hloc, get_neigen, set_neigen, the ed_get_* getters and
    observables).  nsites: number of inequivalent sites."""

    def __init__(self, solver, nsites):
        self.solver = solver
        self.nsites = int(nsites)
        ne, tot = solver.get_neigen()
        # ed_init_solver_lattice: every site starts from the initial sizes
        self.neigen = np.tile(np.asarray(ne, np.int32), (self.nsites, 1))
        self.ntotal = np.full(self.nsites, int(tot), np.int32)

    def solve(self, baths, hloc=None, sectors=None, group=None):
        """Solve every site; returns a dict of [Nsites, ...] arrays: gmats,
        greal, smats, sreal (Nspin, Nspin, Norb, Norb, L), dens, docc, magz
        (Norb), egs -- identical on every rank of the group."""
        import torch
        import torch.distributed as dist

        baths = np.asarray(baths, np.float64)
        if baths.ndim != 2 or baths.shape[0] != self.nsites:
            raise ValueError("ed_solve_lattice: bath must be [Nsites, Nb]")
        distributed = group is not None or (dist.is_available() and dist.is_initialized())
        size = dist.get_world_size(group) if distributed else 1
        rank = dist.get_rank(group) if distributed else 0
        p = self.solver.params
        ns, no = p.nspin, p.norb
        gm = np.zeros((self.nsites, ns, ns, no, no, p.lmats), np.complex128)
        gr = np.zeros((self.nsites, ns, ns, no, no, p.lreal), np.complex128)
        sm = np.zeros_like(gm)
        sr = np.zeros_like(gr)
        obs = np.zeros((self.nsites, 3, no))
        egs = np.zeros(self.nsites)
        neig = np.zeros_like(self.neigen)
        ntot = np.zeros_like(self.ntotal)
        for ilat in range(rank, self.nsites, size):
            self.solver.set_neigen(self.neigen[ilat], self.ntotal[ilat])
            if hloc is not None:
                self.solver.set_hloc(hloc[ilat])
            self.solver.ed_solve(baths[ilat], sectors=sectors)
            gm[ilat] = self.solver.ed_get_gimp_matsubara()
            sm[ilat] = self.solver.ed_get_sigma_matsubara()
            if p.lreal > 0:
                gr[ilat] = self.solver.ed_get_gimp_real()
                sr[ilat] = self.solver.ed_get_sigma_real()
            ob = self.solver.observables()
            obs[ilat] = [ob["dens"], ob["docc"], ob["magz"]]
            egs[ilat] = self.solver.egs()
            neig[ilat], ntot[ilat] = self.solver.get_neigen()
        self.last_reduce_ms = 0.0
        if size > 1:
            backend = dist.get_backend(group)
            dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" \
                else torch.device("cpu")
            # one flat float64 buffer: the arrays of every site, zero for the
            # sites of other ranks; one sum gives each rank all sites
            parts = [gm.view(np.float64), gr.view(np.float64), sm.view(np.float64),
                     sr.view(np.float64), obs, egs, neig.astype(np.float64),
                     ntot.astype(np.float64)]
            flat = np.concatenate([a.reshape(-1) for a in parts])
            t = torch.from_numpy(flat).to(dev)
            if dev.type == "cuda":
                # device time of the exchange (events on the stream NCCL joins)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
                e1.record()
                e1.synchronize()
                self.last_reduce_ms = e0.elapsed_time(e1)
            else:
                dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
            flat = t.cpu().numpy()
            off = 0
            out = []
            for a in parts:
                out.append(flat[off:off + a.size].reshape(a.shape))
                off += a.size
            gm = out[0].copy().view(np.complex128).reshape(gm.shape)
            gr = out[1].copy().view(np.complex128).reshape(gr.shape)
            sm = out[2].copy().view(np.complex128).reshape(sm.shape)
            sr = out[3].copy().view(np.complex128).reshape(sr.shape)
            obs, egs = out[4], out[5]
            neig = np.rint(out[6]).astype(np.int32)
            ntot = np.rint(out[7]).astype(np.int32)
        self.neigen, self.ntotal = neig, ntot
        return dict(gmats=gm, greal=gr, smats=sm, sreal=sr, dens=obs[:, 0], docc=obs[:, 1],
                    magz=obs[:, 2], egs=egs)


def ed_solve_lattice(solver, baths, hloc=None, sectors=None, group=None, state=None):
    """One lattice solve; state (a LatticeSolver of this solver) carries the
    per-site eigenspace sizes from one DMFT iteration to the next."""
    st = state if state is not None else LatticeSolver(solver, np.asarray(baths).shape[0])
    return st.solve(baths, hloc=hloc, sectors=sectors, group=group)
