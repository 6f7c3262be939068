"""Benchmark of the exact-diagonalization impurity solve on B200.

Workload (one step): one impurity solve of the single-orbital Hubbard model on
a Bethe-lattice bath, Ns=14 (Nbath=13), U=3, beta=100, half filling, sector
nup=ndw=7 (dim 11,778,624): Lanczos ground state to the ARPACK-style residual
tolerance 1e-12, observables, particle and hole Green's-function chains of 200
steps, G and Sigma on Lmats=4096 Matsubara points.  Seeded synthetic bath:
e_k ~ U[-1,1], V_k = 0.5 + U[-0.1,0.1] (numpy default_rng(seed)).

The timed form is the mixed-precision solver (FP32 vectors, compensated FP64
alpha/beta, FP64 refinement of the ground state, FP64 continued fractions);
the plain-FP64 drop-in path is timed beside it on the same inputs and their
differences are reported.

Output: one JSON line (rank 0).  Multi-GPU: independent replicas (one solve
per rank per step, weak scaling), launched with torch.distributed.run.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dmft-ed_b200"))

import numpy as np  # noqa: E402

METRIC = ("DMFT-step solve time & H·v GB/s at Ns=14: mixed vs FP64 GPU, "
          "|ΔE0|/|E0|≤1e-10")
UNIT = "DMFT-steps/s"
NBATH, U, BETA, LMATS, NGF, SEED = 13, 3.0, 100.0, 4096, 200, 1
NUP = NDW = 7


def seeded_bath(seed=SEED, nbath=NBATH):
    rng = np.random.default_rng(seed)
    e = rng.uniform(-1.0, 1.0, size=nbath)
    v = 0.5 + rng.uniform(-0.1, 0.1, size=nbath)
    return np.concatenate([e, v])


def measured_peak_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(name):
    """Per-launch DRAM bytes of a kernel from its committed ncu summary
    (profiles/<name>.md line 'dram_bytes_per_launch: N')."""
    p = os.path.join(ROOT, "profiles", name + ".md")
    try:
        for line in open(p):
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def l2_flush(dev):
    """Write a 256 MB buffer (> 126 MB L2) between timed steps."""
    import torch
    buf = getattr(l2_flush, "buf", None)
    if buf is None:
        buf = l2_flush.buf = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    buf.fill_(1.0)
    torch.cuda.synchronize(dev)


def seeded_bath_2orb(seed=4, norb=2, nbath=4):
    """Two-orbital finite-temperature workload: e_k ~ U[-1.5,1.5], V_k = 0.4 +
    U[-0.1,0.1] per orbital (default_rng(seed)); user-bath layout e then V,
    k fastest, then orbital."""
    rng = np.random.default_rng(seed)
    e = rng.uniform(-1.5, 1.5, size=(norb, nbath))
    v = 0.4 + rng.uniform(-0.1, 0.1, size=(norb, nbath))
    return np.concatenate([e.reshape(-1), v.reshape(-1)])


def config_pins():
    """Oracle fixtures of the workload configurations (tests/golden), or None."""
    try:
        return np.load(os.path.join(ROOT, "tests", "golden", "config_pins.npz"))
    except OSError:
        return None


def finite_t_workload(dmfted, device, steps, warmup):
    """Norb=2, Nbath=4 (Ns=10), U=3, J=0.5, Ust=U-2J, beta=50, Nspin=2 (the
    same bath for both spins): every one of the 121 sectors diagonalised,
    lanc_nstates_total=16 lowest states kept, the particle/hole chains of
    every kept state, spin and orbital -- all in the persistent work-queue
    kernels."""
    b1 = seeded_bath_2orb()
    nb = b1.size // 2
    bath = np.concatenate([b1[:nb], b1[:nb], b1[nb:], b1[nb:]])  # Nspin=2, same bath per spin
    pins = config_pins()
    out = {}
    ref_g = None
    for prec in (dmfted.FP64, dmfted.MIXED):
        p = dmfted.default_params(norb=2, nbath=4, nspin=2, uloc=[3.0, 3.0], ust=2.0, jh=0.5,
                                  beta=50.0, lmats=LMATS, lreal=0, lanc_nstates_total=16,
                                  precision=prec, device=device)
        s = dmfted.EDSolver(p)
        oracle = None
        for w in range(max(1, warmup)):
            s.ed_solve(bath)
            if w == 0 and pins is not None and "cfg4_gmats" in pins:
                # the first solve (lanc_nstates_total = 16, Neigen = 6) against
                # the oracle fixture; later solves adapt the state counts
                e, _, z = s.eigenspace()
                g0 = s.ed_get_gimp_matsubara()
                oracle = dict(
                    fixture="tests/golden/config_pins.npz cfg4 (first solve)",
                    dE0_rel=abs(e[0] - float(pins["cfg4_e"][0])) / abs(float(pins["cfg4_e"][0])),
                    dZ_rel=abs(z - float(pins["cfg4_zeta"])) / float(pins["cfg4_zeta"]),
                    max_dG=max(float(np.abs(g0[i, i, a, a] - pins["cfg4_gmats"][i, a]).max())
                               for i in range(2) for a in range(2)))
        ms, launches = [], 0
        for _ in range(steps):
            s.launch_count(reset=True)
            s.ed_solve(bath)
            ms.append(s.timings()["total_ms"])
            launches = s.launch_count()
        e, secs, z = s.eigenspace()
        g = s.ed_get_gimp_matsubara()
        tm = s.timings()
        if ref_g is None:
            ref_g = g
        out["fp64" if prec == dmfted.FP64 else "mixed"] = dict(
            ms_per_solve=statistics.median(ms), launches_per_solve=launches,
            states_kept=len(e), gf_chains=tm["hv_gf"] // NGF, diag_ms=tm["diag_ms"],
            gf_ms=tm["gf_ms"], max_dG_vs_fp64=float(np.abs(g - ref_g).max()),
            vs_oracle=oracle, autotune=s.autotune_log())
        s.close()
    return out


def chi2_inputs(nbath=9, L=1000, beta=100.0, nbatch=4096, seed=5):
    """Delta(iwn) = sum_k V_k^2/(iwn - e_k) of a seeded bath plus complex
    Gaussian noise (sigma 1e-4), weight 1/wn, and nbatch seeded parameter sets
    around the bath."""
    rng = np.random.default_rng(seed)
    wm = np.pi / beta * (2.0 * np.arange(1, L + 1) - 1.0)
    e0 = rng.uniform(-1.0, 1.0, nbath)
    v0 = 0.5 + rng.uniform(-0.1, 0.1, nbath)
    z = 1j * wm
    delta = (v0[None, :] ** 2 / (z[:, None] - e0[None, :])).sum(axis=1)
    delta = delta + 1e-4 * (rng.normal(size=L) + 1j * rng.normal(size=L))
    w = 1.0 / wm
    a = np.concatenate([e0, v0])[None, :] + 0.05 * rng.normal(size=(nbatch, 2 * nbath))
    return a, wm, delta, w


def differentiation_workload(dmfted, device, steps, warmup, solver64, isec, bath):
    """(a) Hellmann-Feynman dE0/d{e_k, V_k} on the Ns=14 ground state, with
    central differences (h=1e-5) for two parameters; (b) chi^2 of the Delta
    fit and its reverse-mode gradient for 4096 parameter sets (Nbath=9,
    Lfit=1000), device pointers, timed with CUDA events."""
    import torch
    solver64.ed_solve(bath, sectors=[isec])
    obs_ms = solver64.timings()["obs_ms"]
    t0 = time.perf_counter()
    grad = solver64.hf_gradient()  # hop expectations over the ground state (synchronous)
    grad_ms = (time.perf_counter() - t0) * 1e3
    h = 1e-5
    fd_err = 0.0
    for i in (0, NBATH):  # e_1 and V_1
        ep = []
        for sgn in (1, -1):
            b = bath.copy()
            b[i] += sgn * h
            solver64.ed_solve(b, sectors=[isec])
            ep.append(solver64.egs())
        fd = (ep[0] - ep[1]) / (2 * h)
        fd_err = max(fd_err, abs(fd - grad[i]) / max(1.0, abs(fd)))
    solver64.ed_solve(bath, sectors=[isec])
    a, wm, delta, w = chi2_inputs()
    dev = torch.device("cuda", device)
    nbatch, n2 = a.shape
    da = torch.from_numpy(a).to(dev)
    dx = torch.from_numpy(wm).to(dev)
    dg = torch.from_numpy(np.ascontiguousarray(delta).view(np.float64)).to(dev)
    dw = torch.from_numpy(w).to(dev)
    dc = torch.empty(nbatch, dtype=torch.float64, device=dev)
    dgr = torch.empty(nbatch * n2, dtype=torch.float64, device=dev)
    lib = dmfted.lib()
    torch.cuda.synchronize(dev)  # inputs uploaded before the library's stream reads them

    def call():
        rc = lib.dmfted_chi2_delta_batch_device(solver64.ctx, nbatch, n2 // 2, wm.size,
                                                da.data_ptr(), dx.data_ptr(), dg.data_ptr(),
                                                dw.data_ptr(), dc.data_ptr(), dgr.data_ptr())
        assert rc == 0, lib.dmfted_last_error()
    for _ in range(warmup):
        call()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(steps):
        call()
    torch.cuda.synchronize(dev)
    chi2_ms = (time.perf_counter() - t0) / steps * 1e3
    return dict(
        hf=dict(params=2 * NBATH, obs_phase_ms=obs_ms, gradient_call_ms=grad_ms,
                max_rel_diff_vs_central_fd=fd_err, fd_params="e_1, V_1", h=h),
        chi2=dict(nbatch=nbatch, nbath=n2 // 2, lfit=wm.size, ms_per_batch=chi2_ms,
                  sets_per_s=nbatch / (chi2_ms * 1e-3),
                  timing="wall clock over the device calls, device synchronised"),
        chi2_host=(a, wm, delta, w, dc.cpu().numpy(), dgr.cpu().numpy().reshape(nbatch, n2)))


def dmft_workload(dmfted, device, steps, warmup):
    """The self-consistency around the solve.  (a) The bath-fit minimiser on
    4096 start points at once (the chi^2 workload's target and parameter sets,
    delta scheme, cg_weight as 1/wn there, one CTA per fit).  (b) Whole
    iterations of the Bethe-lattice DMFT loop at the small configuration (Ns=8,
    Nbath=7, U=2, beta=100, Lmats=4096, T=0 with every sector scanned as
    ed_solve does, Weiss-field fit on Lfit=1000 points, 500-point semicircle):
    solve, Sigma, G_loc, Weiss field, fit and mixing, all on the device."""
    from dmfted import bethe
    a, wm, delta, w = chi2_inputs()
    p = dmfted.default_params(nbath=9, beta=100.0, lmats=1000, lreal=0, device=device)
    with dmfted.EDSolver(p) as s:
        s.cg_fit_batch(a[:64], wm, delta, w, scheme=dmfted.CG_DELTA)  # warm-up
        t0 = time.perf_counter()
        am, c2, it = s.cg_fit_batch(a, wm, delta, w, scheme=dmfted.CG_DELTA)
        fit_s = time.perf_counter() - t0
    fits = dict(nbatch=a.shape[0], nbath=a.shape[1] // 2, lfit=wm.size, seconds=fit_s,
                fits_per_s=a.shape[0] / fit_s, mean_iterations=float(np.mean(it)),
                max_iterations=int(np.max(it)), median_chi2=float(np.median(c2)),
                timing="wall clock around the synchronous call (host copies included)")
    p = dmfted.default_params(norb=1, nbath=7, uloc=[2.0], beta=100.0, lmats=LMATS, lreal=0,
                              device=device)
    rng = np.random.default_rng(SEED)
    bath = np.concatenate([rng.uniform(-1.0, 1.0, 7), 0.5 + rng.uniform(-0.1, 0.1, 7)])
    he, wt = bethe.bethe_dos(500, 1.0)
    ms = []
    with dmfted.EDSolver(p) as s:
        prev = None
        for i in range(warmup + steps):
            t0 = time.perf_counter()
            new, weiss, chi2 = bethe.dmft_step(s, bath, he, wt)
            bath = new if prev is None else 0.5 * new + 0.5 * prev
            prev = bath.copy()
            if i >= warmup:
                ms.append((time.perf_counter() - t0) * 1e3)
    loop = dict(workload="Bethe DMFT iteration, Ns=8 (Nbath=7, U=2, beta=100), every sector "
                         "at T=0, Lmats=4096, Weiss fit on Lfit=1000",
                ms_per_iteration=statistics.median(ms), iterations_timed=len(ms),
                last_chi2=float(chi2[0][0]),
                timing="wall clock of the public calls (host arrays in and out)")
    return dict(fit_batch=fits, bethe_iteration=loop,
                fit_host=(a[:8].copy(), wm, delta, w, am[:8].copy(), c2[:8].copy()))


def small_configs_workload(dmfted, device, steps, warmup):
    """The two smaller single-orbital configurations through the same solve:
    Ns=8 (Nbath=7, U=2, sector 4/4, dim 4,900) and Ns=12 (Nbath=11, U=3, bath
    seed 2, sector 6/6, dim 853,776), beta=100, Lmats=4096, 200-step chains;
    median device milliseconds per solve in both precisions."""
    out = {}
    for name, nbath, u, seed, nn in (("ns8_4_4", 7, 2.0, SEED, 4), ("ns12_6_6", 11, 3.0, 2, 6)):
        rng = np.random.default_rng(seed)
        bath = np.concatenate([rng.uniform(-1.0, 1.0, nbath), 0.5 + rng.uniform(-0.1, 0.1, nbath)])
        row = {}
        for prec, tag in ((dmfted.MIXED, "mixed"), (dmfted.FP64, "fp64")):
            p = dmfted.default_params(norb=1, nbath=nbath, uloc=[u], beta=BETA, lmats=LMATS,
                                      lreal=0, lanc_nstates_sector=1, precision=prec,
                                      device=device)
            with dmfted.EDSolver(p) as s:
                isec = s.sector_index(nn, nn)
                for _ in range(warmup):
                    s.ed_solve(bath, sectors=[isec])
                ms = []
                for _ in range(steps):
                    s.ed_solve(bath, sectors=[isec])
                    ms.append(s.timings()["total_ms"])
                row[tag + "_ms"] = statistics.median(ms)
                row[tag + "_e0"] = s.egs()
        out[name] = row
    return out


def fit_cpu(host):
    """The oracle's conjugate-gradient fit (one thread) on the first start
    points of the batch: fits per second and the largest chi^2 difference."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    a, wm, delta, w, am, c2 = host
    t0 = time.perf_counter()
    err = 0.0
    for b in range(a.shape[0]):
        ar, fr, _, _ = O.cg_fit(a[b], wm, delta, w, weiss=False)
        err = max(err, abs(c2[b] - fr) / fr)
    sec = time.perf_counter() - t0
    return dict(fits_per_s=a.shape[0] / sec, cores=1, kind="port", sample=f"{a.shape[0]} fits",
                max_rel_chi2_diff_gpu_vs_oracle=err)


def make_solver(dmfted, precision, device):
    # LANC_NSTATES_SECTOR = 1: the workload is the sector's ground state (the
    # reference then asks sp_eigh for one eigenpair and keeps one state per
    # sector); the default 6 adds the degenerate-copy probes of ed_diag
    p = dmfted.default_params(nbath=NBATH, uloc=[U], beta=BETA, xmu=0.0, lmats=LMATS, lreal=0,
                              lanc_ngfiter=NGF, precision=precision, device=device,
                              lanc_nstates_sector=1)
    return dmfted.EDSolver(p)


def run_ours(args, rank, world, local_rank):
    import torch
    import dmfted
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    bath = seeded_bath()
    pinned = torch.from_numpy(bath).pin_memory()
    solvers = {prec: make_solver(dmfted, prec, local_rank) for prec in (dmfted.MIXED, dmfted.FP64)}
    isec = solvers[dmfted.MIXED].sector_index(NUP, NDW)

    def step(s):
        s.ed_solve(pinned.numpy(), sectors=[isec])
        return s.timings()["total_ms"]

    def e2e_step(s):
        # the public API with host buffers: bath from pinned host memory in,
        # G, Sigma and the observables back to the host
        t0 = time.perf_counter()
        s.ed_solve(pinned.numpy(), sectors=[isec])
        g = s.ed_get_gimp_matsubara()
        sg = s.ed_get_sigma_matsubara()
        ob = s.observables()
        return (time.perf_counter() - t0) * 1e3, g, sg, ob

    if world > 1:
        # one inequivalent lattice site per rank (ed_solve_lattice): site 0 is
        # the single-site workload's bath, site i seeded with SEED + i; the
        # ranks exchange every site's G, Sigma and observables in one
        # all-reduce after their solves
        from dmfted.lattice import LatticeSolver
        site_baths = np.stack([seeded_bath(SEED + i) for i in range(world)])
        lattices = {id(sv): LatticeSolver(sv, world) for sv in solvers.values()}

        def step(s):
            lat = lattices[id(s)]
            lat.solve(site_baths, sectors=[isec])
            return s.timings()["total_ms"] + lat.last_reduce_ms

        def e2e_step(s):
            t0 = time.perf_counter()
            r = lattices[id(s)].solve(site_baths, sectors=[isec])
            return ((time.perf_counter() - t0) * 1e3, r["gmats"][rank], r["smats"][rank],
                    dict(dens=r["dens"][rank], docc=r["docc"][rank], magz=r["magz"][rank]))

    res = {}
    for prec, s in solvers.items():
        for _ in range(args.warmup):
            step(s)
            l2_flush(dev)
        s.launch_count(reset=True)
        dist_barrier(world)
        ms = []
        with ClockSampler(local_rank) as clk:
            for _ in range(args.steps):
                ms.append(step(s))
                l2_flush(dev)
        launches = s.launch_count(reset=True)
        tm = s.timings()
        dist_barrier(world)
        # the same K steps through the public API, L2 flushed between them
        # (outside each step's own interval)
        e2e = []
        for _ in range(args.steps):
            e2e.append(e2e_step(s))
            l2_flush(dev)
        # the H*v roofline: K more steps with an event pair around every H*v
        # launch (the events cost ~3 % of a step, so they stay out of the
        # timed steps above)
        s.hxv_timing(True)
        rms = []
        for _ in range(args.steps):
            rms.append(step(s))
            l2_flush(dev)
        hvt = s.hxv_timing_totals()
        hvt["solve_ms"] = sum(rms)
        s.hxv_timing(False)
        res[prec] = dict(ms=ms, clocks=clk.summary(), launches=launches, e2e_ms=[x[0] for x in e2e],
                         g=e2e[-1][1], e0=s.egs(), obs=e2e[-1][3], tm=tm, hvt=hvt)
    # H*v of the sector alone, both precisions (device events on the library stream)
    s = solvers[dmfted.MIXED]
    s.setup_hv_sector(isec)
    dim = s.sector_dim(isec)
    hv32 = s.time_hxv(fp32=True, warmup=5, reps=50)
    hv64 = s.time_hxv(fp32=False, warmup=5, reps=50)
    extra = {}
    if world == 1 and args.only == "all":
        extra["finite_t_batched"] = finite_t_workload(dmfted, local_rank, args.steps, args.warmup)
        extra["differentiation"] = differentiation_workload(
            dmfted, local_rank, args.steps, args.warmup, solvers[dmfted.FP64], isec, bath)
        extra["self_consistency"] = dmft_workload(dmfted, local_rank, args.steps, args.warmup)
        extra["smaller_configs"] = small_configs_workload(dmfted, local_rank, args.steps,
                                                          args.warmup)
    for sv in solvers.values():
        sv.close()
    return res, dim, hv32, hv64, extra


def dist_barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def lanczos_step_seconds(O, m, hm, nthreads, nsteps):
    """Seconds per step of the oracle's plain three-term Lanczos recurrence
    (one directMatVec_cc product and the vector updates, buffers allocated
    once in C), the unit of work the reference's sp_eigh / sp_lanc_tridiag
    repeat: the time of nsteps + 1 steps minus that of one."""
    v = O.start_vector(hm.size)
    t0 = time.perf_counter()
    O.lanczos_tridiag(m, hm, v, 1, threshold=0.0, nthreads=nthreads)
    t1 = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.lanczos_tridiag(m, hm, v, nsteps + 1, threshold=0.0, nthreads=nthreads)
    return max(time.perf_counter() - t0 - t1, 1e-9) / nsteps


def cpu_sample(nthreads, n_hv):
    """The oracle (CPU restatement of directMatVec_cc with the combined map and
    binary search, complex128, inside its plain Lanczos recurrence) on the same
    sector: the map build and seconds per step over n_hv steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    m = O.seeded_model(SEED, nbath=NBATH, u=U, beta=BETA)
    t0 = time.perf_counter()
    hm = O.build_sector(m.ns, NUP, NDW)
    t_map = time.perf_counter() - t0
    return t_map, lanczos_step_seconds(O, m, hm, nthreads, n_hv)


def factored_cpu(nthreads, n_hv=5):
    """The "best CPU" variant: the device's up/down-factored product restated
    on the host in FP64 (oracle FactoredHxv), on the same sector and bath; its
    set-up, and seconds per H*v over n_hv products."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    m = O.seeded_model(SEED, nbath=NBATH, u=U, beta=BETA)
    t0 = time.perf_counter()
    F = O.FactoredHxv(m, NUP, NDW, nthreads=nthreads)
    t_setup = time.perf_counter() - t0
    x = np.random.default_rng(1).normal(size=F.hmap.size)
    F(x)
    t0 = time.perf_counter()
    for _ in range(n_hv):
        x = F(x)
        x /= np.linalg.norm(x)
    return t_setup, (time.perf_counter() - t0) / n_hv


def best_cpu_line(nthreads, hv_per_step):
    t_setup, t_hv = factored_cpu(nthreads)
    sec = t_setup + t_hv * hv_per_step
    return dict(value=1.0 / sec, unit=UNIT, cores=nthreads, kind="factored-port",
                sample=f"the factored FP64 H*v of the device kernels restated on the host "
                       f"(oracle FactoredHxv), 5 products on the 7/7 sector with {nthreads} "
                       f"threads, scaled to {hv_per_step} H*v per DMFT step plus its set-up",
                s_per_hv=t_hv, setup_s=t_setup)


def chi2_cpu(host, nsample=256):
    """The oracle's chi2_delta / grad_chi2_delta (one thread) on the first
    nsample parameter sets: sets per second, and the largest relative
    difference of the device results on them."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    a, wm, delta, w, c2, gr = host
    t0 = time.perf_counter()
    err = 0.0
    for b in range(nsample):
        rc, rg = O.chi2_delta(a[b], wm, delta, w)
        err = max(err, abs(c2[b] - rc) / abs(rc), float(np.abs(gr[b] - rg).max() / np.abs(rg).max()))
    sec = time.perf_counter() - t0
    return dict(sets_per_s=nsample / sec, cores=1, kind="port", sample=f"{nsample} sets",
                max_rel_diff_gpu_vs_oracle=err)


def cpu_step_seconds(t_map, t_hv, hv_per_step):
    return 3 * t_map + t_hv * hv_per_step


def reference_hv_per_step():
    """H*v products of one DMFT step of the reference on the 7/7 sector: the
    plain Lanczos ground state (its step count, taken from the oracle's own
    run in the cfg3 fixture), the second pass that rebuilds the vector
    (PLAIN_LANCZOS.f90:286-385: one product fewer), and the particle and hole
    chains (2 x lanc_ngfiter)."""
    pins = config_pins()
    nl = int(pins["cfg3_nlanc"]) if pins is not None and "cfg3_nlanc" in pins else 170
    return 2 * nl - 1 + 2 * NGF, nl


def small_solve_check(nthreads, nbath=7, nn=4, u=2.0, seed=SEED, threads=None, reps=50):
    """The model behind the extrapolation (3 map builds + per-product time x
    products) against a complete oracle solve, measured end to end: plain
    Lanczos ground state with its second pass, observables, two 200-step
    chains, G and Sigma on Lmats=4096.  Default: the small configuration (Ns=8,
    sector 4/4, dim 4900, U=2), single-thread and on every core."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    m = O.seeded_model(seed, nbath=nbath, u=u, beta=BETA)
    out = {}
    for nt in (threads or (1, nthreads)):
        t0 = time.perf_counter()
        r = O.solve_t0(m, sectors=[(nn, nn)], nstates_sector=1, lmats=LMATS, nthreads=nt)
        t_full = time.perf_counter() - t0
        t0 = time.perf_counter()
        hm = O.build_sector(m.ns, nn, nn)
        t_map = time.perf_counter() - t0
        t_hv = lanczos_step_seconds(O, m, hm, nt, reps)
        hv = 2 * r["nlanc"] - 1 + 2 * NGF
        out[f"threads_{nt}"] = dict(measured_s=t_full, model_s=cpu_step_seconds(t_map, t_hv, hv),
                                    hv_per_step=hv)
    return out


def reference_arm(args, nthreads):
    """--impl reference: the reference's algorithm (the oracle restatement of
    directMatVec_cc with the combined map and binary search, complex128, and
    the plain Lanczos) timed on the host cores.  A complete Ns=14 step takes
    about a quarter of an hour on 16 threads, so each timed step is a bounded
    sample -- the map build and one product on the same sector -- scaled to
    the products of one DMFT step (kind port-extrapolated).  Once per run: a
    single-thread product (the reference runs one thread per MPI rank), and
    the extrapolation model against complete oracle solves of the small
    configuration, single-thread and on every core."""
    hv_per_step, nl = reference_hv_per_step()
    samples = []
    t_wall0 = time.perf_counter()
    for i in range(args.warmup + args.steps):
        t_map, t_hv = cpu_sample(nthreads, 1)
        if i >= args.warmup:
            samples.append(cpu_step_seconds(t_map, t_hv, hv_per_step))
    t_sampled = time.perf_counter() - t_wall0
    sec = statistics.mean(samples)
    val = 1.0 / sec
    t_map1, t_hv1 = cpu_sample(1, 1)
    single = 1.0 / cpu_step_seconds(t_map1, t_hv1, hv_per_step)
    check = small_solve_check(nthreads)
    # the same check at Ns=12 (sector 6/6, dim 853,776, U=3, bath seed 2), where
    # the products dominate as at Ns=14: every core only (one thread would
    # take about ten minutes)
    check12 = small_solve_check(nthreads, nbath=11, nn=6, u=3.0, seed=2, threads=(nthreads,),
                                reps=2)
    return dict(
        metric=METRIC, value=val, unit=UNIT, n_gpus=args.gpus, steps=args.steps,
        warmup=args.warmup, ms_per_step=sec * 1e3, higher_is_better=True, scaling="weak",
        vs_baseline=None, dtype="c128", data="synthetic", impl="reference",
        config={"workload": "impurity solve Ns=14 (Nbath=13, U=3, beta=100) sector 7/7 "
                            "dim 11778624: Lanczos GS + observables + particle/hole chains "
                            "(200 steps) + G, Sigma on Lmats=4096",
                "lanc_nstates_sector": 1, "parallelism": f"{nthreads} host threads"},
        cpu_baseline=dict(
            value=val, unit=UNIT, cores=nthreads, kind="port-extrapolated",
            sample=(f"per step: the map build and 1 step of the oracle's plain Lanczos "
                    f"recurrence (directMatVec_cc, complex128, binary-search map) on the 7/7 "
                    f"sector with {nthreads} threads, scaled to "
                    f"{hv_per_step} H*v per DMFT step (plain Lanczos: {nl} steps, the second "
                    f"pass, 2 x {NGF} chain steps) + 3 map builds"),
            single_thread=dict(value=single, unit=UNIT, cores=1,
                               sample="the map build and 1 product on one thread, same scaling"),
            best_cpu_factored=best_cpu_line(nthreads, hv_per_step),
            model_check_small_config=check,
            model_check_ns12=check12,
            sampled_wall_s=t_sampled),
        e2e=dict(value=val, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--only", default="all",
                    choices=["all", "headline", "finite_t", "differentiation",
                             "self_consistency"],
                    help="run one workload (profiling); the default prints the full line")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    nthreads = os.cpu_count() or 1

    if args.impl == "reference":
        # the reference's algorithm on the host cores (the CPU restatement; the
        # Fortran reference cannot be built here), rank 0 only
        if rank != 0:
            return
        print(json.dumps(reference_arm(args, nthreads)))
        return

    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    import dmfted
    if args.only in ("finite_t", "differentiation", "self_consistency"):
        # one secondary workload alone, for profiling; rank 0 prints it
        import torch
        torch.cuda.set_device(local_rank)
        if args.only == "finite_t":
            out = finite_t_workload(dmfted, local_rank, args.steps, args.warmup)
        elif args.only == "self_consistency":
            out = dmft_workload(dmfted, local_rank, args.steps, args.warmup)
            out.pop("fit_host")
        else:
            s64 = make_solver(dmfted, dmfted.FP64, local_rank)
            out = differentiation_workload(dmfted, local_rank, args.steps, args.warmup, s64,
                                           s64.sector_index(NUP, NDW), seeded_bath())
            out.pop("chi2_host")
            s64.close()
        if rank == 0:
            print(json.dumps({args.only: out}))
        return
    res, dim, hv32, hv64, extra = run_ours(args, rank, world, local_rank)
    mixed, fp64 = res[dmfted.MIXED], res[dmfted.FP64]
    t_mixed = max_over_ranks(sum(mixed["ms"]) / 1e3, world)
    t_fp64 = max_over_ranks(sum(fp64["ms"]) / 1e3, world)
    t_e2e = max_over_ranks(statistics.mean(mixed["e2e_ms"]) / 1e3, world)
    value = world * args.steps / t_mixed
    peak, peak_kind = measured_peak_gbs()
    hv_bytes32 = 2 * dim * 4
    # the dominant kernel, timed live over the timed solves: every H*v launch
    # (fused Lanczos steps and plain products, FP32 and the FP64 refinement)
    hvt = mixed["hvt"]
    achieved = hvt["bytes"] / (hvt["ms"] * 1e-3) / 1e9
    per_launch = hvt["bytes"] / max(1, hvt["launches"])
    # ncu DRAM bytes of the fused FP32 step on the 7/7 sector, scaled by the
    # algorithmic bytes per launch
    prof = ncu_traffic("k_hxv_lean_lz_ns14_fp32")
    traffic = prof * per_launch / (3 * dim * 4) if prof else None
    g_err = float(np.abs(mixed["g"] - fp64["g"]).max())
    e_err = abs(mixed["e0"] - fp64["e0"]) / abs(fp64["e0"])
    pins = config_pins()
    vs_oracle = None
    if pins is not None and "cfg3_gmats" in pins:
        e_ref = float(pins["cfg3_e0"])
        vs_oracle = dict(fixture="tests/golden/config_pins.npz cfg3 (oracle solve of the same "
                                 "sector and bath)")
        for name, r in (("mixed", mixed), ("fp64", fp64)):
            vs_oracle[name] = dict(dE0_rel=abs(r["e0"] - e_ref) / abs(e_ref),
                                   max_dG=float(np.abs(r["g"][0, 0, 0, 0] -
                                                       pins["cfg3_gmats"]).max()),
                                   max_d_docc=float(np.abs(r["obs"]["docc"] -
                                                           pins["cfg3_docc"]).max()))
    if world > 1:
        dist_barrier(world)
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    line = dict(
        metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps,
        warmup=args.warmup, ms_per_step=t_mixed / args.steps * 1e3, higher_is_better=True,
        scaling="weak", vs_baseline=None, dtype="f32+f64", data="synthetic",
        config={"workload": "impurity solve Ns=14 (Nbath=13, U=3, beta=100) sector 7/7 "
                            "dim 11778624: Lanczos GS (residual tol 1e-12) + observables + "
                            "particle/hole chains (200 steps) + G, Sigma on Lmats=4096",
                "lanc_nstates_sector": 1,
                "precision": "mixed (FP32 vectors, compensated FP64 alpha/beta, FP64 refinement, GF chains with 20 leading FP64 steps)",
                "parallelism": (f"lattice: {world} inequivalent sites, one per GPU, all-reduce "
                                f"of G, Sigma and observables per step" if world > 1 else
                                "single site, 1 GPU"),
                "l2": "flushed (256 MB write) between steps",
                "seed": SEED},
        fp64_dropin=dict(ms_per_step=t_fp64 / args.steps * 1e3,
                         speedup_mixed_vs_fp64=t_fp64 / t_mixed,
                         mixed_vs_fp64_dE0_rel=e_err, mixed_vs_fp64_max_dG=g_err),
        vs_oracle=vs_oracle,
        hv=dict(dim=dim, fp32_us=hv32 * 1e3, fp64_us=hv64 * 1e3,
                fp32_gbs=hv_bytes32 / (hv32 * 1e-3) / 1e9,
                fp64_gbs=2 * dim * 8 / (hv64 * 1e-3) / 1e9,
                hv_per_sec_fp32=1e3 / hv32),
        phases_ms=dict(mixed=mixed["tm"], fp64=fp64["tm"]),
        roofline=dict(bound="hbm", achieved=achieved, peak=peak, unit="GB/s",
                      frac=achieved / peak, traffic=traffic,
                      kernel="k_hxv_lean (fused Lanczos step + plain H*v), every launch of "
                             "K further solves run with an event pair around each H*v",
                      peak_source=peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
                      launches=hvt["launches"], bytes_per_launch=per_launch,
                      avg_launch_us=hvt["ms"] * 1e3 / max(1, hvt["launches"]),
                      share_of_solve=hvt["ms"] / hvt["solve_ms"]),
        e2e=dict(value=world / t_e2e, unit=UNIT, h2d_bytes_per_step=2 * NBATH * 8,
                 d2h_bytes_per_step=2 * LMATS * 16 + 5 * 8),
        gpu_launches=int(mixed["launches"]),
        clocks=mixed["clocks"],
    )
    chi2_host = fit_host = None
    if extra:
        chi2_host = extra["differentiation"].pop("chi2_host")
        fit_host = extra["self_consistency"].pop("fit_host")
        line.update(extra)
    if not args.no_cpu_baseline and world == 1:
        hv_per_step, nl = reference_hv_per_step()
        t_map, t_hv = cpu_sample(nthreads, 2)
        sec = cpu_step_seconds(t_map, t_hv, hv_per_step)
        line["cpu_baseline"] = dict(
            value=1.0 / sec, unit=UNIT, cores=nthreads, kind="port-extrapolated",
            sample=f"2 steps of the oracle's plain Lanczos recurrence (directMatVec_cc, "
                   f"complex128, binary-search map, {nthreads} threads) on the 7/7 sector + "
                   f"the map build, scaled to {hv_per_step} H*v per DMFT step ({nl} "
                   f"plain-Lanczos steps, the second pass, 2 x {NGF} chain steps); "
                   f"{t_hv:.2f} s per step")
        line["cpu_baseline"]["best_cpu_factored"] = best_cpu_line(nthreads, hv_per_step)
        if chi2_host is not None:
            line["differentiation"]["chi2"]["cpu_baseline"] = chi2_cpu(chi2_host)
        if fit_host is not None:
            line["self_consistency"]["fit_batch"]["cpu_baseline"] = fit_cpu(fit_host)
    print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
