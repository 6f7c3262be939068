"""Generate tests/golden/config_pins.npz: oracle answers for the workload
configurations, so that the GPU tests (tests/test_gpu_configs.py) compare the
solver with the CPU restatement of the reference at the full sizes.

  cfg2  single orbital, Nbath=11 (Ns=12), U=3, beta=100, half filling, bath
        seed 2; sector 6/6 (dim 853,776): T=0 solve with Neigen=1 (the ground
        state), observables, particle and hole chains (200 steps), G(iwn) on
        Lmats=4096.
  cfg3  single orbital, Nbath=13 (Ns=14), U=3, beta=100, bath seed 1; sector
        7/7 (dim 11,778,624): the same solve.  One oracle H*v at this size
        costs about 1.4 s on 16 threads, the solve about 560 of them.
        Besides the solve, a check of the product itself: <w|H|v> and 2048
        sampled entries of Hv for two seeded vectors (the full vectors would
        be 188 MB each).
  cfg4  two orbitals, Nbath=4 per orbital (Ns=10), U=3, Ust=2, Jh=0.5,
        beta=50, Nspin=2 with the same bath for both spins, bath seed 4
        (e ~ U[-1.5,1.5], V = 0.4 + U[-0.1,0.1]): every one of the 121
        sectors diagonalised, lanc_nstates_total=16, Neigen=6 per sector,
        the Boltzmann-weighted observables and G(iwn) on Lmats=4096.
  cfg4t the cfg4 solve with ed_twin on.

The oracle is the restatement in oracle/ (test infrastructure); every number
here is what it computes.  Run once on a CPU host:

    python tests/golden/make_config_pins.py [cfg2] [cfg3] [cfg4] [cfg4t]

(cfg3 takes tens of minutes on 8 cores; the others a minute or two).  An
existing npz is updated in place for the configurations named.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

OUT = os.path.join(HERE, "config_pins.npz")
LMATS = 4096


def bath_2orb(seed=4, norb=2, nbath=4):
    rng = np.random.default_rng(seed)
    e = rng.uniform(-1.5, 1.5, size=(norb, nbath))
    v = 0.4 + rng.uniform(-0.1, 0.1, size=(norb, nbath))
    return e, v


def cfg4_model():
    e, v = bath_2orb()
    return O.Model(norb=2, nbath=4, nspin=2, uloc=(3.0, 3.0, 0.0), ust=2.0, jh=0.5, beta=50.0,
                   e=np.stack([e, e]), v=np.stack([v, v]))


def single_orbital(nbath, seed):
    return O.seeded_model(seed, norb=1, nbath=nbath, u=3.0, beta=100.0)


def t0_pin(prefix, m, nup, ndw, nthreads, out):
    t0 = time.time()
    r = O.solve_t0(m, sectors=[(nup, ndw)], nstates_sector=1, lmats=LMATS, nthreads=nthreads)
    out[prefix + "_e0"] = np.array(r["e0"])
    for k in ("dens", "dens_up", "dens_dw", "docc", "magz"):
        out[prefix + "_" + k] = r["obs"][k]
    out[prefix + "_gmats"] = r["gmats"][0, 0]
    out[prefix + "_smats"] = r["smats"][0, 0]
    for c in r["chains"]:
        tag = "p" if c["particle"] else "h"
        out[f"{prefix}_alpha_{tag}"] = c["alpha"]
        out[f"{prefix}_beta_{tag}"] = c["beta"]
        out[f"{prefix}_norm2_{tag}"] = np.array(c["norm2"])
    out[prefix + "_nlanc"] = np.array(r["nlanc"])
    print(f"{prefix}: E0={r['e0']:.15f} ({time.time() - t0:.0f} s)", flush=True)


def hv_pin(prefix, m, nup, ndw, nthreads, out):
    hm = O.build_sector(m.ns, nup, ndw)
    rng = np.random.default_rng(123)
    v = rng.uniform(-1.0, 1.0, hm.size)
    w = rng.uniform(-1.0, 1.0, hm.size)
    hv = O.hxv(m, hm, v.astype(np.complex128), nthreads=nthreads).real
    idx = np.sort(rng.choice(hm.size, 2048, replace=False))
    out[prefix + "_hv_wHv"] = np.array(float(w @ hv))
    out[prefix + "_hv_idx"] = idx.astype(np.int64)
    out[prefix + "_hv_val"] = hv[idx]
    out[prefix + "_hv_norm"] = np.array(float(np.linalg.norm(hv)))


def main(which):
    nthreads = O.lib().or_host_threads()
    out = dict(np.load(OUT)) if os.path.exists(OUT) else {}
    if "cfg2" in which:
        t0_pin("cfg2", single_orbital(11, 2), 6, 6, nthreads, out)
    if "cfg3" in which:
        m = single_orbital(13, 1)
        hv_pin("cfg3", m, 7, 7, nthreads, out)
        t0_pin("cfg3", m, 7, 7, nthreads, out)
    if "cfg4" in which:
        t0 = time.time()
        r = O.solve_finite_t(cfg4_model(), lmats=LMATS, nstates_total=16, nthreads=nthreads)
        out["cfg4_e"] = np.array([s[0] for s in r["states"]])
        out["cfg4_sector"] = np.array([s[1] for s in r["states"]], np.int32)
        out["cfg4_zeta"] = np.array(r["zeta"])
        for k in ("dens", "dens_up", "dens_dw", "docc", "magz"):
            out["cfg4_" + k] = r["obs"][k]
        out["cfg4_gmats"] = r["gmats"]
        print(f"cfg4: {len(r['states'])} states, Z={r['zeta']:.12f} ({time.time() - t0:.0f} s)",
              flush=True)
    if "cfg4t" in which:
        # the same solve with ed_twin (twin entries for the nup != ndw sectors)
        t0 = time.time()
        r = O.solve_finite_t(cfg4_model(), lmats=LMATS, nstates_total=16, nthreads=nthreads,
                             twin=True)
        out["cfg4t_e"] = np.array([s[0] for s in r["states"]])
        out["cfg4t_sector"] = np.array([s[1] for s in r["states"]], np.int32)
        out["cfg4t_zeta"] = np.array(r["zeta"])
        for k in ("dens", "dens_up", "dens_dw", "docc", "magz"):
            out["cfg4t_" + k] = r["obs"][k]
        out["cfg4t_gmats"] = r["gmats"]
        print(f"cfg4t: {len(r['states'])} states, Z={r['zeta']:.12f} ({time.time() - t0:.0f} s)",
              flush=True)
    np.savez_compressed(OUT, **out)


if __name__ == "__main__":
    main(sys.argv[1:] or ["cfg2", "cfg4", "cfg4t", "cfg3"])
