"""Time the on-the-fly H*v of one sector through the library.

    python dmft-ed_b200/dmfted/hvbench.py --nbath 13 --sector 7 7 --fp32 --fused

Builds the single- or multi-orbital model with a seeded bath (e_k ~ U[-1,1],
V_k = 0.5 + U[-0.1,0.1], numpy default_rng(seed)), selects the sector and
times `reps` launches after `warmup` with CUDA events on the library's
stream (dmfted_time_hxv).  Prints the average time per launch and the
algorithmic bandwidth: read x (and v_prev for the fused Lanczos step), write
y, at the vector precision.
"""
import argparse
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import dmfted  # noqa: E402


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--norb", type=int, default=1)
    ap.add_argument("--nbath", type=int, default=13)
    ap.add_argument("--u", type=float, default=3.0)
    ap.add_argument("--sector", type=int, nargs=2, default=(7, 7), metavar=("NUP", "NDW"))
    ap.add_argument("--fp32", action="store_true", help="float32 vectors (default float64)")
    ap.add_argument("--fused", action="store_true", help="the fused Lanczos-step variant")
    ap.add_argument("--step", action="store_true",
                    help="the whole Lanczos step (fused product, w = u - a x, |w|)")
    ap.add_argument("--chain-order", action="store_true",
                    help="the vector order of Green's-function chains")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--reps", type=int, default=50)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    rng = np.random.default_rng(a.seed)
    e = rng.uniform(-1.0, 1.0, size=(a.norb, a.nbath))
    v = 0.5 + rng.uniform(-0.1, 0.1, size=(a.norb, a.nbath))
    p = dmfted.default_params(norb=a.norb, nbath=a.nbath, uloc=[a.u] * a.norb, lmats=16,
                              lreal=0, device=a.device)
    with dmfted.EDSolver(p) as s:
        s.set_bath(np.concatenate([e.reshape(-1), v.reshape(-1)]))
        isec = s.sector_index(*a.sector)
        s.setup_hv_sector(isec)
        dim = s.sector_dim(isec)
        ms = s.time_hxv(fp32=a.fp32, warmup=a.warmup, reps=a.reps, fused=a.fused,
                        chain_order=a.chain_order, whole_step=a.step)
    es = 4 if a.fp32 else 8
    # algorithmic bytes: read x (and v_prev), write y; the whole step has the
    # same three vectors (u is an intermediate)
    nbytes = (3 if (a.fused or a.step) else 2) * dim * es
    print(f"sector {a.sector[0]}/{a.sector[1]} dim {dim} {'fp32' if a.fp32 else 'fp64'}"
          f"{' fused' if a.fused else ''}{' step' if a.step else ''}"
          f"{' chain-order' if a.chain_order else ''}: "
          f"{ms * 1e3:.1f} us/launch, {nbytes / (ms * 1e-3) / 1e9:.0f} GB/s algorithmic")


if __name__ == "__main__":
    main()
