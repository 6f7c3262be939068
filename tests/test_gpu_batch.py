"""The persistent work-queue path (one CTA per sector eigensolve or per
Green's-function chain) against the grid-wide path on the same problems, and
both against the oracle: finite-temperature eigenspace, observables and
G(iwn), including a forced split of the eigensolve into several launches."""
import os

import numpy as np
import pytest

import dmfted
import oracle as O

pytestmark = pytest.mark.gpu


def split_model(seed, norb, nbath, beta, u=3.0, ust=0.0, jh=0.0):
    rng = np.random.default_rng(seed)
    e1 = rng.uniform(-1.5, 1.5, (norb, nbath))
    v1 = 0.4 + rng.uniform(-0.1, 0.1, (norb, nbath))
    e = np.stack([e1, e1 + rng.uniform(-0.2, 0.2, (norb, nbath))])
    v = np.stack([v1, v1 + rng.uniform(-0.05, 0.05, (norb, nbath))])
    ul = [u] * norb + [0.0] * (3 - norb)
    return O.Model(norb=norb, nbath=nbath, nspin=2, uloc=tuple(ul), ust=ust, jh=jh, beta=beta,
                   e=e, v=v)


def solve(m, env, precision=0, total=16, lmats=256):
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        p = dmfted.default_params(norb=m.norb, nbath=m.nbath, nspin=m.nspin, uloc=list(m.uloc),
                                  ust=m.ust, jh=m.jh, beta=m.beta, lmats=lmats, lreal=0,
                                  lanc_nstates_total=total, precision=precision)
        s = dmfted.EDSolver(p)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    s.ed_solve(m.bath_array())
    e, secs, z = s.eigenspace()
    out = dict(e=e, secs=secs, z=z, g=s.ed_get_gimp_matsubara(), obs=s.observables(),
               launches=s.launch_count())
    s.close()
    return out


def agree(a, b, tol_e=1e-10, tol_g=1e-9):
    assert np.array_equal(a["secs"], b["secs"])
    assert np.allclose(a["e"], b["e"], rtol=0, atol=tol_e * max(1.0, np.abs(b["e"]).max()))
    assert abs(a["z"] - b["z"]) <= 1e-10 * b["z"]
    assert np.abs(a["g"] - b["g"]).max() <= tol_g
    for k in ("dens", "docc", "magz"):
        assert np.allclose(a["obs"][k], b["obs"][k], rtol=0, atol=1e-9), k


def test_batch_matches_grid_and_oracle_finite_t():
    m = split_model(21, 2, 2, beta=50.0, ust=2.0, jh=0.5)
    grid = solve(m, {"DMFTED_BATCH_MAX_DIM": "0"})
    batch = solve(m, {"DMFTED_BATCH_MAX_DIM": str(1 << 17)})
    agree(batch, grid)
    assert batch["launches"] < grid["launches"] / 5
    ref = O.solve_finite_t(m, lmats=256, nstates_total=16, nthreads=4)
    re = np.array([x[0] for x in ref["states"]])
    assert np.allclose(batch["e"], re, rtol=0, atol=1e-10 * max(1.0, np.abs(re).max()))
    for ispin in range(2):
        for a in range(2):
            assert np.abs(batch["g"][ispin, ispin, a, a] - ref["gmats"][ispin, a]).max() <= 1e-8


def test_batch_waves_split_by_memory_budget():
    # a 1 MB budget puts every sector of the eigensolve in its own launch
    m = split_model(22, 1, 4, beta=30.0)
    one = solve(m, {"DMFTED_BATCH_MAX_DIM": str(1 << 17)}, total=8)
    waves = solve(m, {"DMFTED_BATCH_MAX_DIM": str(1 << 17), "DMFTED_BATCH_BUDGET_MB": "1"},
                  total=8)
    agree(waves, one, tol_e=1e-12, tol_g=1e-12)


def test_batch_mixed_precision_close_to_fp64():
    # the mixed form keeps FP64 eigenpairs and FP64 batched chains: the FP64 bars
    m = split_model(23, 2, 2, beta=50.0, ust=2.0, jh=0.5)
    f64 = solve(m, {"DMFTED_BATCH_MAX_DIM": str(1 << 17)}, precision=0)
    mix = solve(m, {"DMFTED_BATCH_MAX_DIM": str(1 << 17)}, precision=1)
    assert np.array_equal(mix["secs"], f64["secs"])
    assert np.abs(mix["e"] - f64["e"]).max() <= 1e-10 * max(1.0, np.abs(f64["e"]).max())
    assert np.abs(mix["g"] - f64["g"]).max() <= 1e-8
    # FP32 batched chains (measurement switch) stay within 1e-4
    f32 = solve(m, {"DMFTED_BATCH_MAX_DIM": str(1 << 17), "DMFTED_BATCH_CHAINS_FP32": "1"},
                precision=1)
    assert np.abs(f32["g"] - f64["g"]).max() <= 1e-4


@pytest.mark.parametrize("cl_eigs,cl_gf", [("2", "2"), ("4", "8"), ("8", "4"), ("16", "16")])
def test_batch_clusters_match_single_cta(cl_eigs, cl_gf):
    # one job shared by a cluster of CTAs (interleaved elements, sums folded
    # through distributed shared memory) gives the single-CTA result
    m = split_model(24, 2, 2, beta=50.0, ust=2.0, jh=0.5)
    # 8 states per CTA: the larger sectors of this small model are shared
    base = {"DMFTED_BATCH_MAX_DIM": str(1 << 17), "DMFTED_BATCH_CLUSTER_MIN": "8"}
    one = solve(m, dict(base, DMFTED_BATCH_CLUSTER_EIGS="1", DMFTED_BATCH_CLUSTER_GF="1"))
    many = solve(m, dict(base, DMFTED_BATCH_CLUSTER_EIGS=cl_eigs, DMFTED_BATCH_CLUSTER_GF=cl_gf))
    agree(many, one, tol_e=1e-12, tol_g=1e-11)


def test_batch_autotune_picks_measured_cluster_and_agrees():
    # the autotuner times candidate cluster sizes of each batched phase on
    # first use of a job shape, keeps the fastest, and its results agree
    # with the fixed rule's; later solves of the same shapes re-use the
    # choices (no job shape is measured twice)
    m = split_model(25, 2, 2, beta=50.0, ust=2.0, jh=0.5)
    base = {"DMFTED_BATCH_MAX_DIM": str(1 << 17), "DMFTED_BATCH_CLUSTER_MIN": "8"}
    rule = solve(m, dict(base, DMFTED_AUTOTUNE="0"))
    env = dict(base, DMFTED_AUTOTUNE="1")  # the tuner is opt-in
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        p = dmfted.default_params(norb=m.norb, nbath=m.nbath, nspin=m.nspin, uloc=list(m.uloc),
                                  ust=m.ust, jh=m.jh, beta=m.beta, lmats=256, lreal=0,
                                  lanc_nstates_total=16)
        s = dmfted.EDSolver(p)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    s.ed_solve(m.bath_array())
    log = s.autotune_log()
    assert any(l.startswith("eigs ") and "chosen CL" in l for l in log), log
    assert any(l.startswith("chains ") and "chosen CL" in l for l in log), log
    for line in log:  # the fixed rule's size is always among the measured candidates
        size = line.split("(rule ")[1].rstrip(")")
        assert f" {size}=" in line, line
    e, secs, z = s.eigenspace()
    g = s.ed_get_gimp_matsubara()
    assert np.array_equal(secs, rule["secs"])
    assert np.allclose(e, rule["e"], rtol=0, atol=1e-10 * max(1.0, np.abs(rule["e"]).max()))
    assert np.abs(g - rule["g"]).max() <= 1e-9
    s.ed_solve(m.bath_array())
    s.ed_solve(m.bath_array())
    keys = [l.split(" ->")[0] for l in s.autotune_log()]
    assert len(keys) == len(set(keys))  # each job shape measured once
    s.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_grid_chains_on_two_lanes_equal_in_turn(precision):
    # the grid-wide chains run two at a time on two streams, each with its own
    # reduction scratch and buffers: the same fixed-order arithmetic as one at
    # a time, so the results are bit-identical (odd number of chains included)
    m = split_model(23, 2, 2, beta=50.0, ust=2.0, jh=0.5)
    one = solve(m, {"DMFTED_BATCH_MAX_DIM": "0", "DMFTED_CHAIN_LANES": "1"}, precision=precision)
    two = solve(m, {"DMFTED_BATCH_MAX_DIM": "0", "DMFTED_CHAIN_LANES": "2"}, precision=precision)
    assert np.array_equal(one["g"], two["g"])
    assert np.array_equal(one["e"], two["e"])
    for k in ("dens", "docc", "magz"):
        assert np.array_equal(one["obs"][k], two["obs"][k]), k


@pytest.mark.parametrize("batch_dim", [str(1 << 17), "0"])
def test_jhflag_finite_t_batch_and_grid_match_oracle(batch_dim):
    # spin exchange and pair hopping (HxVint.f90:45-97) in the batched
    # eigensolve and chains (and, with batching off, the grid-wide product)
    m = split_model(23, 2, 2, beta=30.0, ust=2.0, jh=0.5)
    m.jx, m.jp, m.jhflag = 0.4, 0.3, True
    p = dict(norb=2, nbath=2, nspin=2, uloc=list(m.uloc), ust=m.ust, jh=m.jh, jx=m.jx, jp=m.jp,
             jhflag=1, beta=m.beta, lmats=128, lreal=0, lanc_nstates_total=12)
    old = os.environ.get("DMFTED_BATCH_MAX_DIM")
    os.environ["DMFTED_BATCH_MAX_DIM"] = batch_dim
    try:
        s = dmfted.EDSolver(dmfted.default_params(**p))
    finally:
        if old is None:
            os.environ.pop("DMFTED_BATCH_MAX_DIM", None)
        else:
            os.environ["DMFTED_BATCH_MAX_DIM"] = old
    s.ed_solve(m.bath_array())
    e, secs, z = s.eigenspace()
    ref = O.solve_finite_t(m, lmats=128, nstates_total=12, nthreads=4)
    re = np.array([x[0] for x in ref["states"]])
    assert np.allclose(e, re, rtol=0, atol=1e-10 * max(1.0, np.abs(re).max()))
    assert np.array_equal(secs, np.array([x[1] for x in ref["states"]]))
    g = s.ed_get_gimp_matsubara()
    for ispin in range(2):
        for a in range(2):
            assert np.abs(g[ispin, ispin, a, a] - ref["gmats"][ispin, a]).max() <= 1e-8
    assert np.allclose(s.ed_get_doubles(), ref["obs"]["doubles"], atol=1e-9)
    s.close()
