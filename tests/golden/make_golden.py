"""Generate tests/golden/pins.npz: known answers that pin the CPU restatement.

The reference ships no tests, golden vectors or output files, and cannot be
built here (Fortran, unvendored SciFortran/DMFT_Tools).  These fixtures are
independent of both the reference and the restatement: the impurity
Hamiltonian is rebuilt from scratch in second quantisation with explicit
Jordan-Wigner matrices (numpy Kronecker products over all 2*Ns levels, level
l = bit l-1 of the reference's |up>|dw> word), diagonalised densely per
(nup, ndw) sector, and the lowest eigenvalues stored.  A test then checks that
the restatement's sector Hamiltonian (oracle/ed_oracle.c) has the same
spectrum, and that its Green's function obeys the analytic U=0 and V=0 limits
computed here.

Run: python tests/golden/make_golden.py   (seconds; deterministic)
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def jw_ops(nlev):
    """Annihilation operators c_l (l = 0..nlev-1) on 2^nlev states, basis
    index = integer word with bit l = occupation of level l, sign convention
    (-1)^(occupied levels below l) (the reference's c(), ED_SETUP.f90:1055)."""
    dim = 1 << nlev
    ops = []
    for l in range(nlev):
        m = np.zeros((dim, dim))
        for w in range(dim):
            if (w >> l) & 1:
                s = bin(w & ((1 << l) - 1)).count("1")
                m[w & ~(1 << l), w] = -1.0 if s & 1 else 1.0
        ops.append(m)
    return ops


def hamiltonian(norb, nbath, e, v, uloc, ust, jh, xmu, hfmode, hloc_diag, hloc_off=None,
                jx=0.0, jp=0.0):
    """Full Fock-space H of the normal-bath impurity model, normal ed_mode.
    e, v: [2 spins][norb][nbath]; hloc_diag: [2][norb]; hloc_off: [2][norb][norb];
    jx, jp: spin-exchange J c+_{a up} c+_{b dw} c_{a dw} c_{b up} and pair hopping
    J c+_{a up} c+_{a dw} c_{b dw} c_{b up} over a != b (the Jhflag terms)."""
    ns = (nbath + 1) * norb
    c = jw_ops(2 * ns)
    cd = [m.T for m in c]
    n = [cd[l] @ c[l] for l in range(2 * ns)]
    H = np.zeros_like(c[0])

    def lev(s, site):
        return site + s * ns

    for s in range(2):
        for a in range(norb):
            H += (hloc_diag[s][a] - xmu) * n[lev(s, a)]
            for k in range(nbath):
                ms = norb + a * nbath + k
                H += e[s][a][k] * n[lev(s, ms)]
                H += v[s][a][k] * (cd[lev(s, a)] @ c[lev(s, ms)] + cd[lev(s, ms)] @ c[lev(s, a)])
            if hloc_off is not None:
                for b in range(norb):
                    if a != b and hloc_off[s][a][b] != 0.0:
                        H += hloc_off[s][a][b] * cd[lev(s, a)] @ c[lev(s, b)]
    for a in range(norb):
        H += uloc[a] * n[lev(0, a)] @ n[lev(1, a)]
        if hfmode:
            H += -0.5 * uloc[a] * (n[lev(0, a)] + n[lev(1, a)]) + 0.25 * uloc[a] * np.eye(H.shape[0])
    for a in range(norb):
        for b in range(a + 1, norb):
            H += ust * (n[lev(0, a)] @ n[lev(1, b)] + n[lev(0, b)] @ n[lev(1, a)])
            H += (ust - jh) * (n[lev(0, a)] @ n[lev(0, b)] + n[lev(1, a)] @ n[lev(1, b)])
            if hfmode:
                nab = n[lev(0, a)] + n[lev(1, a)] + n[lev(0, b)] + n[lev(1, b)]
                eye = np.eye(H.shape[0])
                H += -0.5 * ust * nab + 0.25 * ust * eye
                H += -0.5 * (ust - jh) * nab + 0.25 * (ust - jh) * eye
    for a in range(norb):
        for b in range(norb):
            if a == b:
                continue
            if jx != 0.0:
                H += jx * cd[lev(0, a)] @ cd[lev(1, b)] @ c[lev(1, a)] @ c[lev(0, b)]
            if jp != 0.0:
                H += jp * cd[lev(0, a)] @ cd[lev(1, a)] @ c[lev(1, b)] @ c[lev(0, b)]
    return H, ns


def sector_spectrum(H, ns, nup, ndw, k):
    words = [w for w in range(1 << (2 * ns))
             if bin(w & ((1 << ns) - 1)).count("1") == nup and bin(w >> ns).count("1") == ndw]
    Hs = H[np.ix_(words, words)]
    return np.linalg.eigvalsh(Hs)[:k]


def main():
    rng = np.random.default_rng(20240611)
    cases = []
    # (norb, nbath, uloc, ust, jh, xmu, hfmode, spin-split, hloc)
    specs = [
        (1, 3, [2.0], 0.0, 0.0, 0.0, True, False, False),
        (1, 4, [3.0], 0.0, 0.0, 0.3, True, True, False),
        (1, 4, [1.5], 0.0, 0.0, -0.2, False, False, False),
        (2, 1, [3.0, 2.5], 2.0, 0.5, 0.1, True, False, True),
        (2, 2, [3.0, 3.0], 2.0, 0.5, 0.0, True, True, False),
        (3, 1, [2.0, 2.5, 3.0], 1.5, 0.3, 0.0, True, False, True),
    ]
    out = {}
    for ic, (norb, nbath, uloc, ust, jh, xmu, hf, split, hoff) in enumerate(specs):
        e1 = rng.uniform(-1, 1, (norb, nbath))
        v1 = 0.5 + rng.uniform(-0.1, 0.1, (norb, nbath))
        if split:
            e2 = e1 + rng.uniform(-0.2, 0.2, (norb, nbath))
            v2 = v1 + rng.uniform(-0.05, 0.05, (norb, nbath))
        else:
            e2, v2 = e1.copy(), v1.copy()
        hd = rng.uniform(-0.3, 0.3, (2, norb)) if hoff else np.zeros((2, norb))
        if not split:
            hd[1] = hd[0]
        ho = None
        if hoff and norb > 1:
            t = rng.uniform(-0.2, 0.2, (norb, norb))
            t = 0.5 * (t + t.T)
            np.fill_diagonal(t, 0.0)
            ho = np.stack([t, t if not split else t * 1.1])
        uloc3 = list(uloc) + [0.0] * (3 - len(uloc))
        H, ns = hamiltonian(norb, nbath, [e1, e2], [v1, v2], uloc3, ust, jh, xmu, hf, hd, ho)
        spec = {}
        for nup in range(ns + 1):
            for ndw in range(ns + 1):
                spec[(nup, ndw)] = sector_spectrum(H, ns, nup, ndw, 4)
        sectors = np.array(sorted(spec.keys()), np.int32)
        low = np.full((len(sectors), 4), np.nan)
        for i, s in enumerate(sectors):
            v = spec[tuple(s)]
            low[i, :len(v)] = v
        pre = f"c{ic}_"
        out[pre + "norb"] = norb
        out[pre + "nbath"] = nbath
        out[pre + "nspin"] = 2 if (split or hoff) else 1
        out[pre + "uloc"] = np.array(uloc3)
        out[pre + "ust"] = ust
        out[pre + "jh"] = jh
        out[pre + "xmu"] = xmu
        out[pre + "hfmode"] = int(hf)
        out[pre + "e"] = np.stack([e1, e2])
        out[pre + "v"] = np.stack([v1, v2])
        out[pre + "hloc_diag"] = hd
        out[pre + "hloc_off"] = ho if ho is not None else np.zeros((2, norb, norb))
        out[pre + "sectors"] = sectors
        out[pre + "low"] = low
        cases.append(ic)
    out["ncases"] = len(cases)
    # U = 0 limit: E0(half filling) = 2 * sum of the N/2 lowest one-body levels
    e = rng.uniform(-1, 1, 5)
    v = 0.5 + rng.uniform(-0.1, 0.1, 5)
    h1 = np.zeros((6, 6))
    h1[1:, 1:] = np.diag(e)
    h1[0, 1:] = v
    h1[1:, 0] = v
    out["u0_e"], out["u0_v"] = e, v
    out["u0_levels"] = np.linalg.eigvalsh(h1)
    # a Jhflag case (spin exchange and pair hopping), from its own generator so
    # that the cases above keep their values
    rng2 = np.random.default_rng(20251203)
    for norb, nbath, jx, jp, split in ((2, 2, 0.4, 0.3, False), (3, 1, 0.3, 0.25, True)):
        ic = len(cases)
        e1 = rng2.uniform(-1, 1, (norb, nbath))
        v1 = 0.5 + rng2.uniform(-0.1, 0.1, (norb, nbath))
        e2 = e1 + rng2.uniform(-0.2, 0.2, (norb, nbath)) if split else e1.copy()
        v2 = v1 + rng2.uniform(-0.05, 0.05, (norb, nbath)) if split else v1.copy()
        uloc3 = [3.0] * norb + [0.0] * (3 - norb)
        hd = np.zeros((2, norb))
        H, ns = hamiltonian(norb, nbath, [e1, e2], [v1, v2], uloc3, 2.0, 0.5, 0.0, True, hd,
                            None, jx, jp)
        spec = {}
        for nup in range(ns + 1):
            for ndw in range(ns + 1):
                spec[(nup, ndw)] = sector_spectrum(H, ns, nup, ndw, 4)
        sectors = np.array(sorted(spec.keys()), np.int32)
        low = np.full((len(sectors), 4), np.nan)
        for i, sec in enumerate(sectors):
            lv = spec[tuple(sec)]
            low[i, :len(lv)] = lv
        pre = f"c{ic}_"
        out[pre + "norb"], out[pre + "nbath"] = norb, nbath
        out[pre + "nspin"] = 2 if split else 1
        out[pre + "uloc"] = np.array(uloc3)
        out[pre + "ust"], out[pre + "jh"], out[pre + "xmu"], out[pre + "hfmode"] = 2.0, 0.5, 0.0, 1
        out[pre + "jx"], out[pre + "jp"] = jx, jp
        out[pre + "e"], out[pre + "v"] = np.stack([e1, e2]), np.stack([v1, v2])
        out[pre + "hloc_diag"], out[pre + "hloc_off"] = hd, np.zeros((2, norb, norb))
        out[pre + "sectors"], out[pre + "low"] = sectors, low
        cases.append(ic)
    out["ncases"] = len(cases)
    np.savez_compressed(os.path.join(HERE, "pins.npz"), **out)
    print("wrote", os.path.join(HERE, "pins.npz"), len(cases), "cases")


if __name__ == "__main__":
    main()
