"""Seeded synthetic impurity models shared by the tests (test helpers).

Bath distributions follow the workload definitions: e_k ~ U[-1,1],
V_k = 0.5 + U[-0.1,0.1] from numpy.random.default_rng(seed)."""
import numpy as np

import oracle as O


def golden_models():
    """Models of tests/golden/pins.npz as oracle.Model objects + their pins."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "pins.npz"))
    out = []
    for ic in range(int(z["ncases"])):
        g = lambda k: z[f"c{ic}_{k}"]
        norb, nbath, nspin = int(g("norb")), int(g("nbath")), int(g("nspin"))
        e, v = g("e")[:nspin], g("v")[:nspin]
        hl = np.zeros((nspin, nspin, norb, norb), complex)
        for s in range(nspin):
            hl[s, s] = np.diag(g("hloc_diag")[s]) + g("hloc_off")[s]
        jx = float(g("jx")) if f"c{ic}_jx" in z else 0.0
        jp = float(g("jp")) if f"c{ic}_jp" in z else 0.0
        m = O.Model(norb=norb, nbath=nbath, nspin=nspin, uloc=tuple(g("uloc")), ust=float(g("ust")),
                    jh=float(g("jh")), jx=jx, jp=jp, jhflag=(jx != 0.0 or jp != 0.0),
                    xmu=float(g("xmu")), hfmode=bool(g("hfmode")), e=e, v=v, hloc=hl)
        out.append((m, g("sectors"), g("low")))
    return out


def hloc_fortran(model):
    return np.asfortranarray(model.hloc)
