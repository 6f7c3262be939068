"""The state list file of a finite-temperature solve: print_state_list's
state_list.ed format written by the library equals the oracle's restatement
of the Fortran format built from the same eigenspace, byte for byte; reading
it back as state_list.restart sets lanc_nstates_total and neigen_sector as
setup_pointers_normal does (ED_SETUP.f90:403-425), and a row whose nup/ndw do
not match its sector is refused with the reference's message."""
import numpy as np
import pytest

import dmfted
import oracle as O

pytestmark = pytest.mark.gpu


def solved():
    rng = np.random.default_rng(3)
    p = dmfted.default_params(norb=2, nbath=2, nspin=2, uloc=[3.0, 3.0], ust=2.0, jh=0.5,
                              beta=20.0, lmats=256, lreal=0, lanc_nstates_total=16)
    nb = dmfted.get_bath_dimension(p)
    bath = np.concatenate([rng.uniform(-1.5, 1.5, nb // 2), 0.4 + rng.uniform(-0.1, 0.1, nb // 2)])
    s = dmfted.EDSolver(p)
    s.ed_solve(bath)
    return s, p


def test_print_and_read_state_list(tmp_path):
    s, p = solved()
    try:
        f = tmp_path / "state_list.ed"
        s.print_state_list(f)
        e, secs, _ = s.eigenspace()
        t = s.sector_tables()
        want = O.print_state_list_text(e, secs, t["getnup"], t["getndw"], t["getdim"], p.beta)
        assert f.read_text() == want
        lines = f.read_text().splitlines()
        assert len(lines) == len(e) + 1
        with dmfted.EDSolver(p) as s2:
            s2.read_state_list(f)
            ne, tot = s2.get_neigen()
            assert tot == len(lines)
            counts = np.bincount(secs - 1, minlength=ne.size)
            assert np.array_equal(ne, np.maximum(1, counts))
            # a row that names a sector with the wrong nup/ndw
            bad = lines[:]
            row = bad[1]
            nup = int(row[43:46])
            bad[1] = row[:43] + f"{(nup + 1) % 5:3d}" + row[46:]
            g = tmp_path / "state_list.restart"
            g.write_text("\n".join(bad) + "\n")
            with pytest.raises(dmfted.DmftedError) as err:
                s2.read_state_list(g)
            assert "nup!=getnup(isector)" in str(err.value)
    finally:
        s.close()
