"""The bath file (hamiltonian.restart / .used) written and read by the
library, against the oracle's restatement of write_dmft_bath's Fortran
formats (byte for byte), and the read of init_dmft_bath.  No device needed."""
import os

import numpy as np
import pytest

import dmfted
import oracle as O


@pytest.mark.parametrize("norb,nspin,nbath", [(1, 1, 7), (2, 2, 4), (3, 1, 2)])
def test_save_bath_matches_fortran_format(tmp_path, norb, nspin, nbath):
    p = dmfted.default_params(norb=norb, nspin=nspin, nbath=nbath)
    nb = dmfted.get_bath_dimension(p)
    rng = np.random.default_rng(norb * 10 + nspin)
    bath = np.concatenate([rng.uniform(-3, 3, nb // 2), rng.uniform(-1, 1, nb // 2)])
    bath[0] = -0.0
    bath[1] = 123.456789012345678
    f = tmp_path / "hamiltonian.restart"
    dmfted.save_bath(p, f, bath)
    assert f.read_text() == O.write_dmft_bath_text(bath, norb, nspin, nbath)
    back = dmfted.read_bath(p, f)
    assert np.abs(back - bath).max() <= 5e-13
    # a second round trip reproduces the file exactly
    g = tmp_path / "again.restart"
    dmfted.save_bath(p, g, back)
    assert g.read_text() == f.read_text()


def test_read_bath_row_count(tmp_path):
    """init_dmft_bath reads min(file lines, Nbath) rows after the header: a
    file with extra lines is read up to Nbath rows; a short file runs the read
    past its end, an error as in the reference."""
    p = dmfted.default_params(norb=1, nspin=1, nbath=2)
    f = tmp_path / "h.restart"
    f.write_text("#Ek_l1_s1 Vk_l1_s1\n  0.5  0.25\n -0.5 0.125\n 9 9\n")
    got = dmfted.read_bath(p, f, np.arange(4, dtype=np.float64))
    assert np.array_equal(got, [0.5, -0.5, 0.25, 0.125])
    p5 = dmfted.default_params(norb=1, nspin=1, nbath=5)
    with pytest.raises(dmfted.DmftedError) as e:
        dmfted.read_bath(p5, f)
    assert "end of file" in str(e.value)


def test_bath_file_errors(tmp_path):
    p = dmfted.default_params(norb=1, nspin=1, nbath=2)
    with pytest.raises(dmfted.DmftedError) as e:
        dmfted.read_bath(p, tmp_path / "missing.restart")
    assert e.value.code == dmfted.ERR_ARG
    f = tmp_path / "bad.restart"
    f.write_text("# header\n 1.0 x\n")
    with pytest.raises(dmfted.DmftedError):
        dmfted.read_bath(p, f)
    with pytest.raises(dmfted.DmftedError) as e:
        dmfted.save_bath(p, tmp_path / "h.restart", np.zeros(3))
    assert "wrong bath dimensions" in str(e.value)


def test_fortran_es_format():
    assert O._fortran_es(1.0, 19, 12) == " 1.000000000000E+00"
    assert O._fortran_es(3.5e-218, 19, 12) == " 3.500000000000-218"
    assert O._fortran_es(2.0e-5, 19, 12) == " 2.000000000000E-05"


def test_observable_file_formats():
    """The oracle's restatement of write_legend / write_energy_info /
    write_energy (ED_OBSERVABLES.f90:715-774,851-857): "#" then A10 labels
    16 characters apart (A10,6X), the 6X after the last label not transmitted;
    the column numbers of z and sig step by Nspin per spin, as the reference
    writes them."""
    t = O.observables_legend_text(1, 1)
    assert t.startswith("#   1dens_1      ") and t.endswith("  12sig_1s1\n")
    fields = [t[1 + 16 * k:11 + 16 * k].strip() for k in range((len(t) - 1 + 6) // 16)]
    assert fields == ["1dens_1", "2docc_1", "3nup_1", "4ndw_1", "5mag_1", "6s2", "7egs",
                      "8sz2_11", "9n2_11", "10z_1s1", "12sig_1s1"]
    t2 = O.observables_legend_text(2, 2)
    labels = t2[1:].split()
    assert labels[20:24] == ["21z_1s1", "22z_2s1", "23z_1s2", "24z_2s2"]
    assert labels[-1] == "28sig_2s2" and len(labels) == 5 * 2 + 2 + 2 * 4 + 2 * 4
    info, last = O.energy_texts([-1.25, 0.0, 0.5, -0.75], [0.1, 0.2, 0.0, 0.0])
    assert info == ("#" + " ".join(lab.rjust(14) for lab in [
        "1<Hi>", "2<V>=<Hi-Ehf>", "3<Eloc>", "4<Ehf>", "5<Dst>", "6<Dnd>", "7<Dse>",
        "8<Dph>"]) + "\n")
    assert last == ("   -1.250000000   -1.750000000   -0.750000000    0.500000000"
                    "    0.100000000    0.200000000    0.000000000    0.000000000\n")
    rec = O.observables_record_text([1.0], [0.25], [0.5], [0.5], [0.0], 0.375, -3.5,
                                    [[0.375]], [[1.5]], [[1.0]], [[0.0]])
    assert rec == " ".join(f"{x:15.9f}" for x in
                           [1.0, 0.25, 0.5, 0.5, 0.0, 0.375, -3.5, 0.375, 1.5, 1.0, 0.0]) + "\n"
    assert O.f15_9(1e7) == "*" * 15
