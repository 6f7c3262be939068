"""The C-ABI library: loads on a machine without a GPU, exports every entry
point include/dmfted.h declares, and fails loudly (status code, message) when
no device is present -- there is no host fallback."""
import ctypes as C
import os
import re

import pytest

import dmfted

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "dmfted.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dmfted_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert sorted(dmfted.EXPORTS) == declared_symbols()


def test_library_exports_every_declared_symbol():
    L = C.CDLL(dmfted.library_path())
    for name in declared_symbols():
        assert hasattr(L, name), name


def test_defaults_match_reference_input_vars():
    p = dmfted.default_params()
    # ED_INPUT_VARS.f90:111-176
    assert (p.norb, p.nbath, p.nspin) == (1, 6, 1)
    assert p.uloc[0] == 2.0 and p.beta == 1000.0 and p.hfmode == 1
    assert (p.lmats, p.lreal, p.lanc_niter, p.lanc_ngfiter) == (5000, 5000, 512, 200)
    assert p.lanc_tolerance == 1e-12 and p.lanc_dim_threshold == 256
    assert (p.lanc_nstates_sector, p.lanc_nstates_total, p.lanc_nstates_step) == (6, 1, 2)
    assert p.gs_threshold == 1e-9 and p.cutoff == 1e-9 and p.eps == 0.01


def test_bath_dimension():
    # get_bath_dimension, normal bath: 2*Nspin*Norb*Nbath (ED_BATH/user_aux.f90)
    assert dmfted.get_bath_dimension(dmfted.default_params(norb=2, nbath=4, nspin=2)) == 32
    assert dmfted.get_bath_dimension(dmfted.default_params(nbath=7)) == 14


def test_argument_errors_are_status_codes():
    # invalid configurations are rejected before any device work
    with pytest.raises(dmfted.DmftedError) as e:
        dmfted.EDSolver(dmfted.default_params(norb=4))
    assert e.value.code == dmfted.ERR_UNSUPPORTED
    with pytest.raises(dmfted.DmftedError) as e:
        dmfted.EDSolver(dmfted.default_params(nspin=3))
    assert e.value.code == dmfted.ERR_UNSUPPORTED


def test_no_gpu_fails_loudly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(dmfted.DmftedError) as e:
        dmfted.EDSolver(dmfted.default_params(nbath=3))
    assert e.value.code == dmfted.ERR_CUDA
