"""Python mirror of the DMFT_ED solver API over the B200 C-ABI (libdmfted.so).

Names follow the reference's Fortran facade (DMFT_ED.f90): ``ed_init_solver``,
``ed_solve``, ``ed_get_sigma_matsubara``, ``ed_get_dens`` ... and the
H*v procedure-pointer contract (``setup_hv_sector`` / ``hxv``).  Every call
goes to the CUDA library; there is no host implementation to fall back on, and
loading fails loudly when the shared object is missing.

Arrays use the reference's shapes: Green's functions are complex
``(Nspin, Nspin, Norb, Norb, L)``; the bath is the flat user array of
``get_bath_dimension()`` entries (e then V, k fastest).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.environ.get("DMFTED_LIB") or os.path.join(os.path.dirname(_HERE), "libdmfted.so")
_lib = None

OK = 0
ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_UNSUPPORTED, ERR_STATE, ERR_NOTCONV, ERR_NORM = range(1, 8)
FP64 = 0
MIXED = 1
CG_DELTA = 0  # cg_scheme: fit the hybridisation Delta(iw_n)
CG_WEISS = 1  # cg_scheme: fit the Weiss field G0(iw_n) (the reference default)


class DmftedError(RuntimeError):
    """A non-zero status from the library; .code is the DMFTED_ERR_* value."""

    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Params(C.Structure):
    """dmfted_params (include/dmfted.h): the ED_INPUT_VARS.f90 variables of the path."""
    _fields_ = [
        ("norb", C.c_int32), ("nbath", C.c_int32), ("nspin", C.c_int32),
        ("hfmode", C.c_int32), ("jhflag", C.c_int32),
        ("uloc", C.c_double * 3),
        ("ust", C.c_double), ("jh", C.c_double), ("jx", C.c_double), ("jp", C.c_double),
        ("xmu", C.c_double), ("beta", C.c_double),
        ("lmats", C.c_int32), ("lreal", C.c_int32),
        ("wini", C.c_double), ("wfin", C.c_double), ("eps", C.c_double),
        ("lanc_niter", C.c_int32), ("lanc_ngfiter", C.c_int32),
        ("lanc_tolerance", C.c_double),
        ("lanc_dim_threshold", C.c_int32), ("lanc_nstates_sector", C.c_int32),
        ("lanc_nstates_total", C.c_int32), ("lanc_nstates_step", C.c_int32),
        ("gs_threshold", C.c_double), ("cutoff", C.c_double),
        ("ed_twin", C.c_int32), ("lfit", C.c_int32), ("cg_weight", C.c_int32),
        ("precision", C.c_int32), ("lanc_ncheck", C.c_int32), ("device", C.c_int32),
        ("lanc_gf_threshold", C.c_double),
        ("cg_niter", C.c_int32), ("cg_scheme", C.c_int32), ("cg_ftol", C.c_double),
        ("cg_stop", C.c_int32), ("cg_eps", C.c_double),
    ]


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)
_vp = C.c_void_p

EXPORTS = {
    "dmfted_default_params": (None, [C.POINTER(Params)]),
    "dmfted_last_error": (C.c_char_p, []),
    "dmfted_version": (C.c_char_p, []),
    "dmfted_init": (C.c_int, [C.POINTER(Params), _dp, C.POINTER(_vp)]),
    "dmfted_free": (C.c_int, [_vp]),
    "dmfted_set_hloc": (C.c_int, [_vp, _dp]),
    "dmfted_get_bath_dimension": (C.c_int, [C.POINTER(Params), _ip]),
    "dmfted_set_bath": (C.c_int, [_vp, _dp, C.c_int32]),
    "dmfted_sector_tables": (C.c_int, [_vp] + [_ip] * 11),
    "dmfted_build_sector": (C.c_int, [_vp, C.c_int32, _ip, C.c_int64]),
    "dmfted_setup_hv_sector": (C.c_int, [_vp, C.c_int32]),
    "dmfted_delete_hv_sector": (C.c_int, [_vp]),
    "dmfted_hxv_c128": (C.c_int, [_vp, C.c_int32, _dp, _dp]),
    "dmfted_hxv_device_f64": (C.c_int, [_vp, _vp, _vp, C.c_int32]),
    "dmfted_hxv_device_f32": (C.c_int, [_vp, _vp, _vp, C.c_int32]),
    "dmfted_lanczos_gs": (C.c_int, [_vp, C.c_int32, _dp, _dp, _ip]),
    "dmfted_gs_lanczos": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32, C.c_double, _dp, _dp,
                                    _ip]),
    "dmfted_lanc_tridiag": (C.c_int, [_vp, C.c_int32, _dp, C.c_int32, _dp, _dp, _ip]),
    "dmfted_lanc_tridiag_noalloc": (C.c_int, [_vp, C.c_int32, _vp, C.c_int32, _vp, _vp, _vp, _vp]),
    "dmfted_add_to_lanczos_gf": (C.c_int, [_vp, C.c_double, C.c_double, C.c_double, C.c_double,
                                           C.c_int32, _dp, _dp, C.c_int32, _dp, _dp]),
    "dmfted_ed_solve": (C.c_int, [_vp, _dp, C.c_int32, _ip, C.c_int32]),
    "dmfted_get_gimp_matsubara": (C.c_int, [_vp, _dp]),
    "dmfted_get_gimp_real": (C.c_int, [_vp, _dp]),
    "dmfted_get_sigma_matsubara": (C.c_int, [_vp, _dp]),
    "dmfted_get_sigma_real": (C.c_int, [_vp, _dp]),
    "dmfted_get_g0imp_matsubara": (C.c_int, [_vp, _dp]),
    "dmfted_get_g0imp_real": (C.c_int, [_vp, _dp]),
    "dmfted_get_observables": (C.c_int, [_vp, _dp, _dp, _dp, _dp, _dp]),
    "dmfted_get_eigenspace": (C.c_int, [_vp, C.c_int32, _dp, _ip, _ip, _dp]),
    "dmfted_get_egs": (C.c_int, [_vp, _dp]),
    "dmfted_get_eimp": (C.c_int, [_vp, _dp]),
    "dmfted_get_doubles": (C.c_int, [_vp, _dp]),
    "dmfted_hf_gradient": (C.c_int, [_vp, _dp, C.c_int32]),
    "dmfted_chi2_delta_batch": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32, _dp, _dp, _dp,
                                          _dp, _dp, _dp]),
    "dmfted_chi2_delta_batch_device": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32, _vp, _vp,
                                                 _vp, _vp, _vp, _vp]),
    "dmfted_chi2_fitgf": (C.c_int, [_vp, _dp, C.c_int32, _dp, C.c_int32, _ip, _dp]),
    "dmfted_cg_fit_batch": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32, _dp, _dp, _dp, _dp,
                                      C.c_int32, C.c_double, _ip, _dp]),
    "dmfted_cg_fit_batch_device": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32, _vp, _vp, _vp,
                                             _vp, C.c_int32, C.c_double, _vp, _vp, _vp]),
    "dmfted_gloc_matsubara_diag": (C.c_int, [_vp, C.c_int32, _dp, _dp, _dp, _dp]),
    "dmfted_gloc_realaxis_diag": (C.c_int, [_vp, C.c_int32, _dp, _dp, _dp, _dp]),
    "dmfted_get_weiss": (C.c_int, [_vp, _dp, _dp, C.c_int32, _dp]),
    "dmfted_save_bath": (C.c_int, [C.c_void_p, C.c_char_p, _dp, C.c_int32]),
    "dmfted_read_bath": (C.c_int, [C.c_void_p, C.c_char_p, _dp, C.c_int32]),
    "dmfted_print_state_list": (C.c_int, [_vp, C.c_char_p]),
    "dmfted_read_state_list": (C.c_int, [_vp, C.c_char_p]),
    "dmfted_print_impg": (C.c_int, [_vp, C.c_char_p, C.c_char_p]),
    "dmfted_print_impsigma": (C.c_int, [_vp, C.c_char_p, C.c_char_p]),
    "dmfted_print_impg0": (C.c_int, [_vp, C.c_char_p, C.c_char_p]),
    "dmfted_read_impsigma": (C.c_int, [_vp, C.c_char_p, C.c_char_p]),
    "dmfted_write_observables": (C.c_int, [_vp, C.c_char_p, C.c_char_p, C.c_int32]),
    "dmfted_write_energy": (C.c_int, [_vp, C.c_char_p, C.c_char_p]),
    "dmfted_time_hxv": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32, _dp]),
    "dmfted_hxv_timing": (C.c_int, [_vp, C.c_int32]),
    "dmfted_autotune_log": (C.c_int, [_vp, C.c_char_p, C.c_int32, C.POINTER(C.c_int32)]),
    "dmfted_get_neigen": (C.c_int, [_vp, _ip, C.c_int32, C.POINTER(C.c_int32)]),
    "dmfted_set_neigen": (C.c_int, [_vp, _ip, C.c_int32, C.c_int32]),
    "dmfted_get_hxv_timing": (C.c_int, [_vp, _dp, _lp, _dp]),
    "dmfted_get_timings": (C.c_int, [_vp, _dp, _lp]),
    "dmfted_launch_count": (C.c_int, [_vp, _lp, C.c_int32]),
}


def library_path():
    return _LIB


def lib():
    """Load libdmfted.so (built by dmft-ed_b200/build.py); raise if absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            raise RuntimeError(f"CUDA library not built: {_LIB} (run python dmft-ed_b200/build.py)")
        L = C.CDLL(_LIB)
        for name, (res, args) in EXPORTS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ck(rc):
    if rc != OK:
        raise DmftedError(rc, lib().dmfted_last_error().decode())


def _p(a, ct=C.c_double):
    return a.ctypes.data_as(C.POINTER(ct)) if a is not None else None


def default_params(**kw):
    """Reference defaults (ED_INPUT_VARS.f90:111-176), overridden by keywords."""
    p = Params()
    lib().dmfted_default_params(C.byref(p))
    for k, v in kw.items():
        if k == "uloc":
            vals = list(v) + [0.0] * (3 - len(v))
            for i in range(3):
                p.uloc[i] = float(vals[i])
        else:
            if not hasattr(p, k):
                raise AttributeError(k)
            setattr(p, k, v)
    return p


def get_bath_dimension(params):
    """get_bath_dimension (ED_BATH/user_aux.f90:11-94), normal bath."""
    nb = C.c_int32()
    _ck(lib().dmfted_get_bath_dimension(C.byref(params), C.byref(nb)))
    return nb.value


def save_bath(params, path, bath):
    """save_dmft_bath: the bath array to a hamiltonian.restart-format file."""
    b = np.ascontiguousarray(bath, np.float64)
    _ck(lib().dmfted_save_bath(C.byref(params), os.fsencode(path), _p(b), b.size))


def read_bath(params, path, bath=None):
    """The bath read of init_dmft_bath (min(lines, Nbath) rows after the
    header) into a copy of bath (zeros when bath is None).  Returns the array."""
    nb = get_bath_dimension(params)
    b = np.zeros(nb) if bath is None else np.array(bath, np.float64, copy=True)
    _ck(lib().dmfted_read_bath(C.byref(params), os.fsencode(path), _p(b), nb))
    return b


def _c128(a):
    return np.ascontiguousarray(a, np.complex128)


class EDSolver:
    """One solver context on one GPU: ed_init_solver ... ed_solve ... ed_get_*."""

    def __init__(self, params=None, hloc=None, **kw):
        self.params = params if params is not None else default_params(**kw)
        self.ctx = C.c_void_p()
        h = None
        if hloc is not None:
            h = np.asfortranarray(np.asarray(hloc, np.complex128))
            h = np.ascontiguousarray(h.reshape(-1, order="F")).view(np.float64)
        self._hkeep = h
        _ck(lib().dmfted_init(C.byref(self.params), _p(h), C.byref(self.ctx)))
        p = self.params
        self.ns = (p.nbath + 1) * p.norb
        self.nsectors = (self.ns + 1) ** 2

    # -- lifetime ----------------------------------------------------------
    def close(self):
        if self.ctx:
            _ck(lib().dmfted_free(self.ctx))
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- set-up --------------------------------------------------------------
    def get_bath_dimension(self):
        return get_bath_dimension(self.params)

    def set_hloc(self, hloc):
        h = np.asfortranarray(np.asarray(hloc, np.complex128))
        h = np.ascontiguousarray(h.reshape(-1, order="F")).view(np.float64)
        _ck(lib().dmfted_set_hloc(self.ctx, _p(h)))

    def set_bath(self, bath):
        b = np.ascontiguousarray(bath, np.float64)
        _ck(lib().dmfted_set_bath(self.ctx, _p(b), b.size))

    def sector_tables(self):
        ns, nsec = self.ns, self.nsectors
        t = {k: np.zeros(n, np.int32) for k, n in [
            ("getsector", (ns + 1) ** 2), ("getnup", nsec), ("getndw", nsec), ("getdim", nsec),
            ("getdimup", nsec), ("getdimdw", nsec), ("getcsector", 2 * nsec),
            ("getcdgsector", 2 * nsec), ("getbathstride", self.params.norb * self.params.nbath),
            ("impindex", 2 * self.params.norb)]}
        n = C.c_int32()
        _ck(lib().dmfted_sector_tables(self.ctx, C.byref(n), *[_p(t[k], C.c_int32) for k in [
            "getsector", "getnup", "getndw", "getdim", "getdimup", "getdimdw", "getcsector",
            "getcdgsector", "getbathstride", "impindex"]]))
        return t

    def sector_index(self, nup, ndw):
        """getSector(nup, ndw), 1-based (ED_SETUP.f90:388-390)."""
        return nup * (self.ns + 1) + ndw + 1

    def sector_dim(self, isector):
        nup, ndw = divmod(isector - 1, self.ns + 1)
        from math import comb
        return comb(self.ns, nup) * comb(self.ns, ndw)

    def build_sector(self, isector):
        dim = self.sector_dim(isector)
        m = np.zeros(dim, np.int32)
        _ck(lib().dmfted_build_sector(self.ctx, isector, _p(m, C.c_int32), dim))
        return m

    # -- H*v -------------------------------------------------------------------
    def setup_hv_sector(self, isector):
        _ck(lib().dmfted_setup_hv_sector(self.ctx, isector))

    def delete_hv_sector(self):
        _ck(lib().dmfted_delete_hv_sector(self.ctx))

    def hxv(self, v):
        """spHtimesV_cc(Nloc, v, Hv) on the current sector (complex128, host)."""
        v = _c128(v)
        hv = np.empty_like(v)
        _ck(lib().dmfted_hxv_c128(self.ctx, v.size, _p(v.view(np.float64)), _p(hv.view(np.float64))))
        return hv

    def time_hxv(self, fp32=False, warmup=3, reps=10, fused=False, chain_order=False,
                 whole_step=False):
        ms = C.c_double()
        flags = (int(fp32) | (2 if fused else 0) | (4 if chain_order else 0)
                 | (8 if whole_step else 0))
        _ck(lib().dmfted_time_hxv(self.ctx, flags, warmup, reps, C.byref(ms)))
        return ms.value

    # -- solvers -------------------------------------------------------------------
    def lanczos_gs(self, isector, want_vector=True):
        e0 = C.c_double()
        nit = C.c_int32()
        psi = np.zeros(self.sector_dim(isector), np.complex128) if want_vector else None
        _ck(lib().dmfted_lanczos_gs(self.ctx, isector, C.byref(e0),
                                    _p(psi.view(np.float64)) if want_vector else None,
                                    C.byref(nit)))
        return e0.value, psi, nit.value

    def gs_lanczos(self, isector, neigen, nitermax=0, tol=0.0, want_vectors=True):
        """sp_eigh / eigh of one sector as ed_diag_c calls them
        (ED_DIAG.f90:133-194): the lowest neigen eigenpairs, degenerate copies
        included.  Returns (evals, vecs[n, dim] complex or None)."""
        dim = self.sector_dim(isector)
        ne = min(neigen, dim)
        ev = np.zeros(ne)
        vec = np.zeros(2 * ne * dim) if want_vectors else None
        nf = C.c_int32()
        _ck(lib().dmfted_gs_lanczos(self.ctx, isector, neigen, nitermax, tol, _p(ev),
                                    _p(vec) if want_vectors else None, C.byref(nf)))
        n = nf.value
        if not want_vectors:
            return ev[:n], None
        v = vec.view(np.complex128).reshape(ne, dim)[:n]
        return ev[:n], v

    def lanc_tridiag(self, isector, vvinit, nlanc):
        """sp_lanc_tridiag(spHtimesV_cc, vvinit, alfa, beta) on sector isector."""
        v = _c128(vvinit)
        a = np.zeros(nlanc)
        b = np.zeros(nlanc)
        used = C.c_int32()
        _ck(lib().dmfted_lanc_tridiag(self.ctx, isector, _p(v.view(np.float64)), nlanc, _p(a),
                                      _p(b), C.byref(used)))
        return a, b, used.value

    def add_to_lanczos_gf(self, vnorm2, ei, egs, zeta, alanc, blanc, isign, lmats, lreal):
        """add_to_lanczos_gf_normal (build_gf_normal.f90:442-488) for one chain on
        the context's frequency grids; returns (gmats[lmats], greal[lreal])."""
        a = np.ascontiguousarray(alanc, np.float64)
        b = np.ascontiguousarray(blanc, np.float64)
        gm = np.zeros(2 * max(lmats, 1))
        gr = np.zeros(2 * max(lreal, 1))
        _ck(lib().dmfted_add_to_lanczos_gf(self.ctx, vnorm2, ei, egs, zeta, a.size, _p(a), _p(b),
                                           isign, _p(gm), _p(gr) if lreal > 0 else None))
        return gm.view(np.complex128)[:lmats], gr.view(np.complex128)[:lreal]

    def ed_solve(self, bath, sectors=None):
        """ed_solve_single (ED_MAIN.f90:251-289); sectors restricts the scan."""
        b = np.ascontiguousarray(bath, np.float64)
        s = None if sectors is None else np.ascontiguousarray(sectors, np.int32)
        _ck(lib().dmfted_ed_solve(self.ctx, _p(b), b.size, _p(s, C.c_int32),
                                  0 if s is None else s.size))

    # -- getters (ED_IO.f90:371-394) -----------------------------------------------
    def _gf(self, fn, L):
        p = self.params
        out = np.zeros((p.nspin, p.nspin, p.norb, p.norb, L), np.complex128, order="F")
        flat = np.zeros(out.size, np.complex128)
        _ck(fn(self.ctx, _p(flat.view(np.float64))))
        return flat.reshape(out.shape, order="F")

    def ed_get_gimp_matsubara(self):
        return self._gf(lib().dmfted_get_gimp_matsubara, self.params.lmats)

    def ed_get_gimp_real(self):
        return self._gf(lib().dmfted_get_gimp_real, self.params.lreal)

    def ed_get_sigma_matsubara(self):
        return self._gf(lib().dmfted_get_sigma_matsubara, self.params.lmats)

    def ed_get_sigma_real(self):
        return self._gf(lib().dmfted_get_sigma_real, self.params.lreal)

    def ed_get_g0imp_matsubara(self):
        return self._gf(lib().dmfted_get_g0imp_matsubara, self.params.lmats)

    def ed_get_g0imp_real(self):
        return self._gf(lib().dmfted_get_g0imp_real, self.params.lreal)

    def observables(self):
        no = self.params.norb
        arrs = [np.zeros(no) for _ in range(5)]
        _ck(lib().dmfted_get_observables(self.ctx, *[_p(a) for a in arrs]))
        return dict(zip(["dens", "dens_up", "dens_dw", "docc", "magz"], arrs))

    def ed_get_dens(self):
        return self.observables()["dens"]

    def ed_get_docc(self):
        return self.observables()["docc"]

    def ed_get_mag(self):
        return self.observables()["magz"]

    def get_neigen(self):
        """neigen_sector(:) and lanc_nstates_total as the next solve will use them."""
        arr = np.zeros(self.nsectors, np.int32)
        tot = C.c_int32()
        _ck(lib().dmfted_get_neigen(self.ctx, _p(arr, C.c_int32), arr.size, C.byref(tot)))
        return arr, tot.value

    def set_neigen(self, neigen, nstates_total):
        arr = np.ascontiguousarray(neigen, np.int32)
        _ck(lib().dmfted_set_neigen(self.ctx, _p(arr, C.c_int32), arr.size, int(nstates_total)))

    def eigenspace(self, cap=4096):
        e = np.zeros(cap)
        s = np.zeros(cap, np.int32)
        n = C.c_int32()
        z = C.c_double()
        _ck(lib().dmfted_get_eigenspace(self.ctx, cap, _p(e), _p(s, C.c_int32), C.byref(n),
                                        C.byref(z)))
        return e[:n.value], s[:n.value], z.value

    def ed_get_eimp(self):
        """[Epot, Eint, Ehartree, Eknot] (ed_get_eimp, ED_IO/get_eimp.f90:1-4)."""
        out = np.zeros(4)
        _ck(lib().dmfted_get_eimp(self.ctx, _p(out)))
        return out

    def ed_get_doubles(self):
        """[Dust, Dund, Dse, Dph] (ed_get_doubles, ED_IO/get_doubles.f90:1-4)."""
        out = np.zeros(4)
        _ck(lib().dmfted_get_doubles(self.ctx, _p(out)))
        return out

    def egs(self):
        e = C.c_double()
        _ck(lib().dmfted_get_egs(self.ctx, C.byref(e)))
        return e.value

    def hf_gradient(self):
        nb = self.get_bath_dimension()
        g = np.zeros(nb)
        _ck(lib().dmfted_hf_gradient(self.ctx, _p(g), nb))
        return g

    def chi2_delta_batch(self, a, xdelta, g, w, grad=True):
        """chi2_delta_normal_normal / grad_chi2_delta_normal_normal for a batch."""
        a = np.ascontiguousarray(np.atleast_2d(a), np.float64)
        nbatch, n2 = a.shape
        xdelta = np.ascontiguousarray(xdelta, np.float64)
        g = _c128(g)
        w = np.ascontiguousarray(w, np.float64)
        chi2 = np.zeros(nbatch)
        gr = np.zeros((nbatch, n2)) if grad else None
        _ck(lib().dmfted_chi2_delta_batch(self.ctx, nbatch, n2 // 2, xdelta.size, _p(a),
                                          _p(xdelta), _p(g.view(np.float64)), _p(w), _p(chi2),
                                          _p(gr)))
        return (chi2, gr) if grad else chi2

    # ---- restart files ----------------------------------------------------
    def print_state_list(self, path):
        """print_state_list: the last solve's eigenspace in state_list.ed format."""
        _ck(lib().dmfted_print_state_list(self.ctx, os.fsencode(path)))

    def read_state_list(self, path):
        """state_list.restart: the per-sector state counts for the next solve."""
        _ck(lib().dmfted_read_state_list(self.ctx, os.fsencode(path)))

    # ---- printed outputs (ED_IO, ED_OBSERVABLES) ---------------------------
    def print_impG(self, dir="", suffix=""):
        """print_impG_normal: impG_l<a><a>_s<s>_iw/_realw<suffix>.ed in dir."""
        _ck(lib().dmfted_print_impg(self.ctx, os.fsencode(dir), suffix.encode()))

    def print_impSigma(self, dir="", suffix=""):
        """print_impSigma_normal: impSigma_l<a><a>_s<s>_iw/_realw<suffix>.ed."""
        _ck(lib().dmfted_print_impsigma(self.ctx, os.fsencode(dir), suffix.encode()))

    def print_impG0(self, dir="", suffix=""):
        """print_impG0_normal: the Weiss field under the impG_... names."""
        _ck(lib().dmfted_print_impg0(self.ctx, os.fsencode(dir), suffix.encode()))

    def read_impSigma(self, dir="", suffix=""):
        """read_impSigma_normal: the impSigma files back into the context."""
        _ck(lib().dmfted_read_impsigma(self.ctx, os.fsencode(dir), suffix.encode()))

    def write_observables(self, dir="", suffix="", legend=False):
        """write_observables (and write_legend when legend): observables_all
        (appended), observables_last, parameters_last<suffix>.ed."""
        _ck(lib().dmfted_write_observables(self.ctx, os.fsencode(dir), suffix.encode(),
                                           1 if legend else 0))

    def write_energy(self, dir="", suffix=""):
        """write_energy_info and write_energy: energy_info.ed, energy_last<suffix>.ed."""
        _ck(lib().dmfted_write_energy(self.ctx, os.fsencode(dir), suffix.encode()))

    # ---- the self-consistency around the solve ----------------------------
    def ed_chi2_fitgf(self, fg, bath, ispin=1):
        """ed_chi2_fitgf (ED_CHI2FIT.f90:86-138), normal bath: the conjugate-gradient
        fit of every orbital's levels and hybridisations of spin ispin to
        fg(ispin,ispin,a,a,:), on the device.  Returns (new bath, iterations[Norb],
        chi2[Norb]); the input bath array is not modified."""
        p = self.params
        fg = np.asarray(fg, np.complex128)
        assert fg.shape[:4] == (p.nspin, p.nspin, p.norb, p.norb), fg.shape
        flat = np.ascontiguousarray(fg.reshape(-1, order="F"))
        b = np.array(bath, np.float64, copy=True)
        it = np.zeros(p.norb, np.int32)
        c2 = np.zeros(p.norb)
        _ck(lib().dmfted_chi2_fitgf(self.ctx, _p(flat.view(np.float64)), int(ispin), _p(b), b.size,
                                    _p(it, C.c_int32), _p(c2)))
        return b, it, c2

    def cg_fit_batch(self, a, xdelta, g, w, scheme=None, zc=0.0):
        """The bath-fit minimiser on a batch of start points (one CTA each), all
        fitting the target g.  Returns (minima, chi2, iterations)."""
        a = np.array(np.atleast_2d(a), np.float64, copy=True, order="C")
        nbatch, n2 = a.shape
        xdelta = np.ascontiguousarray(xdelta, np.float64)
        g = _c128(g)
        w = np.ascontiguousarray(w, np.float64)
        sch = self.params.cg_scheme if scheme is None else scheme
        it = np.zeros(nbatch, np.int32)
        c2 = np.zeros(nbatch)
        _ck(lib().dmfted_cg_fit_batch(self.ctx, nbatch, n2 // 2, xdelta.size, _p(a), _p(xdelta),
                                      _p(g.view(np.float64)), _p(w), int(sch), float(zc),
                                      _p(it, C.c_int32), _p(c2)))
        return a, c2, it

    def _gloc(self, fn, L, he, wt, sigma):
        p = self.params
        wt = np.ascontiguousarray(wt, np.float64)
        he = np.ascontiguousarray(np.broadcast_to(np.asarray(he, np.float64), (p.norb, wt.size)))
        sig = np.ascontiguousarray(np.asarray(sigma, np.complex128).reshape(-1, order="F"))
        out = np.zeros(sig.size, np.complex128)
        _ck(fn(self.ctx, wt.size, _p(he), _p(wt), _p(sig.view(np.float64)),
               _p(out.view(np.float64))))
        return out.reshape((p.nspin, p.nspin, p.norb, p.norb, L), order="F")

    def gloc_matsubara_diag(self, he, wt, sigma):
        """dmft_gloc_matsubara for a lattice Hamiltonian diagonal in spin and
        orbital: he[Norb, Le] (or [Le] for every orbital), wt[Le], sigma as
        ed_get_sigma_matsubara returns it."""
        return self._gloc(lib().dmfted_gloc_matsubara_diag, self.params.lmats, he, wt, sigma)

    def gloc_realaxis_diag(self, he, wt, sigma):
        """dmft_gloc_realaxis on the same grid (w + i eps, the context's Lreal)."""
        return self._gloc(lib().dmfted_gloc_realaxis_diag, self.params.lreal, he, wt, sigma)

    def get_weiss(self, gloc, sigma, scheme=None):
        """dmft_weiss (scheme CG_WEISS) or dmft_delta (CG_DELTA) on the diagonal."""
        p = self.params
        sch = p.cg_scheme if scheme is None else scheme
        gl = np.ascontiguousarray(np.asarray(gloc, np.complex128).reshape(-1, order="F"))
        sig = np.ascontiguousarray(np.asarray(sigma, np.complex128).reshape(-1, order="F"))
        out = np.zeros(gl.size, np.complex128)
        _ck(lib().dmfted_get_weiss(self.ctx, _p(gl.view(np.float64)), _p(sig.view(np.float64)),
                                   int(sch), _p(out.view(np.float64))))
        return out.reshape((p.nspin, p.nspin, p.norb, p.norb, p.lmats), order="F")

    def timings(self):
        t = np.zeros(4)
        n = np.zeros(3, np.int64)
        _ck(lib().dmfted_get_timings(self.ctx, _p(t), _p(n, C.c_int64)))
        return dict(diag_ms=t[0], obs_ms=t[1], gf_ms=t[2], total_ms=t[3], hv_diag=int(n[0]),
                    hv_obs=int(n[1]), hv_gf=int(n[2]))

    def hxv_timing(self, on=True):
        """Record device time and algorithmic bytes of every H*v launch."""
        _ck(lib().dmfted_hxv_timing(self.ctx, int(on)))

    def hxv_timing_totals(self):
        ms, n, b = C.c_double(), C.c_int64(), C.c_double()
        _ck(lib().dmfted_get_hxv_timing(self.ctx, C.byref(ms), C.byref(n), C.byref(b)))
        return dict(ms=ms.value, launches=n.value, bytes=b.value)

    def autotune_log(self):
        """Lines of the autotuner: job-shape key, time per cluster size, choice."""
        need = C.c_int32()
        _ck(lib().dmfted_autotune_log(self.ctx, None, 0, C.byref(need)))
        buf = C.create_string_buffer(need.value)
        _ck(lib().dmfted_autotune_log(self.ctx, buf, need.value, None))
        return [l for l in buf.value.decode().split("\n") if l]

    def launch_count(self, reset=False):
        n = C.c_int64()
        _ck(lib().dmfted_launch_count(self.ctx, C.byref(n), int(reset)))
        return n.value


def ed_init_solver(bath=None, hloc=None, **kw):
    """ed_init_solver (ED_MAIN.f90:67-107): returns the solver context."""
    return EDSolver(hloc=hloc, **kw)
