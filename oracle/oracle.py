"""Python front-end of the CPU restatement in ``oracle/ed_oracle.c``.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA library.  Only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` import this module; the product never does.

Parity status: unpinned against reference outputs (the reference is Fortran
with unvendored SciFortran/DMFT_Tools and ships no tests or golden data).  The
restatement is pinned instead against independent known answers: dense
``numpy.linalg.eigh`` of the explicit sector Hamiltonian, ARPACK
(``scipy.sparse.linalg.eigsh``, the eigensolver family behind SciFortran's
``sp_eigh``), the U=0 and V=0 analytic limits and the particle+hole sum rule.

Each wrapper names the reference routine it restates (file:line relative to
the reference project root).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libedoracle.so")
_lib = None


def build():
    """Compile ed_oracle.c with the committed Makefile (no-op when current)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


class _Model(C.Structure):
    _fields_ = [
        ("norb", C.c_int32), ("nbath", C.c_int32), ("nspin", C.c_int32), ("ns", C.c_int32),
        ("hfmode", C.c_int32), ("jhflag", C.c_int32),
        ("uloc", C.c_double * 3),
        ("ust", C.c_double), ("jh", C.c_double), ("jx", C.c_double), ("jp", C.c_double),
        ("xmu", C.c_double), ("beta", C.c_double),
        ("e", C.POINTER(C.c_double)), ("v", C.POINTER(C.c_double)),
        ("hloc", C.POINTER(C.c_double)),
    ]


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)


def _declare(L):
    L.or_binomial.restype = C.c_int32
    L.or_binomial.argtypes = [C.c_int32, C.c_int32]
    L.or_sector_dim.restype = C.c_int64
    L.or_sector_dim.argtypes = [C.c_int32, C.c_int32, C.c_int32]
    L.or_setup_pointers_normal.argtypes = [C.c_int32, C.c_int32] + [_ip] * 10
    L.or_build_sector.restype = C.c_int64
    L.or_build_sector.argtypes = [C.c_int32, C.c_int32, C.c_int32, _ip]
    L.or_binary_search.restype = C.c_int64
    L.or_binary_search.argtypes = [_ip, C.c_int64, C.c_int32]
    L.or_c.restype = C.c_int32
    L.or_c.argtypes = [C.c_int32, C.c_int32, _ip, _dp]
    L.or_cdg.restype = C.c_int32
    L.or_cdg.argtypes = [C.c_int32, C.c_int32, _ip, _dp]
    L.or_hxv_c128.argtypes = [C.POINTER(_Model), _ip, C.c_int64, _dp, _dp, C.c_int32]
    L.or_build_coo.restype = C.c_int64
    L.or_build_coo.argtypes = [C.POINTER(_Model), _ip, C.c_int64, C.c_int64, _lp, _lp, _dp, _dp]
    L.or_lanczos_tridiag.restype = C.c_int32
    L.or_lanczos_tridiag.argtypes = [C.POINTER(_Model), _ip, C.c_int64, _dp, C.c_int32, _dp, _dp,
                                     C.c_double, C.c_int32]
    L.or_tql2.restype = C.c_int32
    L.or_tql2.argtypes = [C.c_int32, _dp, _dp, _dp]
    L.or_lanczos_gs.restype = C.c_int32
    L.or_lanczos_gs.argtypes = [C.POINTER(_Model), _ip, C.c_int64, _dp, C.c_int32, C.c_double,
                                C.c_int32, _dp, C.c_int32]
    L.or_add_to_lanczos_gf.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int32,
                                       C.c_double, _dp, _dp, C.c_int32, C.c_int32, _dp, C.c_int32,
                                       _dp, C.c_int32, C.c_double, _dp, _dp]
    L.or_gf_vvinit.restype = C.c_double
    L.or_gf_vvinit.argtypes = [C.c_int32, C.c_int32, _ip, C.c_int64, _ip, C.c_int64, _dp, _dp]
    L.or_observables_state.argtypes = [C.POINTER(_Model), _ip, C.c_int64, _dp, C.c_double,
                                       _dp, _dp, _dp, _dp, _dp, _dp]
    L.or_hf_terms_state.argtypes = [C.POINTER(_Model), _ip, C.c_int64, _dp, C.c_double, _dp, _dp]
    L.or_local_energy_state.argtypes = [C.POINTER(_Model), _ip, C.c_int64, _dp, C.c_double, _dp]
    L.or_delta_bath.argtypes = [_dp, _dp, C.c_int32, _dp, C.c_int32, _dp]
    L.or_sigma_normal.argtypes = [_dp, _dp, C.c_int32, C.c_double, C.c_double, _dp, C.c_int32,
                                  _dp, _dp]
    L.or_chi2_delta.restype = C.c_double
    L.or_chi2_delta.argtypes = [_dp, C.c_int32, _dp, _dp, _dp, C.c_int32, _dp]
    L.or_host_threads.restype = C.c_int32
    L.or_factored_setup.restype = C.c_void_p
    L.or_factored_setup.argtypes = [C.POINTER(_Model), _ip, C.c_int64, C.c_int64, C.c_int32]
    L.or_factored_free.argtypes = [C.c_void_p]
    L.or_factored_hxv.argtypes = [C.c_void_p, _dp, _dp, C.c_int32]
    L.or_chi2_model.restype = C.c_double
    L.or_chi2_model.argtypes = [_dp, C.c_int32, _dp, _dp, _dp, C.c_int32, C.c_int32, C.c_double,
                                _dp]
    L.or_cg_fit.restype = C.c_double
    L.or_cg_fit.argtypes = [_dp, C.c_int32, _dp, _dp, _dp, C.c_int32, C.c_int32, C.c_double,
                            C.c_int32, C.c_double, C.c_double, C.c_int32, _ip, _ip]


def _p(a, ct=C.c_double):
    return a.ctypes.data_as(C.POINTER(ct))


# --------------------------------------------------------------------------
@dataclass
class Model:
    """Normal-mode, normal-bath impurity model (the reference's global input
    variables of ED_INPUT_VARS.f90 plus dmft_bath and impHloc)."""
    norb: int = 1
    nbath: int = 7
    nspin: int = 1
    uloc: tuple = (2.0, 0.0, 0.0)
    ust: float = 0.0
    jh: float = 0.0
    jx: float = 0.0
    jp: float = 0.0
    xmu: float = 0.0
    beta: float = 100.0
    hfmode: bool = True
    jhflag: bool = False
    e: np.ndarray = field(default=None)      # [nspin, norb, nbath]
    v: np.ndarray = field(default=None)      # [nspin, norb, nbath]
    hloc: np.ndarray = field(default=None)   # complex [nspin, nspin, norb, norb]

    @property
    def ns(self):
        return (self.nbath + 1) * self.norb

    def __post_init__(self):
        if self.e is None:
            self.e = np.zeros((self.nspin, self.norb, self.nbath))
        if self.v is None:
            self.v = np.zeros((self.nspin, self.norb, self.nbath))
        if self.hloc is None:
            self.hloc = np.zeros((self.nspin, self.nspin, self.norb, self.norb), complex)
        self.e = np.ascontiguousarray(self.e, dtype=np.float64)
        self.v = np.ascontiguousarray(self.v, dtype=np.float64)
        self.hloc = np.asarray(self.hloc, dtype=np.complex128)

    def bath_array(self):
        """User bath array, set_dmft_bath layout (ED_BATH/dmft_aux.f90:493-512):
        e then v, each with k fastest, then iorb, then ispin."""
        return np.concatenate([self.e.reshape(-1), self.v.reshape(-1)])

    def _struct(self):
        hl = np.asfortranarray(self.hloc).reshape(-1, order="F")
        hl = np.ascontiguousarray(np.stack([hl.real, hl.imag], axis=-1).reshape(-1))
        self._keep = (self.e, self.v, hl)
        m = _Model()
        m.norb, m.nbath, m.nspin, m.ns = self.norb, self.nbath, self.nspin, self.ns
        m.hfmode, m.jhflag = int(self.hfmode), int(self.jhflag)
        for i in range(3):
            m.uloc[i] = float(self.uloc[i]) if i < len(self.uloc) else 0.0
        m.ust, m.jh, m.jx, m.jp, m.xmu, m.beta = self.ust, self.jh, self.jx, self.jp, self.xmu, self.beta
        m.e, m.v, m.hloc = _p(self.e), _p(self.v), _p(hl)
        return m


def seeded_model(seed, norb=1, nbath=7, nspin=1, u=2.0, ust=0.0, jh=0.0, xmu=0.0, beta=100.0,
                 e_range=1.0, v0=0.5, v_spread=0.1, hfmode=True):
    """Seeded synthetic bath: e_k ~ U[-e_range, e_range], V_k = v0 + U[-v_spread, v_spread]
    from numpy.random.default_rng(seed), shared by both spins when nspin=2."""
    rng = np.random.default_rng(seed)
    e = rng.uniform(-e_range, e_range, size=(norb, nbath))
    v = v0 + rng.uniform(-v_spread, v_spread, size=(norb, nbath))
    e = np.broadcast_to(e, (nspin, norb, nbath)).copy()
    v = np.broadcast_to(v, (nspin, norb, nbath)).copy()
    ul = [u] * norb + [0.0] * (3 - norb)
    return Model(norb=norb, nbath=nbath, nspin=nspin, uloc=tuple(ul), ust=ust, jh=jh, xmu=xmu,
                 beta=beta, hfmode=hfmode, e=e, v=v)


# ---------------------------------------------------------------- setup ---
def binomial(n1, n2):
    """ED_SETUP.f90:1258-1275."""
    return lib().or_binomial(n1, n2)


def sector_tables(norb, nbath):
    """setup_pointers_normal, ED_SETUP.f90:379-493 (1-based values)."""
    ns = (nbath + 1) * norb
    nsec = (ns + 1) ** 2
    t = {k: np.zeros(n, np.int32) for k, n in [
        ("getsector", (ns + 1) ** 2), ("getnup", nsec), ("getndw", nsec), ("getdim", nsec),
        ("getdimup", nsec), ("getdimdw", nsec), ("getcsector", 2 * nsec),
        ("getcdgsector", 2 * nsec), ("getbathstride", norb * nbath), ("impindex", 2 * norb)]}
    lib().or_setup_pointers_normal(norb, nbath, *[_p(t[k], C.c_int32) for k in [
        "getsector", "getnup", "getndw", "getdim", "getdimup", "getdimdw", "getcsector",
        "getcdgsector", "getbathstride", "impindex"]])
    return t


def build_sector(ns, nup, ndw):
    """build_sector (normal), ED_SETUP.f90:874-891."""
    dim = lib().or_sector_dim(ns, nup, ndw)
    m = np.zeros(dim, np.int32)
    got = lib().or_build_sector(ns, nup, ndw, _p(m, C.c_int32))
    assert got == dim
    return m


def binary_search(a, value):
    """ED_SETUP.f90:1282-1299 (1-based position, 0 if absent)."""
    a = np.ascontiguousarray(a, np.int32)
    return lib().or_binary_search(_p(a, C.c_int32), a.size, value)


# ----------------------------------------------------------------- H*v ----
def hxv(model, hmap, v, nthreads=1):
    """directMatVec_cc, ED_HAMILTONIAN_MATVEC.f90:289-351 (complex128)."""
    v = np.ascontiguousarray(v, np.complex128)
    out = np.empty_like(v)
    ms = model._struct()
    lib().or_hxv_c128(C.byref(ms), _p(hmap, C.c_int32), hmap.size, _p(v.view(np.float64)),
                      _p(out.view(np.float64)), nthreads)
    return out


class FactoredHxv:
    """The up/down-factored FP64 H*v on the CPU (oracle/ed_oracle.c,
    or_factored_*): the device's algorithm restated as the "best CPU" variant
    of the baseline.  Not the reference's algorithm; real models without the
    Jhflag terms only."""

    def __init__(self, model, nup, ndw, nthreads=1):
        self.hmap = build_sector(model.ns, nup, ndw)
        self.dimup = binomial(model.ns, nup)
        self.dimdw = binomial(model.ns, ndw)
        self._ms = model._struct()
        self.nthreads = nthreads
        self.h = lib().or_factored_setup(C.byref(self._ms), _p(self.hmap, C.c_int32), self.dimup,
                                         self.dimdw, nthreads)
        if not self.h:
            raise ValueError("model not factored (Jhflag terms or too many bath levels)")

    def __call__(self, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty_like(x)
        lib().or_factored_hxv(self.h, _p(x), _p(y), self.nthreads)
        return y

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_factored_free(self.h)
            self.h = None


def sparse_h(model, hmap):
    """Explicit sector H (the element set of ed_buildH_c) as a scipy CSR matrix
    with H[i, j] = coefficient that row i applies to v[j]."""
    import scipy.sparse as sp
    dim = hmap.size
    cap = dim * (4 + 2 * model.norb * model.norb + 4 * model.norb * model.nbath + 4 * model.norb ** 2)
    ri = np.zeros(cap, np.int64)
    ci = np.zeros(cap, np.int64)
    re = np.zeros(cap)
    im = np.zeros(cap)
    ms = model._struct()
    n = lib().or_build_coo(C.byref(ms), _p(hmap, C.c_int32), dim, cap, _p(ri, C.c_int64),
                           _p(ci, C.c_int64), _p(re), _p(im))
    assert n < cap
    vals = re[:n] + 1j * im[:n]
    if not np.any(vals.imag):
        vals = vals.real
    return sp.csr_matrix((vals, (ri[:n], ci[:n])), shape=(dim, dim))


# ------------------------------------------------------------- Lanczos ---
def lanczos_tridiag(model, hmap, vin, nitermax, threshold=1e-13, nthreads=1):
    """sp_lanc_tridiag restated from .repo/PLAIN_LANCZOS.f90:87-118,154-180."""
    v = np.ascontiguousarray(vin, np.complex128).copy()
    a = np.zeros(nitermax)
    b = np.zeros(nitermax)
    ms = model._struct()
    n = lib().or_lanczos_tridiag(C.byref(ms), _p(hmap, C.c_int32), hmap.size, _p(v.view(np.float64)),
                                 nitermax, _p(a), _p(b), threshold, nthreads)
    return a, b, n


def tql2(d, e, z=None):
    """ED_GREENS_FUNCTIONS.f90:361-499.  e[1:] is the sub-diagonal."""
    d = np.ascontiguousarray(d, np.float64).copy()
    e = np.ascontiguousarray(e, np.float64).copy()
    n = d.size
    if z is None:
        z = np.eye(n)
    z = np.asfortranarray(z, np.float64).copy(order="F")
    zf = z.reshape(-1, order="F").copy()
    ierr = lib().or_tql2(n, _p(d), _p(e), _p(zf))
    return d, zf.reshape((n, n), order="F"), ierr


def start_vector(dim, seed=1234567):
    """Deterministic complex start vector (the reference seeds ARPACK's resid
    with random numbers from seed 1234567, .repo/ARPACK_LANCZOS.f90:394-403)."""
    rng = np.random.default_rng(seed)
    v = rng.random(dim) + 1j * rng.random(dim)
    return v / np.linalg.norm(v)


def lanczos_gs(model, hmap, nitermax=512, threshold=1e-12, ncheck=10, v0=None, nthreads=1):
    """Ground state by plain Lanczos, .repo/PLAIN_LANCZOS.f90:286-385."""
    v = start_vector(hmap.size) if v0 is None else np.asarray(v0, np.complex128).copy()
    v = np.ascontiguousarray(v)
    e = C.c_double()
    ms = model._struct()
    n = lib().or_lanczos_gs(C.byref(ms), _p(hmap, C.c_int32), hmap.size, _p(v.view(np.float64)),
                            min(nitermax, hmap.size), threshold, ncheck, C.byref(e), nthreads)
    return e.value, v, n


# ------------------------------------------------------------------- GF ---
def matsubara(beta, L):
    """wm = pi/beta*(2n-1), ED_GREENS_FUNCTIONS.f90:114."""
    return np.pi / beta * (2.0 * np.arange(1, L + 1) - 1.0)


def realaxis(wini, wfin, L):
    return np.linspace(wini, wfin, L) if L > 0 else np.zeros(0)


def gf_vvinit(particle, isite, map_i, map_j, psi):
    """vvinit of lanc_build_gf_normal_c, build_gf_normal.f90:97-116,136-155."""
    psi = np.ascontiguousarray(psi, np.complex128)
    vv = np.zeros(map_j.size, np.complex128)
    n2 = lib().or_gf_vvinit(int(particle), isite, _p(map_i, C.c_int32), map_i.size,
                            _p(map_j, C.c_int32), map_j.size, _p(psi.view(np.float64)),
                            _p(vv.view(np.float64)))
    return n2, vv


def add_to_lanczos_gf(vnorm2, ei, egs, zeta, finite_t, beta, alanc, blanc, isign, wm, wr, eps,
                      gm, gr):
    """add_to_lanczos_gf_normal, build_gf_normal.f90:442-488 (accumulates)."""
    alanc = np.ascontiguousarray(alanc, np.float64)
    blanc = np.ascontiguousarray(blanc, np.float64)
    wm = np.ascontiguousarray(wm, np.float64)
    wr = np.ascontiguousarray(wr, np.float64)
    lib().or_add_to_lanczos_gf(vnorm2, ei, egs, zeta, int(finite_t), beta, _p(alanc), _p(blanc),
                               alanc.size, isign, _p(wm), wm.size, _p(wr), wr.size, eps,
                               _p(gm.view(np.float64)), _p(gr.view(np.float64)))


def observables_state(model, hmap, psi, peso):
    """observables_impurity n/docc loop and diagonal bath DM,
    ED_OBSERVABLES.f90:113-160,286-305."""
    no, nb = model.norb, model.nbath
    out = {k: np.zeros(no) for k in ["dens", "dens_up", "dens_dw", "docc", "magz"]}
    out["bath_dm"] = np.zeros(model.nspin * no * nb)
    psi = np.ascontiguousarray(psi, np.complex128)
    ms = model._struct()
    lib().or_observables_state(C.byref(ms), _p(hmap, C.c_int32), hmap.size, _p(psi.view(np.float64)),
                               peso, *[_p(out[k]) for k in ["dens", "dens_up", "dens_dw", "docc",
                                                             "magz", "bath_dm"]])
    return out


def local_energy_state(model, hmap, psi, peso, acc=None):
    """local_energy_impurity's body for one state, ED_OBSERVABLES.f90:454-633:
    adds into acc[8] = [Eknot, Epot without Ehartree, Ehartree, Dust, Dund,
    Dse, Dph, 0]."""
    acc = np.zeros(8) if acc is None else acc
    psi = np.ascontiguousarray(psi, np.complex128)
    ms = model._struct()
    lib().or_local_energy_state(C.byref(ms), _p(hmap, C.c_int32), hmap.size,
                                _p(psi.view(np.float64)), peso, _p(acc))
    return acc


def local_energies(acc):
    """The reference's module variables after local_energy_impurity
    (ED_OBSERVABLES.f90:635): Epot includes Ehartree; ed_Eint is never
    assigned there and stays 0.  Returns eimp = [Epot, Eint, Ehartree, Eknot]
    (ed_get_eimp_, ED_IO/get_eimp.f90:1-4) and doubles = [Dust, Dund, Dse,
    Dph] (ed_get_doubles_, ED_IO/get_doubles.f90:1-4)."""
    eimp = np.array([acc[1] + acc[2], 0.0, acc[2], acc[0]])
    doubles = np.array([acc[3], acc[4], acc[5], acc[6]])
    return eimp, doubles


def hf_terms_state(model, hmap, psi, peso=1.0):
    """<c+_a c_k + h.c.> and <n_k> per physical spin (Hellmann-Feynman operators)."""
    no, nb = model.norb, model.nbath
    hop = np.zeros(2 * no * nb)
    nk = np.zeros(2 * no * nb)
    psi = np.ascontiguousarray(psi, np.complex128)
    ms = model._struct()
    lib().or_hf_terms_state(C.byref(ms), _p(hmap, C.c_int32), hmap.size, _p(psi.view(np.float64)),
                            peso, _p(hop), _p(nk))
    return hop.reshape(2, no, nb), nk.reshape(2, no, nb)


def delta_bath(e_k, v_k, x):
    """delta_bath_mats (normal), ED_BATH_FUNCTIONS.f90:247-257."""
    x = np.ascontiguousarray(x, np.complex128)
    d = np.zeros_like(x)
    e_k = np.ascontiguousarray(e_k, np.float64)
    v_k = np.ascontiguousarray(v_k, np.float64)
    lib().or_delta_bath(_p(e_k), _p(v_k), e_k.size, _p(x.view(np.float64)), x.size,
                        _p(d.view(np.float64)))
    return d


def sigma_normal(e_k, v_k, xmu, hloc_aa, x, g):
    """get_sigma_normal.f90:17-39 with invg0_bath (ED_BATH_FUNCTIONS.f90:1800-1806)."""
    x = np.ascontiguousarray(x, np.complex128)
    g = np.ascontiguousarray(g, np.complex128)
    s = np.zeros_like(x)
    e_k = np.ascontiguousarray(e_k, np.float64)
    v_k = np.ascontiguousarray(v_k, np.float64)
    lib().or_sigma_normal(_p(e_k), _p(v_k), e_k.size, xmu, hloc_aa, _p(x.view(np.float64)), x.size,
                          _p(g.view(np.float64)), _p(s.view(np.float64)))
    return s


def chi2_delta(a, xdelta, g, w, grad=True):
    """chi2_delta_normal_normal / grad_chi2_delta_normal_normal,
    ED_CHI2FIT/fitgf_normal_normal.f90:193-226,256-316."""
    a = np.ascontiguousarray(a, np.float64)
    xdelta = np.ascontiguousarray(xdelta, np.float64)
    g = np.ascontiguousarray(g, np.complex128)
    w = np.ascontiguousarray(w, np.float64)
    gr = np.zeros(a.size) if grad else None
    c2 = lib().or_chi2_delta(_p(a), a.size // 2, _p(xdelta), _p(g.view(np.float64)), _p(w),
                             xdelta.size, _p(gr) if grad else None)
    return (c2, gr) if grad else c2


def chi2_model(a, xdelta, g, w, weiss=False, zc=0.0, grad=True):
    """chi2 of the delta (chi2_delta_normal_normal) or weiss
    (chi2_weiss_normal_normal with g0and_normal_normal) fit and its gradient,
    ED_CHI2FIT/fitgf_normal_normal.f90:193-246,349-362; zc = xmu - Hloc_aa."""
    a = np.ascontiguousarray(a, np.float64)
    xdelta = np.ascontiguousarray(xdelta, np.float64)
    g = np.ascontiguousarray(g, np.complex128)
    w = np.ascontiguousarray(w, np.float64)
    gr = np.zeros(a.size) if grad else None
    c2 = lib().or_chi2_model(_p(a), a.size // 2, _p(xdelta), _p(g.view(np.float64)), _p(w),
                             xdelta.size, int(weiss), float(zc), _p(gr) if grad else None)
    return (c2, gr) if grad else c2


def cg_fit(a, xdelta, g, w, weiss=False, zc=0.0, itmax=500, ftol=1e-5, eps=1e-6, istop=0):
    """fmin_cg as chi2_fitgf_normal_normal calls it (fitgf_normal_normal.f90:82-119),
    restated from the published Polak-Ribiere / Brent algorithm (oracle/ed_oracle.c
    or_cg_fit).  Returns (parameters at the minimum, chi2, iterations, status)."""
    a = np.ascontiguousarray(a, np.float64).copy()
    xdelta = np.ascontiguousarray(xdelta, np.float64)
    g = np.ascontiguousarray(g, np.complex128)
    w = np.ascontiguousarray(w, np.float64)
    it = C.c_int32()
    st = C.c_int32()
    f = lib().or_cg_fit(_p(a), a.size // 2, _p(xdelta), _p(g.view(np.float64)), _p(w),
                        xdelta.size, int(weiss), float(zc), int(itmax), float(ftol), float(eps),
                        int(istop), C.byref(it), C.byref(st))
    return a, f, it.value, st.value


def bethe_dos(le=500, wband=1.0):
    """The Bethe-lattice density-of-states grid of drivers/ed_hm_bethe.f90:38-40:
    He = linspace(-D, D, Le, mesh=de), Wte = dens_bethe(He, D) * de with the
    semicircle dens_bethe(x, D) = 2 sqrt(D^2 - x^2) / (pi D^2) (SciFortran)."""
    he = np.linspace(-wband, wband, le)
    de = he[1] - he[0]
    wt = 2.0 * np.sqrt(np.maximum(wband ** 2 - he ** 2, 0.0)) / (np.pi * wband ** 2) * de
    return he, wt


def gloc_diag(he, wt, wm, xmu, sigma):
    """G_loc(iw_n) = sum_k wt_k / (i w_n + xmu - Sigma(iw_n) - he_k), k in order
    (.repo/ED_GLOC.f90:54-126,257-298 for a 1x1 block; dmft_gloc_matsubara)."""
    z = 1j * np.asarray(wm) + xmu - np.asarray(sigma)
    g = np.zeros_like(z)
    for k in range(len(he)):
        g = g + (1.0 / (z - he[k])) * wt[k]
    return g


def weiss_diag(gloc, sigma, wm, xmu, hloc_aa, weiss=True):
    """dmft_weiss / dmft_delta for a 1x1 block (.repo/ED_WEISS.f90:55-118):
    1/(1/G + Sigma), or i w_n + xmu - Hloc - Sigma - 1/G."""
    ig = 1.0 / np.asarray(gloc)
    if weiss:
        return 1.0 / (ig + sigma)
    return 1j * np.asarray(wm) + xmu - hloc_aa - sigma - ig


# ------------------------------------------------------- restart files ---
def _fortran_es(x, w, d):
    """ESw.d output: d.ddd...E+dd, or d.ddd...+ddd for a three-digit exponent."""
    m, e = f"{x:.{d}E}".split("E")
    ev = int(e)
    s = f"{m}E{'+' if ev >= 0 else '-'}{abs(ev):02d}" if abs(ev) < 100 else \
        f"{m}{'+' if ev >= 0 else '-'}{abs(ev):03d}"
    return s.rjust(w) if len(s) <= w else "*" * w


def write_dmft_bath_text(bath, norb, nspin, nbath):
    """write_dmft_bath, normal bath (ED_BATH/dmft_aux.f90:310-336): the header
    "(90(A21,1X))" and Nbath rows "(90(F21.12,1X))" of ((e, v), orbitals), spins."""
    half = len(bath) // 2
    head = []
    for s in range(nspin):
        for a in range(norb):
            tag = f"l{a + 1}_s{s + 1}"
            head += [f"#Ek_{tag}".rjust(21), f"Vk_{tag}".rjust(21)]
    # the 1X after a record's last item transmits nothing
    rows = [" ".join(head)]
    for k in range(nbath):
        r = []
        for s in range(nspin):
            for a in range(norb):
                io = k + a * nbath + s * nbath * norb
                r += [f"{bath[io]:21.12f}", f"{bath[half + io]:21.12f}"]
        rows.append(" ".join(r))
    return "\n".join(rows) + "\n"


def print_state_list_text(energies, sectors, getnup, getndw, getdim, beta):
    """print_state_list (ED_DIAG.f90:401-445), normal mode: header, then rows
    "(i3,f18.12,2x,ES19.12,1x,2i3,3x,i3,i10)" with exp(-beta (E - E_min))."""
    emin = min(energies)
    out = ["# i       E_i           exp(-(E-E0)/T)       nup ndw  Sect     Dim"]
    for i, (e, isec) in enumerate(zip(energies, sectors)):
        out.append(f"{i + 1:3d}{e:18.12f}  {_fortran_es(np.exp(-beta * (e - emin)), 19, 12)} "
                   f"{getnup[isec - 1]:3d}{getndw[isec - 1]:3d}   {isec:3d}{getdim[isec - 1]:10d}")
    return "\n".join(out) + "\n"


def moments_state(model, hmap, psi, peso):
    """sz2(a,b), n2(a,b) and s2tot of observables_impurity for one state,
    ED_OBSERVABLES.f90:131-160 (impurity orbital a: up bit a, down bit a+Ns)."""
    no, ns = model.norb, model.ns
    m = np.asarray(hmap, np.int64)
    w = peso * np.abs(np.asarray(psi)) ** 2
    nup = np.stack([((m >> a) & 1).astype(np.float64) for a in range(no)])
    ndw = np.stack([((m >> (a + ns)) & 1).astype(np.float64) for a in range(no)])
    sz = (nup - ndw) / 2.0
    nt = nup + ndw
    sz2 = np.array([[np.sum(sz[a] * sz[b] * w) for b in range(no)] for a in range(no)])
    n2 = np.array([[np.sum(nt[a] * nt[b] * w) for b in range(no)] for a in range(no)])
    s2tot = float(np.sum(sz.sum(axis=0) ** 2 * w))
    return sz2, n2, s2tot


def szr(sigma_iw, beta):
    """get_szr (ED_OBSERVABLES.f90:695-708) from Sigma(iw_1), Sigma(iw_2):
    (zimp, simp)."""
    wm1, wm2 = np.pi / beta, 3.0 * np.pi / beta
    s1, s2 = sigma_iw[0].imag, sigma_iw[1].imag
    return 1.0 / (1.0 + abs(s1 / wm1)), s1 - wm1 * (s2 - s1) / (wm2 - wm1)


def observables_legend_text(norb, nspin):
    """write_legend, normal mode (ED_OBSERVABLES.f90:720-731): "(A1,90(A10,6X))"
    labels, the 6X after the last one not transmitted."""
    no, ns = norb, nspin
    lab = []
    lab += [f"{a}dens_{a}" for a in range(1, no + 1)]
    lab += [f"{no + a}docc_{a}" for a in range(1, no + 1)]
    lab += [f"{2 * no + a}nup_{a}" for a in range(1, no + 1)]
    lab += [f"{3 * no + a}ndw_{a}" for a in range(1, no + 1)]
    lab += [f"{4 * no + a}mag_{a}" for a in range(1, no + 1)]
    lab += [f"{5 * no + 1}s2", f"{5 * no + 2}egs"]
    lab += [f"{5 * no + 2 + (a - 1) * no + b}sz2_{a}{b}" for a in range(1, no + 1)
            for b in range(1, no + 1)]
    lab += [f"{(5 + no) * no + 2 + (a - 1) * no + b}n2_{a}{b}" for a in range(1, no + 1)
            for b in range(1, no + 1)]
    lab += [f"{(5 + 2 * no) * no + 2 + (s - 1) * ns + a}z_{a}s{s}" for s in range(1, ns + 1)
            for a in range(1, no + 1)]
    lab += [f"{(6 + 2 * no) * no + 2 + ns + (s - 1) * ns + a}sig_{a}s{s}"
            for s in range(1, ns + 1) for a in range(1, no + 1)]
    return "#" + (" " * 6).join(x.rjust(10)[:10] for x in lab) + "\n"


def f15_9(x):
    """F15.9 (a field too narrow is all '*')."""
    t = f"{x:15.9f}"
    return t if len(t) <= 15 else "*" * 15


def observables_record_text(dens, docc, dens_up, dens_dw, magz, s2tot, egs, sz2, n2, zimp, simp):
    """write_observables, normal mode (ED_OBSERVABLES.f90:786-797): one
    "(90(F15.9,1X))" record; zimp/simp are [spin][orbital]."""
    vals = list(dens) + list(docc) + list(dens_up) + list(dens_dw) + list(magz) + [s2tot, egs]
    vals += list(np.asarray(sz2).reshape(-1)) + list(np.asarray(n2).reshape(-1))
    vals += list(np.asarray(zimp).reshape(-1)) + list(np.asarray(simp).reshape(-1))
    return " ".join(f15_9(v) for v in vals) + "\n"


def energy_texts(eimp, doubles):
    """write_energy_info and write_energy (ED_OBSERVABLES.f90:760-774,851-857)
    from ed_get_eimp = [Epot, Eint, Ehartree, Eknot] and ed_get_doubles =
    [Dust, Dund, Dse, Dph]."""
    names = ["<Hi>", "<V>=<Hi-Ehf>", "<Eloc>", "<Ehf>", "<Dst>", "<Dnd>", "<Dse>", "<Dph>"]
    info = "#" + " ".join(f"{k + 1}{n}".rjust(14)[:14] for k, n in enumerate(names)) + "\n"
    epot, _, ehart, eknot = eimp
    vals = [epot, epot - ehart, eknot, ehart] + list(doubles)
    return info, "".join(f15_9(v) for v in vals) + "\n"


def cg_weights(cg_weight, xdelta):
    """Wdelta of chi2_fitgf_normal_normal, fitgf_normal_normal.f90:44-53."""
    L = xdelta.size
    if cg_weight == 1:
        return np.ones(L)
    if cg_weight == 2:
        return np.arange(1, L + 1, dtype=np.float64)
    if cg_weight == 3:
        return xdelta.copy()
    return np.full(L, float(L))


# ------------------------------------------------------- T=0 pipeline ---
def solve_sector_t0(model, nup, ndw, lmats=4096, lreal=0, wini=-5.0, wfin=5.0, eps=0.01,
                    ngfiter=200, nitermax=512, tol=1e-12, nthreads=1, psi0=None, gs=None):
    """One T=0 impurity solve restricted to sector (nup, ndw): the pipeline of
    ed_solve_single (ED_MAIN.f90:251-289) with diagonalize_impurity
    (ED_DIAG.f90:93-228), observables_impurity (ED_OBSERVABLES.f90:74-160),
    lanc_build_gf_normal_c (build_gf_normal.f90:71-180) and get_sigma_normal.
    Returns a dict with E0, psi, observables, impGmats[ispin, iorb, L], Sigma.
    ``gs=(E0, psi)`` skips the ground-state search (chains from a given state)."""
    ns = model.ns
    hmap = build_sector(ns, nup, ndw)
    if gs is None:
        e0, psi, nl = lanczos_gs(model, hmap, nitermax=nitermax, threshold=tol, v0=psi0,
                                 nthreads=nthreads)
    else:
        e0, psi = gs
        nl = 0
    zeta = 1.0
    obs = observables_state(model, hmap, psi, 1.0 / zeta)
    wm = matsubara(model.beta, lmats)
    wr = realaxis(wini, wfin, lreal)
    no = model.norb
    gm = np.zeros((model.nspin, no, lmats), np.complex128)
    gr = np.zeros((model.nspin, no, lreal), np.complex128)
    chains = []
    for ispin in range(model.nspin):
        for iorb in range(no):
            isite = (iorb + 1) + ispin * ns
            for particle, dn in ((True, 1), (False, -1)):
                jn = (nup + dn, ndw) if ispin == 0 else (nup, ndw + dn)
                if not (0 <= jn[0] <= ns and 0 <= jn[1] <= ns):
                    continue
                jmap = build_sector(ns, *jn)
                n2, vv = gf_vvinit(particle, isite, hmap, jmap, psi)
                vv = vv / np.sqrt(n2)
                nlanc = min(jmap.size, ngfiter)
                a, b, _ = lanczos_tridiag(model, jmap, vv, nlanc, nthreads=nthreads)
                gmt = np.zeros(lmats, np.complex128)
                grt = np.zeros(lreal, np.complex128)
                add_to_lanczos_gf(n2, e0, e0, zeta, False, model.beta, a, b, 1 if particle else -1,
                                  wm, wr, eps, gmt, grt)
                gm[ispin, iorb] += gmt
                gr[ispin, iorb] += grt
                chains.append(dict(ispin=ispin, iorb=iorb, particle=particle, norm2=n2, alpha=a,
                                   beta=b))
    sm = np.zeros_like(gm)
    for ispin in range(model.nspin):
        for iorb in range(no):
            sm[ispin, iorb] = sigma_normal(model.e[ispin, iorb], model.v[ispin, iorb], model.xmu,
                                           model.hloc[ispin, ispin, iorb, iorb].real, 1j * wm,
                                           gm[ispin, iorb])
    return dict(e0=e0, psi=psi, nlanc=nl, obs=obs, gmats=gm, greal=gr, smats=sm, chains=chains,
                map=hmap, wm=wm)


# ------------------------------------------------ finite-T pipeline ---
def _sector_eigs(model, hmap, k):
    """Lowest k eigenpairs of the sector H, degenerate copies included: dense
    eigh (the reference's small-sector branch, ED_DIAG.f90:184-194, used here up
    to 2500 states) or ARPACK eigsh ('SA', the eigensolver family of sp_eigh,
    with the reference's Nblock = 3*Neigen+5 as the minimum of ncv)."""
    H = sparse_h(model, hmap)
    if hmap.size <= 2500:
        w, V = np.linalg.eigh(H.toarray())
        return w[:k], V[:, :k]
    import scipy.sparse.linalg as sla
    ncv = min(hmap.size, max(3 * k + 5, 2 * k + 1, 20))
    w, V = sla.eigsh(H, k=k, which="SA", tol=1e-14, ncv=ncv)
    o = np.argsort(w)
    return w[o], V[:, o]


def _gf_and_obs(model, states, egs, zeta, finite_t, lmats, lreal, wini, wfin, eps, ngfiter,
                nthreads):
    """Observables (ED_OBSERVABLES.f90:113-160, weights exp(-beta(Ei-Egs))/Z or
    1/Z at T=0) and the particle/hole chains of every kept state
    (build_gf_normal.f90:71-180) summed with add_to_lanczos_gf_normal
    (:442-488), followed by get_sigma_normal.  states: [(e, nup, ndw, psi)]."""
    ns, no = model.ns, model.norb
    obs = {k: np.zeros(no) for k in ["dens", "dens_up", "dens_dw", "docc", "magz"]}
    obs["sz2"], obs["n2"], obs["s2tot"] = np.zeros((no, no)), np.zeros((no, no)), 0.0
    eacc = np.zeros(8)
    wm = matsubara(model.beta, lmats)
    wr = realaxis(wini, wfin, lreal)
    gm = np.zeros((model.nspin, no, lmats), np.complex128)
    gr = np.zeros((model.nspin, no, lreal), np.complex128)
    chains = []
    for e, a, b, psi in states:
        hm = build_sector(ns, a, b)
        peso = (np.exp(-model.beta * (e - egs)) if finite_t else 1.0) / zeta
        psi = np.asarray(psi).astype(np.complex128)
        o = observables_state(model, hm, psi, peso)
        for k in ["dens", "dens_up", "dens_dw", "docc", "magz"]:
            obs[k] += o[k]
        sz2, n2, s2 = moments_state(model, hm, psi, peso)
        obs["sz2"] += sz2
        obs["n2"] += n2
        obs["s2tot"] += s2
        local_energy_state(model, hm, psi, peso, eacc)
        for ispin in range(model.nspin):
            for iorb in range(no):
                isite = (iorb + 1) + ispin * ns
                for particle, dn in ((True, 1), (False, -1)):
                    jn = (a + dn, b) if ispin == 0 else (a, b + dn)
                    if not (0 <= jn[0] <= ns and 0 <= jn[1] <= ns):
                        continue
                    jmap = build_sector(ns, *jn)
                    n2, vv = gf_vvinit(particle, isite, hm, jmap, psi)
                    vv = vv / np.sqrt(n2)
                    nlanc = min(jmap.size, ngfiter)
                    al, bl, _ = lanczos_tridiag(model, jmap, vv, nlanc, nthreads=nthreads)
                    gmt = np.zeros(lmats, np.complex128)
                    grt = np.zeros(lreal, np.complex128)
                    add_to_lanczos_gf(n2, e, egs, zeta, finite_t, model.beta, al, bl,
                                      1 if particle else -1, wm, wr, eps, gmt, grt)
                    gm[ispin, iorb] += gmt
                    gr[ispin, iorb] += grt
                    chains.append(dict(ispin=ispin, iorb=iorb, particle=particle, norm2=n2,
                                       alpha=al, beta=bl, e=e, sector=(a, b)))
    sm = np.zeros_like(gm)
    for ispin in range(model.nspin):
        for iorb in range(no):
            sm[ispin, iorb] = sigma_normal(model.e[ispin, iorb], model.v[ispin, iorb], model.xmu,
                                           model.hloc[ispin, ispin, iorb, iorb].real, 1j * wm,
                                           gm[ispin, iorb])
    obs["eimp"], obs["doubles"] = local_energies(eacc)
    return obs, gm, gr, sm, chains, wm


def solve_t0(model, sectors=None, nstates_sector=6, gs_threshold=1e-9, dim_threshold=256,
             lmats=4096, lreal=0, wini=-5.0, wfin=5.0, eps=0.01, ngfiter=200, nitermax=512,
             tol=1e-12, nthreads=1, twin=False):
    """Zero-temperature impurity solve (lanc_nstates_total = 1) over the given
    sectors [(nup, ndw)] in the reference's order (default: all of them):
    ed_diag_c's T=0 branch (ED_DIAG.f90:93-228).  Every sector yields
    Neigen = min(dim, lanc_nstates_sector) eigenpairs (ED_SETUP.f90:423-425),
    from a dense eigh when Neigen == dim or dim <= lanc_dim_threshold
    (:136-137,184-194), else from the Lanczos branch.  Each eigenvalue in turn,
    sector by sector, goes through the ground-state selection of :202-214:
    below oldzero - 10*gs_threshold it empties the list and becomes oldzero;
    within gs_threshold of oldzero it is added and oldzero = min(oldzero, e).
    Z = the number of kept states (ed_analysis, :278-283).  The Lanczos branch
    with Neigen = 1 is the restated plain Lanczos ground state; with Neigen > 1
    it is ARPACK (the eigensolver family of sp_eigh), which returns
    degenerate copies."""
    ns = model.ns
    if sectors is None:
        sectors = [(a, b) for a in range(ns + 1) for b in range(ns + 1)]
    if twin:
        sectors = [(a, b) for a, b in sectors if a >= b]
    from math import comb
    allsecs = [(a, b) for a in range(ns + 1) for b in range(ns + 1)]
    lst = _StateList()
    oldzero = 1000.0
    nl_total = 0
    for a, b in sectors:
        dim = comb(ns, a) * comb(ns, b)
        neigen = min(dim, nstates_sector)
        hm = build_sector(ns, a, b)
        if neigen == 1 and dim > dim_threshold:
            e0, psi, nl = lanczos_gs(model, hm, nitermax=nitermax, threshold=tol,
                                     nthreads=nthreads)
            nl_total += nl
            w, V = [e0], psi[:, None]
        else:
            w, V = _sector_eigs(model, hm, neigen)
        isec = a * (ns + 1) + b + 1
        tsec = b * (ns + 1) + a + 1 if (twin and a != b) else None
        for i in range(neigen):
            en = float(w[i])
            if en < oldzero - 10.0 * gs_threshold:
                oldzero = en
                lst = _StateList()
                lst.add(en, isec, V[:, i], tsec)
            elif abs(en - oldzero) <= gs_threshold:
                oldzero = min(oldzero, en)
                lst.add(en, isec, V[:, i], tsec)
    ordered = [list(x) for x in _materialize(ns, allsecs, lst)]
    egs = min(s[0] for s in ordered)
    zeta = float(len(ordered))
    obs, gm, gr, sm, chains, wm = _gf_and_obs(model, ordered, egs, zeta, False, lmats, lreal,
                                              wini, wfin, eps, ngfiter, nthreads)
    return dict(states=[(s[0], s[1], s[2]) for s in ordered], psis=[s[3] for s in ordered],
                egs=egs, e0=egs, zeta=zeta, obs=obs, gmats=gm, greal=gr, smats=sm, chains=chains,
                wm=wm, nlanc=nl_total)


def twin_vector(ns, nup, ndw, vec):
    """es_return_cvector for a twin entry (ED_EIGENSPACE.f90:399-430): the
    vector in the twin sector (ndw, nup) rebuilt from the state's vector of
    sector (nup, ndw) through twin_sector_order (ED_SETUP.f90:1098-1126):
    Order = the permutation that sorts flip_state(map(i)) (up and down words
    exchanged, :1136-1161), vector(i) = cvec(Order(i))."""
    hm = build_sector(ns, nup, ndw).astype(np.int64)
    mask = (1 << ns) - 1
    flipped = ((hm >> ns) & mask) | ((hm & mask) << ns)
    order = np.argsort(flipped, kind="stable")
    return np.asarray(vec)[order]


class _StateList:
    """state_list with es_insert_state / es_add_state / es_pop_state
    (ED_EIGENSPACE.f90:126-299): entries [e, isector, vec, itwin]; a twin
    entry follows its state, carries no vector and leaves with it."""

    def __init__(self):
        self.s = []

    def insert(self, e, isec, v, twin_sec=None):
        i = 0
        while i < len(self.s) and not (e <= self.s[i][0]):
            i += 1
        self.s.insert(i, [e, isec, v, False])
        if twin_sec is not None:
            self.s.insert(i + 1, [e, twin_sec, None, True])

    def pop(self):
        tw = self.s[-1][3]
        self.s.pop()
        if tw and self.s:
            self.s.pop()

    def add(self, e, isec, v, twin_sec=None, size=None):
        if size is None or len(self.s) < size:
            self.insert(e, isec, v, twin_sec)
        elif e < self.s[-1][0]:
            self.pop()
            self.insert(e, isec, v, twin_sec)


def _materialize(ns, secs, lst):
    """(e, nup, ndw, vector) of every entry; twin entries get their vector
    from the state before them."""
    out = []
    for i, (e, isec, v, tw) in enumerate(lst.s):
        a, b = secs[isec - 1]
        if tw:
            pa, pb = secs[lst.s[i - 1][1] - 1]
            v = twin_vector(ns, pa, pb, lst.s[i - 1][2])
        out.append((e, a, b, v))
    return out


def solve_finite_t(model, lmats=256, lreal=0, wini=-5.0, wfin=5.0, eps=0.01, ngfiter=200,
                   nstates_sector=6, nstates_total=16, nstates_step=2, cutoff=1e-9, nthreads=1,
                   twin=False):
    """Finite-temperature solve over every sector: ed_diag_c (ED_DIAG.f90:93-228,
    finite-T branch with es_add_state's size cap, ED_EIGENSPACE.f90:126-151),
    ed_analysis (ED_DIAG.f90:248-398: Z before trimming, Neigen adaptation,
    cutoff trimming), observables with Boltzmann weights and the GF chains of
    every kept state (build_gf_normal.f90:71-180,442-488).  twin: ed_twin
    (sectors with nup < ndw skipped, twin entries for nup != ndw,
    ED_SETUP.f90:429-438, ED_DIAG.f90:111-123)."""
    ns = model.ns
    if nstates_total != 1:
        nstates_sector += nstates_sector % 2
        nstates_total += nstates_total % 2
    secs = [(a, b) for a in range(ns + 1) for b in range(ns + 1)]
    from math import comb
    neigen = [min(comb(ns, a) * comb(ns, b), nstates_sector) for a, b in secs]
    lst = _StateList()

    for isec0, (a, b) in enumerate(secs):
        if twin and a < b:
            continue
        tsec = b * (ns + 1) + a + 1 if (twin and a != b) else None
        hm = build_sector(ns, a, b)
        k = min(hm.size, neigen[isec0])
        w, V = _sector_eigs(model, hm, k)
        for i in range(k):
            lst.add(float(w[i]), isec0 + 1, V[:, i], tsec, nstates_total)
    states = lst.s
    egs = min(s[0] for s in states)
    zeta = sum(np.exp(-model.beta * (s[0] - egs)) for s in states)
    count = np.zeros(len(secs), int)
    for s in states:
        count[s[1] - 1] += 1
    new_neigen = []
    for i in range(len(secs)):
        ne = neigen[i] + (1 if count[i] > 0 else -1)
        if ne > count[i]:
            ne = count[i] + 1
        new_neigen.append(max(ne, 1))
    if np.exp(-model.beta * (states[-1][0] - egs)) > cutoff:
        new_total = nstates_total + nstates_step
    else:
        while len(states) > 1 and np.exp(-model.beta * (states[-1][0] - egs)) <= cutoff:
            lst.pop()
        new_total = max(len(states), nstates_step) + nstates_step
    st4 = _materialize(ns, secs, lst)
    obs, gm, gr, sm, chains, wm = _gf_and_obs(model, st4, egs, zeta, True, lmats, lreal, wini,
                                              wfin, eps, ngfiter, nthreads)
    return dict(states=[(s[0], s[1]) for s in lst.s], egs=egs, zeta=zeta, obs=obs, gmats=gm,
                greal=gr, smats=sm, neigen=new_neigen, nstates_total=new_total)
