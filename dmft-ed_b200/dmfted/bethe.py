"""The DMFT loop of the reference's Bethe-lattice driver on the device.

Mirrors drivers/ed_hm_bethe.f90:53-88: solve the impurity problem, read Sigma,
form the local Green's function on the semicircular density-of-states grid
(dmft_gloc_matsubara), the Weiss field or hybridisation (dmft_weiss /
dmft_delta), fit the bath to it (ed_chi2_fitgf), mix the bath with the previous
one (wmixing) and test convergence on the fitted function (check_convergence).
Every numeric step runs in the CUDA library; this module only sequences the
calls, as the Fortran driver does.
"""
import numpy as np

from . import CG_WEISS, EDSolver


def bethe_dos(le=500, wband=1.0):
    """He = linspace(-D, D, Le, mesh=de), Wte = dens_bethe(He, D)*de
    (drivers/ed_hm_bethe.f90:38-40) with the semicircle
    dens_bethe(x, D) = 2 sqrt(D^2 - x^2) / (pi D^2)."""
    he = np.linspace(-wband, wband, le)
    de = he[1] - he[0]
    wt = 2.0 * np.sqrt(np.maximum(wband ** 2 - he ** 2, 0.0)) / (np.pi * wband ** 2) * de
    return he, wt


class Convergence:
    """check_convergence of DMFT_Tools (absent from the tree; restated): the
    relative change err = sum|X - X_old| / sum|X| of the fitted function; the
    loop has converged after nsuccess consecutive iterations with err < eps."""

    def __init__(self, eps=1e-5, nsuccess=1):
        self.eps, self.nsuccess = eps, nsuccess
        self.old, self.count, self.err = None, 0, 1.0

    def __call__(self, x):
        x = np.asarray(x)
        if self.old is not None:
            self.err = float(np.abs(x - self.old).sum() / np.abs(x).sum())
            self.count = self.count + 1 if self.err < self.eps else 0
        self.old = x.copy()
        return self.count >= self.nsuccess


def dmft_step(solver: EDSolver, bath, he, wt, bath_prev=None, wmixing=0.5, scheme=None,
              sectors=None):
    """One iteration of the loop: returns (new bath, fitted function, fit chi2)."""
    solver.ed_solve(bath, sectors=sectors)
    smats = solver.ed_get_sigma_matsubara()
    gmats = solver.gloc_matsubara_diag(he, wt, smats)
    weiss = solver.get_weiss(gmats, smats, scheme)
    new = np.array(bath, np.float64, copy=True)
    chi2 = []
    for ispin in range(1, solver.params.nspin + 1):
        new, _, c2 = solver.ed_chi2_fitgf(weiss, new, ispin=ispin)
        chi2.append(c2)
    if bath_prev is not None:
        new = wmixing * new + (1.0 - wmixing) * np.asarray(bath_prev)
    return new, weiss, np.array(chi2)


def dmft_loop(solver: EDSolver, bath, le=500, wband=1.0, nloop=100, wmixing=0.5,
              dmft_error=1e-5, nsuccess=1, sectors=None):
    """The whole loop of drivers/ed_hm_bethe.f90:53-88; returns the final
    bath and the number of iterations."""
    he, wt = bethe_dos(le, wband)
    conv = Convergence(dmft_error, nsuccess)
    bath = np.array(bath, np.float64, copy=True)
    prev = None
    for iloop in range(1, nloop + 1):
        bath_fit, weiss, _ = dmft_step(solver, bath, he, wt, None, wmixing, None, sectors)
        # Bath = wmixing*Bath + (1-wmixing)*Bath_ after the first loop
        bath = bath_fit if iloop == 1 else wmixing * bath_fit + (1.0 - wmixing) * prev
        prev = bath.copy()
        if conv(weiss[0, 0, 0, 0]):
            break
    return bath, iloop


__all__ = ["bethe_dos", "Convergence", "dmft_step", "dmft_loop", "CG_WEISS"]
