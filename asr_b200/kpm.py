"""Kernel polynomial method on an explicit supercell: ``kpm_moments`` / ``kpm_dos`` (src/reference/asr_kpm.f90:39-87) on
the realisation operator ``lmto_real_op`` (src/reference/asr_lmto_realization.f90:14-191), n species, on the GPU."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib
from .augcls import Context, default_context, _f64, _i32, _pd, _pi


class Supercell:
    """One realisation (species per site) of the alloy on a periodic supercell: H = E_nu + h - h o h, h = c + d S d."""

    def __init__(self, nbr, spc, c, d, o=None, e=None, block=None, block0=None, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        nbr = _i32(nbr)                 # (nslot, nsite)
        spc = _i32(spc)
        c, d = _f64(c), _f64(d)
        nsp = c.shape[1]
        o = _f64(o) if o is not None else np.zeros_like(c, order="F")
        e = _f64(e) if e is not None else np.zeros_like(c, order="F")
        block = _f64(block)
        block0 = _f64(block0) if block0 is not None else None
        self.n, self.ns, self.nsp = nbr.shape[1], nbr.shape[0], nsp
        h = C.c_void_p()
        check(lib().asr_supercell_build(self.ctx.h, self.n, self.ns, _pi(nbr), _pi(spc), nsp, _pd(c), _pd(d), _pd(o), _pd(e),
                                        _pd(block), _pd(block0), C.byref(h)))
        self.h = h

    def free(self):
        if getattr(self, "h", None):
            lib().asr_supercell_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    @property
    def dim(self):
        return 9 * self.n

    def apply(self, x):
        """``real_apply``: y = H x, x (9 n,) or (9 n, nvec)."""
        x = _f64(x)
        one = x.ndim == 1
        X = x.reshape(self.dim, -1, order="F")
        Y = np.zeros_like(X, order="F")
        check(lib().asr_supercell_apply(self.h, _pd(X), _pd(Y), X.shape[1]))
        return Y[:, 0] if one else Y

    def kpm_moments(self, cen: float, sc: float, nmom: int, nvec: int, seed: int = 0, v0: int = 0, precision: str = "fp64",
                    doubling: bool = True):
        """mu(0:nmom-1) over the Rademacher vectors v0 .. v0+nvec-1 (counter-based generator, see include/asr_b200.h)."""
        mu = np.zeros(nmom)
        check(lib().asr_kpm_moments(self.ctx.h, self.h, cen, sc, nmom, v0, nvec, seed, _lib.FP32 if precision == "fp32" else _lib.FP64,
                                    int(bool(doubling)), _pd(mu)))
        return mu


def kpm_dos(mu, cen: float, sc: float, e):
    """``kpm_dos``: Jackson-kernel DOS on the grid e."""
    mu = np.ascontiguousarray(mu, np.float64)
    e = np.ascontiguousarray(e, np.float64)
    rho = np.zeros(e.shape[0])
    check(lib().asr_kpm_dos(_pd(mu), mu.shape[0], cen, sc, _pd(e), e.shape[0], _pd(rho)))
    return rho


def sro_layout(nbr, z: int, conc, alpha=None, seed: int = 0, sweeps: int = 20):
    """Species per site (1-based) with first-shell Warren-Cowley parameters alpha (nsp, nsp; unlike pairs used).
    nbr (nslot, nsite) 1-based, the first z slots being the first shell.  Returns (spc, achieved alpha)."""
    nbr = _i32(nbr)
    conc = np.ascontiguousarray(conc, np.float64)
    nsp = conc.shape[0]
    al = _f64(alpha) if alpha is not None else None
    spc = np.zeros(nbr.shape[1], np.int32)
    aout = np.zeros((nsp, nsp), order="F")
    check(lib().asr_sro_layout(nbr.shape[1], z, _pi(nbr), nbr.shape[0], nsp, _pd(conc), _pd(al), seed, sweeps, _pi(spc), _pd(aout)))
    return spc, aout


def fcc_supercell(l: int, conc, alpha1: float | None, seed: int, sweeps: int = 20):
    """fcc l^3 conventional cells with NN + NNN slots (12 + 6); species with first-shell alpha_ab = alpha1 for every
    unlike pair.  Returns (nbr (18, n), spc, bvec, achieved alpha)."""
    from .lattices import periodic_graph_shells
    g, coord, bvec = periodic_graph_shells("fcc", l, 4)
    ns = bvec.shape[1]
    nbr = np.asfortranarray(g.nbr.reshape(g.n, ns).T)
    nsp = len(conc)
    alpha = None
    if alpha1 is not None:
        alpha = np.full((nsp, nsp), float(alpha1))
        np.fill_diagonal(alpha, 0.0)
    spc, aout = sro_layout(nbr, 12, conc, alpha, seed, sweeps)
    return nbr, spc, bvec, aout
