"""ctypes front end of the CPU oracle (asr_oracle.cpp).

TEST INFRASTRUCTURE, NOT PRODUCT CODE: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs
use this module, and only as the checker.  Each method names the reference routine it restates.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int)
_l = C.POINTER(C.c_long)


def build():
    """Compile the oracle library in place (make)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_last_error.restype = C.c_char_p
        L.orc_build.restype = C.c_int
        L.orc_build_targets.restype = C.c_int
        L.orc_build.argtypes = [C.c_int, _i, _i, C.c_int, _i, _i, C.c_int, _d, C.c_int, _i, _i, C.c_int, _d, C.c_int, C.c_int,
                                C.c_int, _i, _i, _d, C.c_int, C.c_int, _d, C.POINTER(C.c_void_p)]
        L.orc_build_targets.argtypes = L.orc_build.argtypes[:-1] + [_i, C.c_int, _i, _i, C.POINTER(C.c_void_p)]
        L.orc_edc_green_proj.argtypes = [C.c_void_p, C.c_int, _d, _d, _d, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                                         C.c_int, C.c_int, _i, _i, _d, _d, _d, _d, _i]
        L.orc_epi_blocks.argtypes = [C.c_void_p, C.c_int, _d, _d, _d, _d, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, _d,
                                     _i]
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_dims.argtypes = [C.c_void_p, _i]
        L.orc_tables.argtypes = [C.c_void_p] + [_i] * 8 + [_d, _d, _i, _i, _i, _d, _d]
        L.orc_set_start.argtypes = [C.c_void_p, C.c_int]
        L.orc_set_chi.argtypes = [C.c_void_p, _d]
        L.orc_set_params.argtypes = [C.c_void_p, _d, _d, _d, _d]
        L.orc_freeze_site.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.orc_freeze_any.argtypes = [C.c_void_p, C.c_int, C.c_int, _i]
        L.orc_unfreeze.argtypes = [C.c_void_p]
        L.orc_set_class_conc.argtypes = [C.c_void_p, C.c_int, _d]
        L.orc_apply.argtypes = [C.c_void_p, _d, _d]
        L.orc_rand_c.argtypes = [C.c_void_p, _d, _d, _d]
        L.orc_project_c.argtypes = [C.c_void_p, _d]
        L.orc_hp_c.argtypes = [C.c_void_p, _d, _d]
        L.orc_chain_eigvals.argtypes = [C.c_int, _d, _d, _d]
        L.orc_cf_species.argtypes = [_d, _d, _d, C.c_int, C.c_double, C.c_double, C.c_int, _d, _d, _d, _d, _l]
        L.orc_bp_asymptote.argtypes = [_d, _d, C.c_int, _d, _d, _i]
        L.orc_tridiag_extreme.restype = C.c_double
        L.orc_tridiag_extreme.argtypes = [C.c_int, _d, _d, C.c_int]
        L.orc_terminated_green.argtypes = [_d, _d, C.c_int, C.c_int, C.c_int, C.c_int, _d, C.c_int, _d, _d]
        L.orc_terminator_coefs.argtypes = [_d, _d, C.c_int, C.c_int, C.c_double, C.c_double, _d, _d]
        L.orc_sqrt_tail.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, _d]
        L.orc_periodic_g.argtypes = [C.c_double, C.c_double, _d, _d, C.c_int, _d]
        L.orc_lanczos.argtypes = [C.c_void_p, _d, C.c_int, C.c_double, _d, _d, _i]
        L.orc_set_apply_threads.argtypes = [C.c_int]
        L.orc_apply_threads.restype = C.c_int
        L.orc_edc_green.argtypes = [C.c_void_p, C.c_int, _d, _d, _d, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double,
                                    C.c_int, C.c_int, _d, _d, _d, _i, _l]
        L.orc_edc_green_blk.argtypes = [C.c_void_p, C.c_int, _d, _d, _d, _d, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int,
                                        C.c_int, _d, _i, _d, _d, _l]
        L.orc_chain_greens.argtypes = [C.c_void_p, C.c_int, _d, _i, C.c_int, _i, _i, _d, C.c_int, C.c_int, C.c_double,
                                       C.c_int, C.c_int, C.c_int, _d, _l, C.c_int, _d, _d, _i]
        L.orc_ed3_blocks.argtypes = [C.c_void_p, C.c_int, _d, _d, _d, _d, _d, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                     C.c_double, C.c_int, C.c_int, _d, _i, _d, _d, _d, _l]
        L.orc_gauss_legendre.argtypes = [C.c_int, _d, _d]
        L.orc_contour_nodes.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, _d, _d]
        L.orc_contour_nodes_closed.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, _d, _d]
        L.orc_contour_nodes_fermi.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, _d, _d]
        L.orc_contour_moment.restype = C.c_double
        L.orc_contour_moment.argtypes = [_d, _d, _d, C.c_int, C.c_double, C.c_int]
        L.orc_rademacher.restype = C.c_double
        L.orc_rademacher.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
        L.orc_real_apply.argtypes = [C.c_int, C.c_int, _i, _i, _d, _d, _d, _d, _d, _d, _d, _d]
        L.orc_kpm_moments.argtypes = [C.c_int, C.c_int, _i, _i, _d, _d, _d, _d, _d, _d, C.c_double, C.c_double, C.c_int,
                                      C.c_int, C.c_int, C.c_uint64, _d]
        L.orc_kpm_dos.argtypes = [_d, C.c_int, C.c_double, C.c_double, _d, C.c_int, _d]
        _LIB = L
    return _LIB


class apply_threads:
    """Context manager: the node loops of the oracle's operator applications on n threads (all host threads by default)
    inside the block, serial again after it.  Every node is computed by one thread with the same operations, so the
    results are the same bits as on one thread; only single-chain oracle calls use it (chain_greens' tasks stay serial)."""

    def __init__(self, n: int = 0):
        self.n = n if n > 0 else len(os.sched_getaffinity(0))

    def __enter__(self):
        self.prev = lib().orc_apply_threads()
        lib().orc_set_apply_threads(self.n)
        return self

    def __exit__(self, *exc):
        lib().orc_set_apply_threads(self.prev)
        return False


def _pd(a):
    return a.ctypes.data_as(_d) if a is not None else None


def _pi(a):
    return a.ctypes.data_as(_i) if a is not None else None


def _f64(a, cplx=False):
    a = np.asarray(a, dtype=np.complex128 if cplx else np.float64)
    return np.asfortranarray(a)


def _i32(a):
    return np.asfortranarray(np.asarray(a, dtype=np.int32))


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().orc_last_error().decode())


TAILS = {"none": 0, "hull": 1, "bp": 2, "avg2": 3}


class OracleOp:
    """Restatement of ``augcls_op`` (src/asr_augcls.f90:45-68) built by ``build_augcls_operator`` (:596-823)."""

    def __init__(self, graph, model, cls, perm, dmat, start=1, maxlevel=4, maxrank=0, flippable=None, stype=None, tsite=None):
        """tsite (1-based target sites, optional): the target links of build_augcls_operator (src/asr_augcls.f90:808-820)
        become self.tnode, self.tgop (nsmax, nt), 1-based (tnode 0: no node)."""
        L = lib()
        self._keep = []
        nbr_ptr, nbr = _i32(graph.nbr_ptr), _i32(graph.nbr)
        nsc, spc, conc = _i32(model.nsc), _i32(model.spc), _f64(model.conc)
        cls, perm, dmat = _i32(cls), _i32(perm), _f64(dmat)
        fl = _i32(flippable) if flippable is not None else None
        st = _i32(stype) if stype is not None else None
        block, block0 = _f64(model.block), _f64(model.block0)
        h = C.c_void_p()
        args = (graph.n, _pi(nbr_ptr), _pi(nbr), model.ncls, _pi(nsc), _pi(spc), spc.shape[0], _pd(conc), model.nsp, _pi(cls),
                _pi(perm), perm.shape[1], _pd(dmat), start, maxlevel, maxrank, _pi(fl), _pi(st), _pd(block), block.shape[2],
                block.shape[3], _pd(block0))
        self.tnode = self.tgop = None
        if tsite is None:
            rc = L.orc_build(*args, C.byref(h))
        else:
            ts = _i32(np.atleast_1d(tsite))
            nsm = int(np.max(nsc))
            self.tnode = np.zeros((nsm, ts.shape[0]), np.int32, order="F")
            self.tgop = np.zeros((nsm, ts.shape[0]), np.int32, order="F")
            rc = L.orc_build_targets(*args, _pi(ts), ts.shape[0], _pi(self.tnode), _pi(self.tgop), C.byref(h))
        _check(rc)
        self.h = h
        dims = np.zeros(7, dtype=np.int32)
        L.orc_dims(h, _pi(dims))
        self.nn, self.nslot, self.nsmax, self.nop, self.ncls, self.ntype, self.nstab = (int(x) for x in dims)
        self.nsp = model.nsp

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_free(self.h)
            self.h = None

    @property
    def dim(self):
        return 9 * self.nn

    def tables(self) -> dict:
        nn, ns, nsm, nop = self.nn, self.nslot, self.nsmax, self.nop
        t = dict(flipr=np.zeros((nsm, nn), np.int32, order="F"), flipg=np.zeros((nsm, nn), np.int32, order="F"),
                 hopr=np.zeros((ns, nn), np.int32, order="F"), hopg=np.zeros((ns, nn), np.int32, order="F"),
                 lst=np.zeros(nn, np.int32), site=np.zeros(nn, np.int32), ncl=np.zeros(nn, np.int32),
                 level=np.zeros(nn, np.int32), norb=np.zeros(nn), sq=np.zeros(nn), stab_ptr=np.zeros(nn + 1, np.int32),
                 stab=np.zeros(max(self.nstab, 1), np.int32), pi=np.zeros((9, nop), np.int32, order="F"),
                 sg=np.zeros((9, nop), order="F"), mt=np.zeros((nsm, nsm, nsm, self.ncls), order="F"))
        lib().orc_tables(self.h, *[_pi(t[k]) for k in ("flipr", "flipg", "hopr", "hopg", "lst", "site", "ncl", "level")],
                         _pd(t["norb"]), _pd(t["sq"]), _pi(t["stab_ptr"]), _pi(t["stab"]), _pi(t["pi"]), _pd(t["sg"]),
                         _pd(t["mt"]))
        t["stab"] = t["stab"][: self.nstab]
        return t

    # ---- parameters (src/asr_augcls.f90:107-185)
    def set_params(self, c, d, o, e):
        self._p = [_f64(x) for x in (c, d, o, e)]
        lib().orc_set_params(self.h, *[_pd(x) for x in self._p])

    def set_start(self, l0):
        _check(lib().orc_set_start(self.h, l0))

    def set_chi(self, chi):
        _check(lib().orc_set_chi(self.h, _pd(_f64(chi))))

    def freeze_site(self, site, sp):
        """``augcls_freeze_site`` (src/asr_augcls.f90:129-142): sp must belong to the start node's class when the site is the
        start site."""
        _check(lib().orc_freeze_site(self.h, site, sp))

    def freeze_any(self, site, sp):
        """``augcls_freeze_any`` (src/asr_augcls.f90:147-161): any species index; returns the number of nodes on the site."""
        n = C.c_int(0)
        _check(lib().orc_freeze_any(self.h, site, sp, C.byref(n)))
        return n.value

    def unfreeze(self):
        lib().orc_unfreeze(self.h)

    def set_class_conc(self, kap, conc):
        _check(lib().orc_set_class_conc(self.h, kap, _pd(_f64(conc))))

    # ---- application
    def apply(self, x):
        """``augcls_apply``: y = H x, real, normalised coordinates."""
        x = _f64(x)
        y = np.zeros_like(x)
        lib().orc_apply(self.h, _pd(x), _pd(y))
        return y

    def rand_c(self, par, x):
        """``augcls_rand_c``: w = X x, complex par (9, nsp)."""
        par = _f64(par, True)
        x = _f64(x, True)
        w = np.zeros_like(x)
        lib().orc_rand_c(self.h, _pd(par), _pd(x), _pd(w))
        return w

    def project_c(self, x):
        x = _f64(x, True).copy()
        lib().orc_project_c(self.h, _pd(x))
        return x

    def hp_c(self, x):
        x = _f64(x, True)
        y = np.zeros_like(x)
        lib().orc_hp_c(self.h, _pd(x), _pd(y))
        return y

    # ---- chains
    def lanczos(self, v0, nmax, tiny=1.0e-12):
        """Reference ``lanczos`` (src/reference/asr_recursion.f90:17-58) on ``augcls_apply``."""
        v0 = _f64(v0)
        a = np.zeros(nmax)
        b = np.zeros(nmax)
        n = C.c_int()
        lib().orc_lanczos(self.h, _pd(v0), nmax, tiny, _pd(a), _pd(b), C.byref(n))
        return a, b, n.value

    def edc_green(self, ed, z, iv, nlev, depth_tol=0.0, tail="hull", project=True):
        """``edc_green`` (src/asr_edc.f90:75-164): returns (g, a, b, mused, nfall)."""
        dc, dl, en = _f64(ed["dc"]), _f64(ed["dl"]), _f64(ed["enu"])
        g = np.zeros(2)
        a = np.zeros(nlev, np.complex128)
        b = np.zeros(nlev, np.complex128)
        m = C.c_int()
        nf = C.c_long(0)
        lib().orc_edc_green(self.h, dl.shape[1], _pd(dc), _pd(dl), _pd(en), z.real, z.imag, iv, nlev, depth_tol, TAILS[tail],
                            int(project), _pd(g), _pd(a), _pd(b), C.byref(m), C.byref(nf))
        return complex(g[0], g[1]), a[: m.value], b[: m.value], m.value, nf.value

    def edc_green_proj(self, ed, z, iv, nlev, tnode, tgop, tw, tail="hull", project=True):
        """``edc_green_proj`` (src/asr_edc.f90:174-232): returns (g, gp (9, nt), gp4 (9, nt), mused)."""
        dc, dl, en = _f64(ed["dc"]), _f64(ed["dl"]), _f64(ed["enu"])
        tnode, tgop, tw = _i32(tnode), _i32(tgop), _f64(tw)
        nt = tnode.shape[1]
        g = np.zeros(2)
        gp = np.zeros((9, nt), np.complex128, order="F")
        gp4 = np.zeros((9, nt), np.complex128, order="F")
        m = C.c_int()
        lib().orc_edc_green_proj(self.h, dl.shape[1], _pd(dc), _pd(dl), _pd(en), z.real, z.imag, iv, nlev, TAILS[tail],
                                 int(project), nt, _pi(tnode), _pi(tgop), _pd(tw), _pd(g), _pd(gp), _pd(gp4), C.byref(m))
        return complex(g[0], g[1]), gp, gp4, m.value

    def epi_blocks(self, ed, v9, z, nlev, tail="hull", project=True):
        """``epi_start`` + ``epi_blocks`` (src/asr_epi.f90:578-663) on the operator's current parameters, frozen sites and
        characters: returns (x (4,) complex = X0, X1, X2, X1 mismatch; (m0, m1))."""
        dc, dl, en = _f64(ed["dc"]), _f64(ed["dl"]), _f64(ed["enu"])
        x = np.zeros(4, np.complex128)
        m = np.zeros(2, np.int32)
        _check(lib().orc_epi_blocks(self.h, dl.shape[1], _pd(dc), _pd(dl), _pd(en), _pd(_f64(v9)), z.real, z.imag, nlev,
                                    TAILS[tail], int(project), _pd(x), _pi(m)))
        return x, (int(m[0]), int(m[1]))

    def edc_green_blk(self, ed, zs, iv, nlev, depth_tol=0.0, tail="hull", project=True):
        """``edc_green_blk`` (src/asr_edc.f90:237-316): returns (g(nb), mused(nb), a(nlev, nb), b(nlev, nb))."""
        dc, dl, en = _f64(ed["dc"]), _f64(ed["dl"]), _f64(ed["enu"])
        zs = np.ascontiguousarray(zs, dtype=np.complex128)
        nb = zs.shape[0]
        g = np.zeros(nb, np.complex128)
        mu = np.zeros(nb, np.int32)
        a = np.zeros((nb, nlev), np.complex128)   # memory order of Fortran a(nlev, nb)
        b = np.zeros((nb, nlev), np.complex128)
        nf = C.c_long(0)
        lib().orc_edc_green_blk(self.h, dl.shape[1], _pd(dc), _pd(dl), _pd(en), _pd(zs), nb, iv, nlev,
                                depth_tol, TAILS[tail], int(project), _pd(g), _pi(mu),
                                _pd(a), _pd(b), C.byref(nf))
        return g, mu, a.T, b.T

    def ed3_blocks(self, ed3, zs, iv, nlev, depth_tol=0.0, tail="hull", project=True):
        """``ed3_blocks`` (src/asr_ed3.f90:242-265) per energy on the operator's current parameters (set_params with
        c = g, d, o = e = 0; start site frozen to the central species; set_start(iv)).  Returns (bk (4, nz), m (2, nz),
        a, b, c (nz, 2, nlev))."""
        ns = int(np.asarray(ed3["dl"]).shape[1])
        arrs = [_f64(ed3[k]) for k in ("dc", "dl", "enu", "o", "p")]
        zs = np.atleast_1d(np.asarray(zs, np.complex128))
        nz = zs.shape[0]
        bk = np.zeros((nz, 4), np.complex128)
        m = np.zeros((nz, 2), np.int32)
        a = np.zeros((nz, 2, nlev), np.complex128)
        b = np.zeros((nz, 2, nlev), np.complex128)
        c = np.zeros((nz, 2, nlev), np.complex128)
        nf = C.c_long(0)
        for j in range(nz):
            _check(lib().orc_ed3_blocks(self.h, ns, *[_pd(x) for x in arrs], int(ed3["central"]), zs[j].real, zs[j].imag, iv,
                                        nlev, depth_tol, TAILS[tail], int(project), _pd(bk[j]), _pi(m[j]), _pd(a[j]), _pd(b[j]),
                                        _pd(c[j]), C.byref(nf)))
        return bk.T, m.T, a, b, c

    def chain_greens(self, groups, gcomp, iorb, nlevq, zs, nbe, depth_tol=0.0, tail="hull", project=True, nthreads=0,
                     coefs=False):
        """``chain_greens`` (src/asr_class_scf.f90:966-1160): groups is a list of dicts with c, d, o, e, dc, dl, enu;
        gcomp the central species (0: none frozen); iorb the start orbitals; nlevq (ngroup, norb) depths.  Returns
        (gz (nz, norb, ngroup), chain-steps); with coefs also dict(a, b = (nlevmax, nz, norb, ngroup), m = (nz, norb,
        ngroup)) of every chain."""
        nsp = self.nsp
        P = np.concatenate([np.concatenate([_f64(gq[k]).ravel(order="F") for k in ("c", "d", "o", "e", "dc", "dl", "enu")])
                            for gq in groups])
        gcomp, iorb = _i32(gcomp), _i32(iorb)
        nlevq = _i32(nlevq)
        zs = np.ascontiguousarray(zs, dtype=np.complex128)
        nz = zs.shape[0]
        gz = np.zeros((len(groups), len(iorb), nz), np.complex128)   # memory order of Fortran gz(nz, norb, ngroup)
        steps = C.c_long(0)
        assert P.shape[0] == len(groups) * (4 * 9 * nsp + 9 + 18 * nsp)
        ld = int(np.max(nlevq)) if coefs else 1
        az = np.zeros((len(groups), len(iorb), nz, ld), np.complex128) if coefs else None
        bz = np.zeros_like(az) if coefs else None
        mz = np.zeros((len(groups), len(iorb), nz), np.int32) if coefs else None
        _check(lib().orc_chain_greens(self.h, len(groups), _pd(P), _pi(gcomp), len(iorb), _pi(iorb), _pi(nlevq),
                                      _pd(zs), nz, nbe, depth_tol, TAILS[tail], int(project), nthreads,
                                      _pd(gz), C.byref(steps), ld, _pd(az) if coefs else None, _pd(bz) if coefs else None,
                                      _pi(mz) if coefs else None))
        if not coefs:
            return gz.transpose(2, 1, 0), steps.value
        return gz.transpose(2, 1, 0), steps.value, dict(a=az.transpose(3, 2, 1, 0), b=bz.transpose(3, 2, 1, 0),
                                                        m=mz.transpose(2, 1, 0))


def dos_final(oop, groups, gcomp, iorb, nlevq, lorb, worb, pcomp, spin, ncomp, nspin, emin, emax, eta, ndos, nthreads=0,
              depth_tol=0.0, tail="hull"):
    """``dos_final`` (src/asr_class_scf.f90:1912-1931) on the oracle: energies e_ie = emin + (emax - emin)(ie - 1) /
    max(ndos - 1, 1), ``chain_greens`` at e + i eta for the groups (parameter sets) x start orbitals iorb, then
    edos(ie, l, comp, spin) -= worb(o) Im G / pi for l = lorb(o); group q of the parameter sets belongs to component
    pcomp[q] and spin spin[q] (1-based).  Returns (e, edos (ndos, 3, ncomp, nspin))."""
    e = np.array([emin + (emax - emin) * ie / max(ndos - 1, 1) for ie in range(ndos)])
    gz, _ = oop.chain_greens(groups, gcomp, iorb, nlevq, e + 1j * eta, 4, depth_tol=depth_tol, tail=tail, nthreads=nthreads)
    edos = np.zeros((ndos, 3, ncomp, nspin))
    for q in range(len(groups)):
        for o in range(len(iorb)):
            edos[:, lorb[o], pcomp[q] - 1, spin[q] - 1] -= worb[o] * gz[:, o, q].imag / np.pi
    return e, edos


# ---------------------------------------------------------------------------------------------- free functions
def chain_eigvals(a, b):
    a = np.ascontiguousarray(a, np.complex128)
    b = np.ascontiguousarray(b, np.complex128)
    ev = np.zeros(a.shape[0], np.complex128)
    rc = lib().orc_chain_eigvals(a.shape[0], _pd(a), _pd(b), _pd(ev))
    if rc:
        raise RuntimeError("chain_eigvals: QR did not converge")
    return ev


def cf_species(a, b, m, z, tail="hull", c=None, want_pv=False):
    """``cf_species`` (src/asr_chain.f90:67-167): returns (g11, f, edges, pv, nfall)."""
    a = np.ascontiguousarray(a, np.complex128)
    b = np.ascontiguousarray(b, np.complex128)
    if b.shape[0] < a.shape[0]:
        b = np.concatenate([b, np.zeros(a.shape[0] - b.shape[0], np.complex128)])
    cc = np.ascontiguousarray(c if c is not None else np.zeros(a.shape[0]), np.complex128)
    g = np.zeros(2)
    f = np.zeros(2)
    e = np.zeros(2, np.complex128)
    pv = np.zeros(max(m, 1), np.complex128)
    nf = C.c_long(0)
    lib().orc_cf_species(_pd(a), _pd(b), _pd(cc), m, z.real, z.imag,
                         TAILS[tail], _pd(g), _pd(f), _pd(e), _pd(pv), C.byref(nf))
    return complex(g[0], g[1]), complex(f[0], f[1]), e, (pv if want_pv else None), nf.value


def bp_asymptote(a, b, n):
    """``bp_asymptote`` (src/reference/asr_terminator.f90:39-67): (ainf, binf, niter, converged)."""
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    ai, bi, it = C.c_double(), C.c_double(), C.c_int()
    ok = lib().orc_bp_asymptote(_pd(a), _pd(b), n, C.byref(ai), C.byref(bi), C.byref(it))
    return ai.value, bi.value, it.value, bool(ok)


METHODS = {"sqrt-last": 0, "sqrt-avg2": 1, "beer-pettifor": 2, "periodic2": 3}


def terminated_green(a, b, n, z, method="beer-pettifor", join="butt", ninterp=0):
    """``make_terminator`` + ``terminated_green`` (src/reference/asr_terminator.f90:83-126) at the energies z."""
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    z = np.ascontiguousarray(np.atleast_1d(z), np.complex128)
    g = np.zeros(z.shape[0], np.complex128)
    tp = np.zeros(3)
    _check(lib().orc_terminated_green(_pd(a), _pd(b), n, METHODS[method], 1 if join == "luchini-nex" else 0, ninterp,
                                      _pd(z), z.shape[0], _pd(g), _pd(tp)))
    return g, tp


def terminator_coefs(a, b, n, ninterp, ainf, binf):
    ta = np.zeros(n + ninterp)
    tb = np.zeros(n + ninterp)
    lib().orc_terminator_coefs(_pd(np.ascontiguousarray(a, np.float64)), _pd(np.ascontiguousarray(b, np.float64)), n, ninterp,
                               ainf, binf, _pd(ta), _pd(tb))
    return ta, tb


def sqrt_tail(z, ainf, binf):
    t = np.zeros(2)
    lib().orc_sqrt_tail(z.real, z.imag, ainf, binf, _pd(t))
    return complex(t[0], t[1])


def periodic_g(z, ap, bp):
    ap = np.ascontiguousarray(ap, np.float64)
    bp = np.ascontiguousarray(bp, np.float64)
    g = np.zeros(2)
    lib().orc_periodic_g(z.real, z.imag, _pd(ap), _pd(bp), ap.shape[0], _pd(g))
    return complex(g[0], g[1])


def tridiag_extreme(d, e, upper):
    d = np.ascontiguousarray(d, np.float64)
    e = np.ascontiguousarray(e, np.float64)
    return lib().orc_tridiag_extreme(d.shape[0], _pd(d), _pd(e), int(upper))


def gauss_legendre(n):
    x = np.zeros(n)
    w = np.zeros(n)
    lib().orc_gauss_legendre(n, _pd(x), _pd(w))
    return x, w


def contour_nodes(ebot, ef, n, eta_end=None):
    z = np.zeros(n, np.complex128)
    w = np.zeros(n, np.complex128)
    lib().orc_contour_nodes(ebot, ef, n, -1.0 if eta_end is None else eta_end, _pd(z), _pd(w))
    return z, w


def contour_nodes_closed(ebot, ef, eta, n_arc, n_vert):
    z = np.zeros(n_arc + n_vert, np.complex128)
    w = np.zeros(n_arc + n_vert, np.complex128)
    lib().orc_contour_nodes_closed(ebot, ef, eta, n_arc, n_vert, _pd(z), _pd(w))
    return z, w


def contour_nodes_fermi(ebot, mu, kt, npole, n_main, n_step):
    n = 4 + n_main + n_step + 8 + npole
    z = np.zeros(n, np.complex128)
    w = np.zeros(n, np.complex128)
    lib().orc_contour_nodes_fermi(ebot, mu, kt, npole, n_main, n_step, _pd(z), _pd(w))
    return z, w


def contour_moment(z, w, g, enu, k):
    z = np.ascontiguousarray(z, np.complex128)
    w = np.ascontiguousarray(w, np.complex128)
    g = np.ascontiguousarray(g, np.complex128)
    return lib().orc_contour_moment(_pd(z), _pd(w), _pd(g), z.shape[0],
                                    enu, k)


def rademacher(seed, v, q):
    return lib().orc_rademacher(seed, v, q)


def real_apply(nbr, spc, c, d, o, e, block, block0, x):
    """``real_apply`` (src/reference/asr_lmto_realization.f90:149-191) on an explicit supercell, n species."""
    nbr = _i32(nbr)
    spc = _i32(spc)
    x = _f64(x)
    y = np.zeros_like(x)
    lib().orc_real_apply(nbr.shape[1], nbr.shape[0], _pi(nbr), _pi(spc), *[_pd(_f64(t)) for t in (c, d, o, e, block, block0)],
                         _pd(x), _pd(y))
    return y


def kpm_moments(nbr, spc, c, d, o, e, block, block0, cen, sc, nmom, v0, nvec, seed):
    """``kpm_moments`` (src/reference/asr_kpm.f90:39-65) with the counter-based Rademacher vectors."""
    nbr = _i32(nbr)
    spc = _i32(spc)
    mu = np.zeros(nmom)
    args = [_f64(t) for t in (c, d, o, e, block, block0)]
    lib().orc_kpm_moments(nbr.shape[1], nbr.shape[0], _pi(nbr), _pi(spc), *[_pd(t) for t in args], cen, sc, nmom, v0, nvec,
                          seed, _pd(mu))
    return mu


def kpm_dos(mu, cen, sc, e):
    mu = np.ascontiguousarray(mu, np.float64)
    e = np.ascontiguousarray(e, np.float64)
    rho = np.zeros(e.shape[0])
    lib().orc_kpm_dos(_pd(mu), mu.shape[0], cen, sc, _pd(e), e.shape[0], _pd(rho))
    return rho
