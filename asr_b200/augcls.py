"""Site-class augmented-space operator: the drop-in for ``augcls_op`` (src/asr_augcls.f90:45-68).

Same names, argument meaning and error behaviour as the reference (errors raise ``AsrError`` where the reference stops):

* ``build_augcls_operator(g, mdl, cls, perm, dmat, start, maxlevel, maxrank=, flippable=, stype=)`` -- :596-823,
  built on the GPU;
* ``AugclsOp.set_params / freeze_site / freeze_any / set_start / set_chi / set_class_conc`` -- :107-185;
* ``AugclsOp.apply`` (``linop%apply``, ``augcls_apply`` :275-297), ``rand_c`` (:419-446), ``project_c`` (:329-348);
* ``AugclsOp.tables()`` -- host copies of the node tables in the reference layout (1-based).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib


def _f64(a, cplx=False):
    return np.asfortranarray(np.asarray(a, dtype=np.complex128 if cplx else np.float64))


def _i32(a):
    return np.asfortranarray(np.asarray(a, dtype=np.int32))


def _pd(a):
    return a.ctypes.data_as(_lib.d_p) if a is not None else None


def _pi(a):
    return a.ctypes.data_as(_lib.i_p) if a is not None else None


class Context:
    """Device context (stream and workspace) on one GPU: ``asr_ctx_create``."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().asr_ctx_create(device, C.byref(h)))
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            lib().asr_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        check(lib().asr_ctx_sync(self.h))

    def set_stream(self, stream_ptr: int | None):
        """Run on the caller's CUDA stream (e.g. ``torch.cuda.current_stream().cuda_stream``); None: the own stream."""
        check(lib().asr_ctx_set_stream(self.h, C.c_void_p(stream_ptr) if stream_ptr else None))

    KERNEL_KINDS = {"step": 0, "lanczos": 1, "kpm": 2, "adjoint": 3, "adj_step": 4, "adj_vec": 5, "adj_grad": 6,
                    "adj_scal": 7}

    def hold_workspace(self, on: bool):
        """Keep the device vector memory of the chain runs and the adjoint in this context between calls (on) or free it
        (off, the default)."""
        check(lib().asr_ctx_hold_workspace(self.h, int(bool(on))))

    def profile(self, on: bool):
        """Start (and clear) or stop the per-launch event timing of the hot kernels."""
        check(lib().asr_ctx_profile(self.h, int(bool(on))))

    def kernel_stats(self, kind: str = "step") -> dict:
        """Summed device time, launches and algorithmic bytes and flops of one kernel kind since ``profile(True)``:
        'step' (chain step operator), 'lanczos' (Lanczos update), 'kpm' (Chebyshev step), 'adjoint' (reverse level), and
        the reverse level's parts 'adj_step' (operator on wbar), 'adj_vec' (vector updates), 'adj_grad' (parameter
        gradient) and 'adj_scal' (dot sums and scalars)."""
        ms, n, by, fl = C.c_double(), C.c_int64(), C.c_double(), C.c_double()
        check(lib().asr_ctx_kernel_stats_kind(self.h, self.KERNEL_KINDS[kind], C.byref(ms), C.byref(n), C.byref(by),
                                              C.byref(fl)))
        return dict(ms=ms.value, launches=n.value, bytes=by.value, flops=fl.value)

    def launches(self) -> int:
        """Kernels launched by this context so far."""
        n = C.c_int64()
        check(lib().asr_ctx_launches(self.h, C.byref(n)))
        return n.value

    def stats(self):
        """(ed_nchain, ed_nlev, ed_nfall) counters of src/asr_chain.f90:14-17."""
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().asr_ctx_stats(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value


_DEFAULT_CTX = {}


def default_context(device: int = 0) -> Context:
    if device not in _DEFAULT_CTX:
        _DEFAULT_CTX[device] = Context(device)
    return _DEFAULT_CTX[device]


class AugclsOp:
    """The group-reduced site-class operator on the device."""

    def __init__(self, ctx: Context, handle, nsp: int):
        self.ctx = ctx
        self.h = handle
        dims = np.zeros(8, np.int32)
        check(lib().asr_op_dims(self.h, _pi(dims)))
        self.nn, self.nslot, self.nsmax, self.nop, self.ncls, self.ntype, self.nstab, self.nsp = (int(x) for x in dims)
        z = np.zeros((9, self.nsp), order="F")
        self.params = dict(c=z, d=z, o=z, e=z)

    def free(self):
        if getattr(self, "h", None):
            lib().asr_op_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    @property
    def dim(self) -> int:
        """``augcls_dim``: 9 nn."""
        return 9 * self.nn

    def tables(self) -> dict:
        nn, ns, nsm = self.nn, self.nslot, self.nsmax
        t = dict(flipr=np.zeros((nsm, nn), np.int32, order="F"), flipg=np.zeros((nsm, nn), np.int32, order="F"),
                 hopr=np.zeros((ns, nn), np.int32, order="F"), hopg=np.zeros((ns, nn), np.int32, order="F"),
                 lst=np.zeros(nn, np.int32), site=np.zeros(nn, np.int32), ncl=np.zeros(nn, np.int32),
                 level=np.zeros(nn, np.int32), norb=np.zeros(nn), sq=np.zeros(nn), stab_ptr=np.zeros(nn + 1, np.int32),
                 stab=np.zeros(max(self.nstab, 1), np.int32))
        check(lib().asr_op_export_tables(self.h, *[_pi(t[k]) for k in ("flipr", "flipg", "hopr", "hopg", "lst", "site", "ncl",
                                                                        "level")],
                                         _pd(t["norb"]), _pd(t["sq"]), _pi(t["stab_ptr"]), _pi(t["stab"])))
        t["stab"] = t["stab"][: self.nstab]
        return t

    # ---- state
    def set_params(self, c, d, o, e):
        """``augcls_set_params``: species parameters (9, nsp) of H = E_nu + h - h o h, h = c + d S d."""
        args = [_f64(x) for x in (c, d, o, e)]
        for a in args:
            if a.shape != (9, self.nsp):
                raise ValueError("augcls_set_params: number of species changed")
        check(lib().asr_op_set_params(self.h, *[_pd(a) for a in args]))
        self.params = dict(c=args[0], d=args[1], o=args[2], e=args[3])

    def freeze_site(self, site: int, sp: int):
        """``augcls_freeze_site`` (src/asr_augcls.f90:129-142): freeze the (non-flippable) site to species sp of its
        class; at the start site sp must belong to the start node's class."""
        check(lib().asr_op_freeze_site(self.h, site, sp))

    def freeze_any(self, site: int, sp: int) -> int:
        """``augcls_freeze_any`` (src/asr_augcls.f90:147-161): freeze the site to any species index 1..nsp (a path species,
        the partner of a pair); returns the number of nodes on the site (0: outside the node set)."""
        n = C.c_int(0)
        check(lib().asr_op_freeze_any(self.h, site, sp, C.byref(n)))
        return n.value

    def hp_c(self, x):
        """``augcls_hp_c`` (src/asr_augcls.f90:301-320): h x = (c + D S D) x for complex x (dim,) or (dim, nvec) in
        normalised coordinates."""
        x = np.asarray(x, np.complex128)
        one = x.ndim == 1
        xs = np.asfortranarray(x.reshape(self.dim, -1))
        y = np.zeros_like(xs, order="F")
        check(lib().asr_op_hp_c(self.h, _pd(xs), _pd(y), xs.shape[1]))
        return y[:, 0] if one else y

    def unfreeze(self):
        check(lib().asr_op_unfreeze(self.h))

    def set_start(self, l0: int):
        """``augcls_set_start``: chi(g) = D(g)[l0, l0]."""
        check(lib().asr_op_set_start(self.h, l0))

    def set_chi(self, chi):
        check(lib().asr_op_set_chi(self.h, _pd(_f64(chi))))

    def set_class_conc(self, kap: int, conc):
        check(lib().asr_op_set_class_conc(self.h, kap, _pd(_f64(conc))))

    # ---- application (linop interface)
    def apply(self, x):
        """y = H x, real, normalised coordinates; x of shape (9 nn,) or (9 nn, nvec)."""
        x = _f64(x)
        one = x.ndim == 1
        X = x.reshape(self.dim, -1, order="F")
        Y = np.zeros_like(X, order="F")
        check(lib().asr_op_apply(self.h, _pd(X), _pd(Y), X.shape[1]))
        return Y[:, 0] if one else Y

    def rand_c(self, par, x):
        """``augcls_rand_c``: w = X x with complex parameters par (9, nsp)."""
        par = _f64(par, True)
        x = _f64(x, True)
        one = x.ndim == 1
        X = x.reshape(self.dim, -1, order="F")
        W = np.zeros_like(X, order="F")
        check(lib().asr_op_rand_c(self.h, _pd(par), _pd(X), _pd(W),
                                  X.shape[1]))
        return W[:, 0] if one else W

    def project_c(self, x):
        """``augcls_project_c`` (returns the projected copy)."""
        X = _f64(x, True).reshape(self.dim, -1, order="F").copy(order="F")
        one = np.ndim(x) == 1
        check(lib().asr_op_project_c(self.h, _pd(X), X.shape[1]))
        return X[:, 0] if one else X


def build_augcls_operator(g, mdl, cls, perm, dmat, start: int, maxlevel: int, maxrank: int | None = None, flippable=None,
                          stype=None, ctx: Context | None = None, tsite=None):
    """``build_augcls_operator`` (src/asr_augcls.f90:596-823) on the GPU.

    g: ``Graph`` (1-based CSR); mdl: ``ClassModel`` (nsc, spc, conc, block, block0, nsp); cls (nsite); perm (nsite, nop);
    dmat (9, 9, nop); flippable (nsite, bool) and stype (nsite) optional.  With ``tsite`` (target graph sites, 1-based)
    returns (op, tnode, tgop): tnode (nsmax, nt) the node of each target alone in local state k (1-based, 0: none) and
    tgop (nsmax, nt) the operation mapping it onto that node (1-based), as the reference's optional outputs (:808-820)."""
    ctx = ctx or default_context()
    nbr_ptr, nbr = _i32(g.nbr_ptr), _i32(g.nbr)
    nsc, spc, conc = _i32(mdl.nsc), _i32(mdl.spc), _f64(mdl.conc)
    cls, perm, dmat = _i32(cls), _i32(perm), _f64(dmat)
    fl = _i32(np.asarray(flippable).astype(np.int32)) if flippable is not None else None
    st = _i32(stype) if stype is not None else None
    block = _f64(mdl.block)
    if block.ndim == 3:
        block = np.asfortranarray(block.reshape(9, 9, block.shape[2], 1))
    block0 = _f64(mdl.block0) if mdl.block0 is not None else None
    if block0 is not None and block0.ndim == 2:
        block0 = np.asfortranarray(block0.reshape(9, 9, 1))
    h = C.c_void_p()
    args = (ctx.h, g.n, _pi(nbr_ptr), _pi(nbr), int(nsc.shape[0]), _pi(nsc), _pi(spc), spc.shape[0], _pd(conc), mdl.nsp, _pi(cls),
            _pi(perm), perm.shape[1], _pd(dmat), start, maxlevel, int(maxrank or 0), _pi(fl), _pi(st), _pd(block), block.shape[2],
            block.shape[3], _pd(block0))
    if tsite is None:
        check(lib().asr_op_build(*args, C.byref(h)))
        return AugclsOp(ctx, h, mdl.nsp)
    ts = _i32(np.atleast_1d(tsite))
    nsm = int(np.max(nsc))
    tnode = np.zeros((nsm, ts.shape[0]), np.int32, order="F")
    tgop = np.zeros((nsm, ts.shape[0]), np.int32, order="F")
    check(lib().asr_op_build_targets(*args, _pi(ts), ts.shape[0], _pi(tnode), _pi(tgop), C.byref(h)))
    return AugclsOp(ctx, h, mdl.nsp), tnode, tgop
