"""Batched recursion chains and continued fractions on the GPU.

* ``chains_run`` -- the batched chain scheduler (``chain_greens`` / ``chain_worker``, src/asr_class_scf.f90:966-1160):
  every (group, energy) chain of the energy-dependent route, or one real chain per group in the plain route, in lanes of
  32 chains per tile;
* ``edc_green_blk`` -- ``edc_green_blk`` (src/asr_edc.f90:237-316) on the operator's current parameters;
* ``chains_proj`` / ``edc_green_proj`` -- ``edc_green_proj`` (src/asr_edc.f90:174-232): the chains with their
  first-order projections on target states (off-site elements for the Bloch spectral function);
* ``lanczos`` -- the plain real chain (src/reference/asr_recursion.f90:17-58) on ``augcls_apply``;
* ``cf_species`` -- terminated continued fractions (src/asr_chain.f90:67-167) for many (chain, energy) pairs.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check, lib
from .augcls import AugclsOp, Context, default_context, _f64, _pd, _pi

PREC = {"fp64": _lib.FP64, "fp32": _lib.FP32}


@dataclass
class ChainSpec:
    """One chain group (``asr_chain_group``): the operator parameters of the chain (9, nsp each), the energy-dependent
    diagonal X(z) = z pa + pb (edc route), the species frozen on the start site, the start orbital and the depth."""
    c: np.ndarray
    d: np.ndarray
    o: np.ndarray
    e: np.ndarray
    pa: np.ndarray | None = None
    pb: np.ndarray | None = None
    frozen_sp: int = 0
    start_orb: int = 1
    nlev: int = 16


def _groups(specs):
    arr = (_lib.ChainGroup * len(specs))()
    keep = []
    for q, s in enumerate(specs):
        vals = {}
        for k in ("c", "d", "o", "e", "pa", "pb"):
            v = getattr(s, k)
            if v is None:
                vals[k] = None
            else:
                a = _f64(v)
                keep.append(a)
                vals[k] = _pd(a)
        arr[q] = _lib.ChainGroup(vals["c"], vals["d"], vals["o"], vals["e"], vals["pa"], vals["pb"], int(s.frozen_sp),
                                 int(s.start_orb), int(s.nlev), 0)
    return arr, keep


def chains_run(op: AugclsOp, specs, z, mode: str = "edc", depth_tol: float = 0.0, tail: str = "hull", precision: str = "fp64",
               project: bool = True, coefs: bool = False):
    """Run every chain; returns dict(g=(nz, ngroup) complex, m=(nz, ngroup), a, b=(nlevmax, nz, ngroup) if coefs).

    mode 'edc': one complex-symmetric chain per (group, energy); mode 'plain': one real chain per group, whose terminated
    fraction (tail 'bp': Beer-Pettifor, 'avg2', 'none', 'hull') is evaluated at every energy."""
    z = np.ascontiguousarray(np.atleast_1d(z), dtype=np.complex128)
    nz = z.shape[0]
    ng = len(specs)
    nlevmax = max(s.nlev for s in specs)
    arr, keep = _groups(specs)
    g = np.zeros((ng, nz), np.complex128)
    m = np.zeros((ng, nz), np.int32)
    nab = 1 if mode == "plain" else nz
    a = np.zeros((ng, nab, nlevmax), np.complex128) if coefs else None
    b = np.zeros((ng, nab, nlevmax), np.complex128) if coefs else None
    check(lib().asr_chains_run(op.ctx.h, op.h, arr, ng, _pd(z), nz,
                               _lib.MODE_PLAIN if mode == "plain" else _lib.MODE_EDC, float(depth_tol), _lib.TAILS[tail],
                               PREC[precision], int(bool(project)), _pd(g),
                               _pd(a) if coefs else None, _pd(b) if coefs else None, _pi(m)))
    out = dict(g=g.T, m=m.T)
    if coefs:
        out["a"] = a.transpose(2, 1, 0)
        out["b"] = b.transpose(2, 1, 0)
    return out


def chains_adjoint(op: AugclsOp, specs, z, w, tail: str = "hull", precision: str = "fp64", project: bool = True,
                   stride: int = 0):
    """Reverse mode of the energy-dependent chains (o = 0, fixed depth): returns (g (nz, ngroup), grad) where
    grad[q, kind, s, l] = sum_j w[j, q] dG[j, q] / dpar_kind(l, s) of group q, kind 0: c (equally e and pb, which enter
    as c + e + pb), 1: d, 2: pa.  w (nz, ngroup) complex seeds.  stride > 0: Lanczos vectors kept every ``stride``
    levels and recomputed in between; 0: every level kept when it fits in half the free device memory, else every
    ceil(sqrt(depth)) levels (the same G; the same gradient to rounding, bitwise on the operators of the stride tests)."""
    z = np.ascontiguousarray(np.atleast_1d(z), dtype=np.complex128)
    nz = z.shape[0]
    ng = len(specs)
    w = np.asarray(w, np.complex128).reshape(nz, ng)
    wl = np.ascontiguousarray(w.T)                       # lane order (group, energy)
    arr, keep = _groups(specs)
    g = np.zeros((ng, nz), np.complex128)
    grad = np.zeros((ng, 3, op.nsp, 9), np.complex128)
    check(lib().asr_chains_adjoint(op.ctx.h, op.h, arr, ng, _pd(z), nz, _pd(wl), _lib.TAILS[tail], PREC[precision],
                                   int(bool(project)), int(stride), _pd(g), _pd(grad)))
    return g.T, grad


KINDS_EXT = ("c", "d", "pa", "o", "e")


def chains_adjoint_ext(op: AugclsOp, specs, z, w, depth_tol: float = 0.0, tail: str = "hull", precision: str = "fp64",
                       project: bool = True, stride: int = 0):
    """Reverse mode of the energy-dependent chains on the whole operator form H = E_nu + h - h o h + X(z) (o != 0 allowed),
    with the depth test of src/asr_edc.f90:121-127 when depth_tol > 0 (the derivative at the depth each chain stopped at)
    and every tail.  Returns (g (nz, ngroup), m (nz, ngroup), grad) with grad[q, kind, s, l] = sum_j w[j, q]
    dG[j, q] / dpar_kind(l, s), kinds ``KINDS_EXT`` = c, d, pa, o, e (pb enters as e does)."""
    z = np.ascontiguousarray(np.atleast_1d(z), dtype=np.complex128)
    nz = z.shape[0]
    ng = len(specs)
    w = np.asarray(w, np.complex128).reshape(nz, ng)
    wl = np.ascontiguousarray(w.T)
    arr, keep = _groups(specs)
    g = np.zeros((ng, nz), np.complex128)
    m = np.zeros((ng, nz), np.int32)
    grad = np.zeros((ng, 5, op.nsp, 9), np.complex128)
    check(lib().asr_chains_adjoint_ext(op.ctx.h, op.h, arr, ng, _pd(z), nz, _pd(wl), float(depth_tol), _lib.TAILS[tail],
                                       PREC[precision], int(bool(project)), int(stride), _pd(g), _pi(m), _pd(grad)))
    return g.T, m.T, grad


def ed3_blocks(op: AugclsOp, groups, z, depth_tol: float = 0.0, tail: str = "hull", precision: str = "fp64",
               project: bool = True, coefs: bool = False):
    """``ed3_blocks`` (src/asr_ed3.f90:242-265) for every group at every energy.  groups: dicts with g, d, o, p, dl, enu
    ((9, nsp) each), dc (9), central, start_orb, nlev (``synthetic.ed3_params`` builds them).  Returns dict(bk=(4, nz, ngroup)
    complex: G_11, (hG)_11, (hGh)_11, q1 mismatch; m=(2, nz, ngroup) depths of the |a> and |v> chains; a, b, c =
    (nlevmax, 2, nz, ngroup) if coefs)."""
    z = np.ascontiguousarray(np.atleast_1d(z), dtype=np.complex128)
    nz, ng = z.shape[0], len(groups)
    arr = (_lib.Ed3Group * ng)()
    keep = []
    for q, gr in enumerate(groups):
        vals = {}
        for k in ("g", "d", "dc", "dl", "enu", "o", "p"):
            a = _f64(gr[k])
            keep.append(a)
            vals[k] = _pd(a)
        arr[q] = _lib.Ed3Group(vals["g"], vals["d"], vals["dc"], vals["dl"], vals["enu"], vals["o"], vals["p"], int(gr["central"]),
                               int(gr["start_orb"]), int(gr["nlev"]), 0)
    nlevmax = max(int(gr["nlev"]) for gr in groups)
    bk = np.zeros((ng, nz, 4), np.complex128)
    m = np.zeros((ng, nz, 2), np.int32)
    cf = [np.zeros((ng, nz, 2, nlevmax), np.complex128) for _ in range(3)] if coefs else [None] * 3
    check(lib().asr_ed3_blocks(op.ctx.h, op.h, arr, ng, _pd(z), nz, float(depth_tol), _lib.TAILS[tail], PREC[precision],
                               int(bool(project)), _pd(bk), _pi(m), *[_pd(x) if x is not None else None for x in cf]))
    out = dict(bk=bk.transpose(2, 1, 0), m=m.transpose(2, 1, 0))
    if coefs:
        out["a"], out["b"], out["c"] = (x.transpose(3, 2, 1, 0) for x in cf)
    return out


def dos_final(op: AugclsOp, specs, comp, spin, lorb, worb, ncomp: int, nspin: int, emin: float, emax: float, eta: float,
              ndos: int, depth_tol: float = 0.0, tail: str = "hull", precision: str = "fp64"):
    """``dos_final`` (src/asr_class_scf.f90:1912-1931): the l-resolved DOS at ndos uniform real energies on [emin, emax]
    (Im z = eta) from the chains of every group.  comp, spin (1-based) and lorb (0 s, 1 p, 2 d) per group, worb the
    orbital-group size of its start orbital.  Returns (e (ndos,), edos (ndos, 3, ncomp, nspin))."""
    ng = len(specs)
    arr, keep = _groups(specs)
    comp, spin, lorb = (np.ascontiguousarray(x, np.int32) for x in (comp, spin, lorb))
    worb = np.ascontiguousarray(worb, np.float64)
    if not (comp.size == spin.size == lorb.size == worb.size == ng):
        raise ValueError("dos_final: one component, spin, l and weight per group")
    e = np.zeros(ndos)
    edos = np.zeros((ndos, 3, ncomp, nspin), order="F")
    check(lib().asr_dos_final(op.ctx.h, op.h, arr, ng, _pi(comp), _pi(spin), _pi(lorb), _pd(worb), int(ncomp), int(nspin),
                              float(emin), float(emax), float(eta), int(ndos), float(depth_tol), _lib.TAILS[tail],
                              PREC[precision], _pd(e), _pd(edos)))
    return e, edos


def chains_run_lanes(op: AugclsOp, specs, lane_group, lane_z, depth_tol: float = 0.0, tail: str = "hull",
                     precision: str = "fp64", project: bool = True):
    """The tasks of ``chain_worker`` (src/asr_class_scf.f90:1071-1160) as explicit lanes of the edc route: lane L runs
    group lane_group[L] (0-based) at energy lane_z[L].  Returns (g (nlane,), m (nlane,)), bitwise those of ``chains_run``
    for the same (group, energy)."""
    lg = np.ascontiguousarray(np.asarray(lane_group, np.int64) + 1, np.int32)
    lz = np.ascontiguousarray(lane_z, np.complex128)
    if lg.shape != lz.shape or lg.ndim != 1:
        raise ValueError("chains_run_lanes: one group and one energy per lane")
    arr, keep = _groups(specs)
    g = np.zeros(lz.shape[0], np.complex128)
    m = np.zeros(lz.shape[0], np.int32)
    check(lib().asr_chains_run_lanes(op.ctx.h, op.h, arr, len(specs), _pi(lg), _pd(lz), lz.shape[0], float(depth_tol),
                                     _lib.TAILS[tail], PREC[precision], int(bool(project)), _pd(g), _pi(m)))
    return g, m


def chains_run_lanes_device(op: AugclsOp, specs, lane_group, z_dev, g_dev, depth_tol: float = 0.0, tail: str = "hull",
                            precision: str = "fp64", project: bool = True):
    """Device-resident ``chains_run_lanes``: z_dev / g_dev device pointers (ints) of complex128 arrays of one entry per lane;
    lane_group (0-based) on the host."""
    lg = np.ascontiguousarray(np.asarray(lane_group, np.int64) + 1, np.int32)
    arr, keep = _groups(specs)
    check(lib().asr_chains_run_lanes_dev(op.ctx.h, op.h, arr, len(specs), _pi(lg), C.c_void_p(z_dev), lg.shape[0],
                                         float(depth_tol), _lib.TAILS[tail], PREC[precision], int(bool(project)),
                                         C.c_void_p(g_dev)))


def chains_run_device(op: AugclsOp, specs, z_dev, g_dev, nz: int, mode: str = "edc", depth_tol: float = 0.0, tail: str = "hull",
                      precision: str = "fp64", project: bool = True):
    """Device-resident form: z_dev / g_dev are device pointers (ints, e.g. torch tensor data_ptr()) of complex128 arrays;
    g_dev receives (ngroup, nz) in row-major order (lane order)."""
    arr, keep = _groups(specs)
    check(lib().asr_chains_run_dev(op.ctx.h, op.h, arr, len(specs), C.c_void_p(z_dev), nz,
                                   _lib.MODE_PLAIN if mode == "plain" else _lib.MODE_EDC, float(depth_tol), _lib.TAILS[tail],
                                   PREC[precision], int(bool(project)), C.c_void_p(g_dev), None, None, None))


def edc_green_blk(op: AugclsOp, ed: dict, zs, iv: int, nlev: int, depth_tol: float = 0.0, tail: str = "hull",
                  precision: str = "fp64", project: bool = True):
    """``edc_green_blk`` (src/asr_edc.f90:237-316) on the operator's current parameters (set_params / freeze_site /
    set_start): ed holds dc (9), dl (9, nsp), enu (9, nsp).  Returns (g(nb), mused(nb), a(nlev, nb), b(nlev, nb))."""
    if not 1 <= iv <= 9:
        raise ValueError("edc_green_blk: the start component must lie on node 1")
    dc = np.asarray(ed["dc"], float)
    dl = np.asarray(ed["dl"], float)
    en = np.asarray(ed["enu"], float)
    pa = np.asfortranarray(1.0 - dc[:, None] / dl)
    pb = np.asfortranarray(dc[:, None] * en / dl)
    p = op.params
    spec = ChainSpec(c=p["c"], d=p["d"], o=p["o"], e=p["e"], pa=pa, pb=pb, frozen_sp=0, start_orb=iv, nlev=nlev)
    r = chains_run(op, [spec], zs, "edc", depth_tol, tail, precision, project, coefs=True)
    return r["g"][:, 0], r["m"][:, 0], r["a"][:, :, 0], r["b"][:, :, 0]


def chains_proj(op: AugclsOp, specs, z, tnode, tgop, tw, tail: str = "hull", precision: str = "fp64", project: bool = True):
    """``edc_green_proj`` (src/asr_edc.f90:174-232) for every (group, energy): each chain runs its full depth and its
    Lanczos vectors are projected on the target states.  tnode, tgop (nsmax, nt) from ``build_augcls_operator(...,
    tsite=...)``; tw (9, nsmax, nt) or (9, nsmax, nt, ngroup) dressing weights.  Returns dict(g (nz, ngroup), gp, gp4
    (9, nt, nz, ngroup), m (nz, ngroup)); gp4 uses the chain cut four steps earlier."""
    z = np.ascontiguousarray(np.atleast_1d(z), dtype=np.complex128)
    nz, ng = z.shape[0], len(specs)
    tnode = np.asfortranarray(tnode, dtype=np.int32)
    tgop = np.asfortranarray(tgop, dtype=np.int32)
    nsm, nt = tnode.shape
    tw = np.asarray(tw, dtype=np.float64)
    if tw.ndim == 3:
        tw = np.repeat(tw[..., None], ng, axis=3)
    if tw.shape != (9, nsm, nt, ng):
        raise ValueError(f"chains_proj: tw must be (9, {nsm}, {nt}[, {ng}]), got {tw.shape}")
    tw = np.asfortranarray(tw)
    arr, keep = _groups(specs)
    g = np.zeros((ng, nz), np.complex128)
    gp = np.zeros((ng, nz, nt, 9), np.complex128)
    gp4 = np.zeros((ng, nz, nt, 9), np.complex128)
    m = np.zeros((ng, nz), np.int32)
    check(lib().asr_chains_proj(op.ctx.h, op.h, arr, ng, _pd(z), nz, _lib.TAILS[tail], PREC[precision], int(bool(project)), nt,
                                _pi(tnode), _pi(tgop), _pd(tw), _pd(g), _pd(gp), _pd(gp4), _pi(m)))
    return dict(g=g.T, gp=gp.transpose(3, 2, 1, 0), gp4=gp4.transpose(3, 2, 1, 0), m=m.T)


def edc_green_proj(op: AugclsOp, ed: dict, z, iv: int, nlev: int, tnode, tgop, tw, tail: str = "hull", precision: str = "fp64",
                   project: bool = True):
    """``edc_green_proj`` (src/asr_edc.f90:174-232) at one energy on the operator's current parameters (as
    ``edc_green_blk``): returns (g, gp (9, nt), gp4 (9, nt))."""
    dc = np.asarray(ed["dc"], float)
    dl = np.asarray(ed["dl"], float)
    en = np.asarray(ed["enu"], float)
    p = op.params
    spec = ChainSpec(c=p["c"], d=p["d"], o=p["o"], e=p["e"], pa=np.asfortranarray(1.0 - dc[:, None] / dl),
                     pb=np.asfortranarray(dc[:, None] * en / dl), frozen_sp=0, start_orb=iv, nlev=nlev)
    r = chains_proj(op, [spec], np.atleast_1d(z), tnode, tgop, tw, tail, precision, project)
    return r["g"][0, 0], r["gp"][:, :, 0, 0], r["gp4"][:, :, 0, 0]


def autotune(op: AugclsOp, specs, z, precision: str = "fp64", levels: int = 8) -> dict:
    """Choose the batch shape (tiles per batch, nodes per warp) of the chains on this operator by timing the given groups
    (depth capped at ``levels``, at most 64 energies); a candidate must beat the built-in default by 3 %.  Later calls in
    this precision use the choice; at that shape the step kernel with fixed-offset link gathers (the same bits) is kept
    when it is 3 % faster than the general one.  Returns dict(tiles_per_batch, nodes_per_warp, ms_tiles (4, 8, 16, 32
    tiles at 4 nodes per warp), ms_npw (1, 2, 4, 8 nodes per warp), link_gather ("fixed-offset" or "general"),
    ms_link (general, fixed-offset step at the chosen shape))."""
    z = np.ascontiguousarray(np.atleast_1d(z), dtype=np.complex128)
    arr, keep = _groups(specs)
    tpb, npw = C.c_int(), C.c_int()
    times = np.zeros(8)
    check(lib().asr_autotune(op.ctx.h, op.h, arr, len(specs), _pd(z), z.shape[0], PREC[precision], int(levels), C.byref(tpb),
                             C.byref(npw), _pd(times)))
    st = tuning(op, precision)
    return dict(tiles_per_batch=tpb.value, nodes_per_warp=npw.value, ms_tiles=times[:4].tolist(), ms_npw=times[4:].tolist(),
                link_gather=st["link_gather"], ms_link=st["ms_link"])


def tuning(op: AugclsOp, precision: str = "fp64") -> dict:
    """The operator's tuned state in this precision (``asr_op_tuning``): tiles_per_batch and nodes_per_warp (0: never
    tuned), link_gather, ms_link."""
    tpb, npw, link = C.c_int(), C.c_int(), C.c_int()
    ms = np.zeros(2)
    check(lib().asr_op_tuning(op.h, PREC[precision], C.byref(tpb), C.byref(npw), C.byref(link), _pd(ms)))
    return dict(tiles_per_batch=tpb.value, nodes_per_warp=npw.value,
                link_gather="fixed-offset" if link.value == 1 else "general", ms_link=ms.tolist())


def set_tuning(op: AugclsOp, precision: str = "fp64", tiles_per_batch: int = 0, nodes_per_warp: int = 0,
               link_gather: str = "general"):
    """Pin the tuned state in this precision (``asr_op_set_tuning``): 0 restores the built-in shape defaults;
    link_gather "general" or "fixed-offset" (the same results)."""
    if link_gather not in ("general", "fixed-offset"):
        raise ValueError(link_gather)
    check(lib().asr_op_set_tuning(op.h, PREC[precision], int(tiles_per_batch), int(nodes_per_warp),
                                  1 if link_gather == "fixed-offset" else 0))


def lanczos(op: AugclsOp, l0: int, nmax: int, precision: str = "fp64"):
    """Reference ``lanczos`` (src/reference/asr_recursion.f90:17-58) from e_(node 1, l0) on the operator's parameters.
    Returns (a(nmax), b(nmax), n) with b(n) of the last step."""
    p = op.params
    spec = ChainSpec(c=p["c"], d=p["d"], o=p["o"], e=p["e"], start_orb=l0, nlev=nmax)
    r = chains_run(op, [spec], np.zeros(1, complex), "plain", 0.0, "none", precision, project=False, coefs=True)
    n = int(r["m"][0, 0])
    return r["a"][:, 0, 0].real.copy(), r["b"][:, 0, 0].real.copy(), n


def cf_species(a, b, m, z, tail: str = "hull", ctx: Context | None = None, edges: bool = False):
    """``cf_species`` for chains a, b (ld, nchain) complex of depths m (nchain) at energies z (nz, nchain) -> g (nz, nchain)."""
    ctx = ctx or default_context()
    a = np.asfortranarray(np.asarray(a, np.complex128))
    b = np.asfortranarray(np.asarray(b, np.complex128))
    if a.ndim == 1:
        a = a.reshape(-1, 1, order="F")
        b = b.reshape(-1, 1, order="F")
    ld, nc = a.shape
    if b.shape[0] < ld:
        b = np.asfortranarray(np.vstack([b, np.zeros((ld - b.shape[0], nc))]))
    m = np.ascontiguousarray(np.broadcast_to(np.asarray(m, np.int32), (nc,)))
    z = np.asfortranarray(np.asarray(z, np.complex128).reshape(-1, nc) if np.ndim(z) else np.full((1, nc), z))
    if z.shape[1] != nc:
        z = np.asfortranarray(np.repeat(z.reshape(-1, 1), nc, axis=1))
    nz = z.shape[0]
    g = np.zeros((nz, nc), np.complex128, order="F")
    e = np.zeros((2, nz, nc), np.complex128, order="F") if edges else None
    nf = C.c_int64(0)
    check(lib().asr_cf_eval(ctx.h, _pd(a), _pd(b), _pi(m), ld, nc, _pd(z), nz,
                            _lib.TAILS[tail], _pd(g), _pd(e) if edges else None, C.byref(nf)))
    return (g, e, nf.value) if edges else g
