"""Effective pair interactions from the recursion: the block chains on the device and the host-side thermodynamic
integration around them.

Host-side restatement of the reference's ``asr_epi`` (src/asr_epi.f90) for the edc route:

* ``EpiPar`` / ``epi_path`` / ``epi_setup`` (:80-178): species parameters (E_nu, c = C - E_nu, d = |sqrt(Delta)|, o) per
  orbital, the straight path of site 0 between two species with its lambda-derivatives, and the scaled operator
  parameters (c = (D_c / D_s) c_s, d = D_c^1/2, o = o_s D_s / D_c, e = 0; the path point is species ns + 1) with the
  energy-dependent diagonal e_s(z) = z - D_c (z - E_nu,s) / D_s;
* ``epi_integrand`` (:182-189): [G dH/dlambda]_LL from the central blocks X0, X1, X2 (the constant -2 kappa left out);
* ``epi_adapted`` (:290-328): symmetry-adapted start vectors of an abelian group of involutions;
* ``epi_pair_ops`` (:333-363): the pair group (class-preserving D4h about z, reduced to an abelian group of involutions);
* ``epi_exchange``, ``epi_skip``, ``epi_mirror`` (:257-285);
* ``epi_pair_list`` / ``epi_pair_ops_c`` / ``epi_pair_list_c`` (:365-568): the pair types of the first shells of the
  origin (orbits of the class-preserving operations, representative with the largest pair group), on periodic cubic
  cells and on site clusters;
* ``epi_blocks`` -- the two projected chains per start vector and energy on the device (``asr_epi_blocks``);
* ``pair_table`` -- U(c, s) = int_0^1 dlambda [dOmega/dlambda (c0 -> c | s) - dOmega/dlambda (c0 -> c | s0)] with
  Gauss-Legendre nodes in lambda and dOmega/dlambda = -(1/pi) Im sum_j w_j sum_a epi_integrand (the contour weights w_j).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check, lib
from .augcls import AugclsOp, _pd, _pi
from .chains import PREC, ChainSpec, _groups
from .crystal import is_monomial
from .lattices import class_ops, cubic_site_perms

__all__ = ["EpiPar", "EpiPath", "epi_path", "epi_setup", "epi_integrand", "epi_adapted", "epi_pair_ops", "epi_exchange",
           "epi_skip", "epi_mirror", "EpiPair", "epi_pair_list", "epi_pair_ops_c", "epi_pair_list_c", "epi_blocks", "trace_at",
           "pair_table"]

ORB_L = np.array([0, 1, 1, 1, 2, 2, 2, 2, 2])


@dataclass
class EpiPar:
    """One species per orbital: E_nu, c = C - E_nu, d = |sqrt(Delta)|, o (each (9,))."""
    e: np.ndarray
    c: np.ndarray
    d: np.ndarray
    o: np.ndarray


@dataclass
class EpiPath:
    """Site 0 at lambda on the path: parameters and their lambda-derivatives (dk = d(ln d)/dlambda)."""
    e: np.ndarray
    c: np.ndarray
    d: np.ndarray
    o: np.ndarray
    de: np.ndarray
    dc: np.ndarray
    dk: np.ndarray
    dox: np.ndarray


def epi_path(a: EpiPar, b: EpiPar, lam: float) -> EpiPath:
    """The straight path from species a (lambda = 0) to species b (lambda = 1)."""
    d = a.d + lam * (b.d - a.d)
    return EpiPath(e=a.e + lam * (b.e - a.e), c=a.c + lam * (b.c - a.c), d=d, o=a.o + lam * (b.o - a.o),
                   de=b.e - a.e, dc=b.c - a.c, dk=(b.d - a.d) / d, dox=b.o - a.o)


def epi_setup(par: list[EpiPar], pt: EpiPath):
    """Scaled operator parameters for species 1..ns (par) and the path point as species ns + 1: returns (c, d, o, e) each
    (9, ns + 1) Fortran and the edc parameters dict(dc (9), dl (9, ns + 1), enu (9, ns + 1), pa, pb)."""
    ns = len(par)
    dc = pt.d ** 2
    c = np.zeros((9, ns + 1), order="F")
    d = np.zeros((9, ns + 1), order="F")
    o = np.zeros((9, ns + 1), order="F")
    dl = np.zeros((9, ns + 1), order="F")
    enu = np.zeros((9, ns + 1), order="F")
    for s, p in enumerate(par):
        ds = p.d ** 2
        c[:, s] = dc / ds * p.c
        d[:, s] = pt.d
        o[:, s] = p.o * ds / dc
        dl[:, s] = ds
        enu[:, s] = p.e
    c[:, ns], d[:, ns], o[:, ns] = pt.c, pt.d, pt.o
    dl[:, ns], enu[:, ns] = dc, pt.e
    e = np.zeros((9, ns + 1), order="F")
    pa = np.asfortranarray(1.0 - dc[:, None] / dl)
    pb = np.asfortranarray(dc[:, None] * enu / dl)
    return (c, d, o, e), dict(dc=dc, dl=dl, enu=enu, pa=pa, pb=pb)


def epi_integrand(pt: EpiPath, l: int, z: complex, x) -> complex:
    """[G dH/dlambda]_LL for a start vector of orbital character l (1-based orbital index) from X0, X1, X2 at z."""
    i = l - 1
    return ((pt.de[i] + pt.dc[i]) * x[0] - 2.0 * pt.dc[i] * pt.o[i] * x[1] - pt.dox[i] * x[2]
            + 2.0 * pt.dk[i] * ((z - pt.e[i] - pt.c[i]) * x[0] + 2.0 * pt.c[i] * pt.o[i] * x[1] - pt.o[i] * x[2]))


def epi_adapted(d: np.ndarray):
    """Start vectors vec (9, 9) (columns, orthonormal, each inside one l) with D(g) vec_a = chi(g, a) vec_a for an abelian
    group of involutions with orbital matrices d (9, 9, nop); lo (9) the first orbital index of each vector's l."""
    d = np.asarray(d, dtype=float)
    nop = d.shape[2]
    for g in range(nop):
        if np.max(np.abs(d[:, :, g] - d[:, :, g].T)) > 1e-9:
            raise ValueError("epi_adapted: an operation is not an involution (the group must be abelian, all of order 2)")
    vec = np.zeros((9, 9))
    lo = np.zeros(9, dtype=np.int64)
    for i1, i2 in ((0, 1), (1, 4), (4, 9)):
        m = np.zeros((i2 - i1, i2 - i1))
        for g in range(nop):      # a generic combination: one eigenvalue per character
            m += np.sqrt(g + 1 + 0.37) * d[i1:i2, i1:i2, g]
        m = 0.5 * (m + m.T)
        _, v = np.linalg.eigh(m)
        vec[i1:i2, i1:i2] = v
        lo[i1:i2] = i1 + 1
    chi = np.zeros((nop, 9))
    for a in range(9):
        v = vec[:, a]
        v[np.abs(v) < 1e-12] = 0.0
        k = int(np.argmax(np.abs(v)))
        if v[k] < 0:
            v = -v
        v = v / np.linalg.norm(v)
        vec[:, a] = v
        for g in range(nop):
            w = d[:, :, g] @ v
            x = float(v @ w)
            if abs(abs(x) - 1.0) > 1e-8 or np.max(np.abs(w - x * v)) > 1e-8:
                raise ValueError("epi_adapted: a start vector is not a common eigenvector of the group")
            chi[g, a] = np.sign(x)
    return vec, chi, lo


def epi_pair_ops(coord: np.ndarray, mg: int, cls):
    """The pair group: the operations of D4h about z that keep the classes (the partner carries a class of its own),
    reduced to the sign changes of the axes when they do not all commute (partner on the z axis).  Returns (perm, mats)."""
    p0, m0 = class_ops(coord, mg, cls)
    n = m0.shape[2]
    one = np.eye(3, dtype=np.int64)
    abel = True
    for i in range(n):
        if not np.array_equal(m0[:, :, i] @ m0[:, :, i], one):
            abel = False
        for j in range(i + 1, n):
            if not np.array_equal(m0[:, :, i] @ m0[:, :, j], m0[:, :, j] @ m0[:, :, i]):
                abel = False
    keep = [True] * n if abel else [bool(np.count_nonzero(m0[:, :, i] - np.diag(np.diag(m0[:, :, i]))) == 0) for i in range(n)]
    sel = [i for i in range(n) if keep[i]]
    return np.asfortranarray(p0[:, sel]), np.asfortranarray(m0[:, :, sel])


def epi_exchange(u: np.ndarray) -> np.ndarray:
    """V(p, q) = U(p, p) + U(q, q) - U(p, q) - U(q, p) of one sublattice."""
    u = np.asarray(u, dtype=float)
    dg = np.diag(u)
    return dg[:, None] + dg[None, :] - u - u.T


def epi_skip(sym: bool, same: bool, c: int, s: int) -> bool:
    """With the pair-exchange symmetry (one sublattice) the entries 1 < s < c (1-based) are not computed."""
    return sym and same and 1 < s < c


def epi_mirror(u: np.ndarray) -> np.ndarray:
    """Copy the entries above the diagonal into the skipped ones below it (columns 2 .. c - 1 of row c, 1-based)."""
    u = np.array(u, dtype=float)
    for c in range(2, u.shape[0]):
        for s in range(1, c):
            u[c, s] = u[s, c]
    return u


@dataclass
class EpiPair:
    """One pair type: shell (1-based), representative partner site (1-based), multiplicity, squared length (half-lattice
    units squared), partner class, order of its pair group, partner - origin vector (half-lattice units; Cartesian alat
    units in ``rvec``) and the vectors of every member (``orbit`` / ``rorbit``, columns)."""
    shell: int
    site: int
    mult: int
    r2: int
    cls2: int
    nop: int
    vec: np.ndarray
    orbit: np.ndarray
    rvec: np.ndarray | None = None
    rorbit: np.ndarray | None = None


def epi_pair_list(coord: np.ndarray, mg: int, cls, nshell: int) -> list[EpiPair]:
    """Pair types of the origin (site 1) with the sites of its first nshell shells on a periodic cubic cell (coordinates in
    half-lattice units, period mg): each shell splits into orbits of the class-preserving cubic operations; the
    representative is the member with the largest pair group.  A shell that does not fit into the cell raises ValueError."""
    coord = np.asarray(coord, dtype=np.int64)
    cls = np.asarray(cls, dtype=np.int64)
    n = coord.shape[1]
    v = (coord - coord[:, :1] + mg // 2) % mg - mg // 2
    r2 = np.sum(v * v, axis=0)
    shells, rcur = [], 0
    for ish in range(1, nshell + 1):
        rnext = int(np.min(r2[r2 > rcur]))
        if 4 * rnext >= mg * mg:
            raise ValueError(f"epi: shell {ish} does not fit into the supercell (increase the supercell)")
        shells.append(rnext)
        rcur = rnext
    p48, _ = cubic_site_perms(coord, mg)
    keep = [k for k in range(48) if np.array_equal(cls[p48[:, k] - 1], cls)]
    pairs, done = [], np.zeros(n, dtype=bool)
    for ish, sh in enumerate(shells, start=1):
        for i in range(1, n):
            if r2[i] != sh or done[i]:
                continue
            inorb = np.zeros(n, dtype=bool)
            inorb[p48[i, keep] - 1] = True
            done |= inorb
            best, site = 0, -1
            for j in np.nonzero(inorb)[0]:
                cl2 = cls.copy()
                cl2[j] = cls.max() + 1
                pp, _ = epi_pair_ops(coord, mg, cl2)
                if pp.shape[1] > best:
                    best, site = pp.shape[1], int(j)
            pairs.append(EpiPair(shell=ish, site=site + 1, mult=int(inorb.sum()), r2=int(sh), cls2=int(cls[site]), nop=best,
                                 vec=v[:, site].copy(), orbit=v[:, inorb].copy()))
    return pairs


def epi_pair_ops_c(perm: np.ndarray, rot: np.ndarray, cls) -> np.ndarray:
    """Pair group on a site cluster: of the site operations (identity first) the monomial ones that keep the z axis and
    the classes, reduced to the sign changes of the axes when they do not all commute.  Returns 0-based indices."""
    perm = np.asarray(perm)
    rot = np.asarray(rot, dtype=float)
    cls = np.asarray(cls)
    tol = 1e-9
    nk = perm.shape[1]
    keep = [bool(is_monomial(rot[:, :, k]) and abs(abs(rot[2, 2, k]) - 1.0) < tol and np.array_equal(cls[perm[:, k] - 1], cls))
            for k in range(nk)]
    sel = [k for k in range(nk) if keep[k]]
    one = np.eye(3)
    abel = all(np.max(np.abs(rot[:, :, i] @ rot[:, :, i] - one)) <= tol for i in sel) and all(
        np.max(np.abs(rot[:, :, i] @ rot[:, :, j] - rot[:, :, j] @ rot[:, :, i])) <= tol for a, i in enumerate(sel) for j in sel[a + 1:])
    if not abel:
        sel = [k for k in sel if np.max(np.abs(rot[:, :, k] - np.diag(np.diag(rot[:, :, k])))) < tol]
    if not sel or sel[0] != 0:
        raise RuntimeError("epi_pair_ops_c: operation 1 is not the identity")
    return np.array(sel, dtype=np.int64)


def _box_key(x: float) -> float:
    return x + 1.0e6 if x < -1.0e-7 else x


def _box_order(hv: np.ndarray) -> list[int]:
    """Indices in the order of a periodic box: by z, then y, then x, each component >= 0 increasing before the negative
    values increasing (a stable sort with a tolerance)."""
    import functools

    def cmp(a, b):
        for c in (2, 1, 0):
            ka, kb = _box_key(hv[c, a]), _box_key(hv[c, b])
            if ka < kb - 1.0e-7:
                return -1
            if ka > kb + 1.0e-7:
                return 1
        return 0
    return sorted(range(hv.shape[1]), key=functools.cmp_to_key(cmp))


def epi_pair_list_c(disp: np.ndarray, perm: np.ndarray, rot: np.ndarray, cls, nshell: int) -> list[EpiPair]:
    """``epi_pair_list`` on a site cluster (``crystal.crystal_graph`` + ``graph_site_ops``): disp (3, n) displacements from
    site 1 (alat units); members, orbits and ties follow the order of a periodic box.  A shell outside the cluster raises
    ValueError."""
    disp = np.asarray(disp, dtype=float)
    perm = np.asarray(perm)
    cls = np.asarray(cls, dtype=np.int64)
    tol = 1e-9
    n = disp.shape[1]
    r2 = np.sum(disp * disp, axis=0)
    h = np.rint(2.0 * disp).astype(np.int64)
    shells, rcur = [], 0.0
    for ish in range(1, nshell + 1):
        above = r2 > rcur + tol
        if not above.any():
            raise ValueError(f"epi: shell {ish} lies outside the site cluster (raise the levels)")
        rcur = float(np.min(r2[above]))
        shells.append(rcur)
    sub = np.nonzero(r2 <= rcur + tol)[0]
    ordr = [int(sub[q]) for q in _box_order(2.0 * disp[:, sub])]
    keep = [k for k in range(perm.shape[1]) if np.array_equal(cls[perm[:, k] - 1], cls)]
    pairs, done = [], np.zeros(n, dtype=bool)
    for ish, sh in enumerate(shells, start=1):
        for i in ordr:
            if i == 0 or abs(r2[i] - sh) > tol or done[i]:
                continue
            inorb = np.zeros(n, dtype=bool)
            inorb[perm[i, keep] - 1] = True
            done |= inorb
            best, site = 0, -1
            for j in ordr:
                if not inorb[j]:
                    continue
                cl2 = cls.copy()
                cl2[j] = cls.max() + 1
                nop = len(epi_pair_ops_c(perm, rot, cl2))
                if nop > best:
                    best, site = nop, j
            members = [j for j in ordr if inorb[j]]
            pairs.append(EpiPair(shell=ish, site=site + 1, mult=int(inorb.sum()), r2=int(round(4.0 * sh)), cls2=int(cls[site]),
                                 nop=best, vec=h[:, site].copy(), orbit=h[:, members].copy(), rvec=disp[:, site].copy(),
                                 rorbit=disp[:, members].copy()))
    return pairs


def epi_blocks(op: AugclsOp, params, ed: dict, vec: np.ndarray, chi: np.ndarray, lo, z, nlev: int, tail: str = "hull",
               precision: str = "fp64", project: bool = True):
    """The central blocks of every start vector at every energy (epi_start + epi_blocks, src/asr_epi.f90:578-663) on the
    device: params (c, d, o, e) and ed from ``epi_setup``; vec (9, na) start vectors with characters chi (nop, na) and
    orbital characters lo (na).  The operator carries the frozen path site and partner (``freeze_any``).  Returns
    x (4, nz, na) complex (X0, X1, X2, X1 mismatch) and the depths m (2, nz, na)."""
    c, d, o, e = params
    z = np.ascontiguousarray(np.atleast_1d(z), dtype=np.complex128)
    vec = np.asarray(vec, dtype=float)
    na, nz = vec.shape[1], z.shape[0]
    specs = [ChainSpec(c=c, d=d, o=o, e=e, pa=ed["pa"], pb=ed["pb"], frozen_sp=0, start_orb=int(lo[a]), nlev=nlev)
             for a in range(na)]
    arr, keep = _groups(specs)
    v9 = np.asfortranarray(vec)
    ch = np.asfortranarray(np.asarray(chi, dtype=float)[: op.nop, :na])
    x = np.zeros((na, nz, 4), np.complex128)
    m = np.zeros((na, nz, 2), np.int32)
    check(lib().asr_epi_blocks(op.ctx.h, op.h, arr, _pd(v9), _pd(ch), na, _pd(z), nz, _lib.TAILS[tail], PREC[precision],
                               int(bool(project)), _pd(x), _pi(m)))
    return x.transpose(2, 1, 0), m.transpose(2, 1, 0)


def trace_at(op: AugclsOp, par: list[EpiPar], a: int, b: int, lam: float, dmat: np.ndarray, z, nlev: int, tail: str = "hull",
             precision: str = "fp64", project: bool = True):
    """sum_a epi_integrand over the symmetry-adapted start vectors of the pair group (dmat) with site 0 on the path a -> b
    (1-based species) at lambda, at every energy z.  The operator is built for ns + 1 species with the path site and the
    partner frozen.  Returns (trace (nz,), largest relative X1 mismatch)."""
    pt = epi_path(par[a - 1], par[b - 1], lam)
    params, ed = epi_setup(par, pt)
    vec, chi, lo = epi_adapted(dmat)
    op.set_params(*params)
    x, _ = epi_blocks(op, params, ed, vec, chi, lo, z, nlev, tail, precision, project)
    z = np.atleast_1d(z)
    tr = np.zeros(z.shape[0], np.complex128)
    for ia in range(9):
        for j in range(z.shape[0]):
            tr[j] += epi_integrand(pt, int(lo[ia]), z[j], x[:, j, ia])
    mism = float(np.max(np.abs(x[3]) / np.maximum(np.abs(x[1]), 1e-300)))
    return tr, mism


def pair_table(op_for, par: list[EpiPar], spc_origin, spc_partner, dmat: np.ndarray, z, w, nlam: int, nlev: int,
               tail: str = "hull", precision: str = "fp64"):
    """U(c, s) (len(spc_origin) x len(spc_partner)) by thermodynamic integration: for every partner species s the
    operator ``op_for(s)`` (path site frozen to species ns + 1, partner to s), every origin species c != c0 and lambda at
    the Gauss-Legendre nodes, dOmega/dlambda (c0 -> c | s) = -(1/pi) Im sum_j w_j trace; U(c, s) = the lambda integral
    of dOmega/dlambda(c | s) - dOmega/dlambda(c | s0).  c0, s0 are the first entries of the lists (1-based species)."""
    xg, wg = np.polynomial.legendre.leggauss(nlam)
    lam, wl = 0.5 * (xg + 1.0), 0.5 * wg
    w = np.asarray(w, dtype=np.complex128)
    domega = np.zeros((len(spc_origin), len(spc_partner)))
    for js, s in enumerate(spc_partner):
        op = op_for(s)
        for ic, c in enumerate(spc_origin):
            if ic == 0:
                continue
            acc = 0.0
            for lq, wq in zip(lam, wl):
                tr, _ = trace_at(op, par, spc_origin[0], c, float(lq), dmat, z, nlev, tail, precision)
                acc += wq * (-np.imag(np.sum(w * tr)) / np.pi)
            domega[ic, js] = acc
    return domega - domega[:, :1]
