"""Configuration-averaged Bloch spectral function A(k, E) from the chains (route edc).

Host-side restatement of the caller of ``edc_green_proj`` in the reference's ``asr_spectral`` (src/asr_spectral.f90) and
``spectral_final`` (src/asr_class_scf.f90:1520-1800):

* ``spectral_kpath`` (:59-77), ``spectral_window`` (:175-188), ``spectral_unfold`` (:190-198), ``spectral_dressing``
  (:200-229) with ``augn_basis`` (src/asr_augcls.f90:73-91);
* ``spectral_structure_ok`` / ``spectral_origin_classes`` (:83-148): every sublattice one space-group orbit, and the
  basis sites grouped into origin classes by pure translations and inversions (with the sign of the mapping and the site
  fraction of each class);
* ``spectral_targets`` -- the targets of one origin class (src/asr_class_scf.f90:1562-1586): cluster sites within rmax,
  with the origin class and mapping sign of each target's basis site;
* ``spectral_sum_origins`` -- the Bloch sum over several origin classes (src/asr_class_scf.f90:1588-1601, 1693-1746):
  the partner of every target in the origin class of the target's own basis site (at -R, or +R through an inversion),
  the average with it, and the windowed sums weighted by the site fractions of the origin classes;
* ``bloch_spectral`` -- one origin class (a Bravais sublattice whose sites are related by translations or inversion):
  the D2h-reduced operator with the target sites within rmax, one projected chain per (spin, central component, start
  orbital, energy) on the device (``chains_proj``), the averaged off-site elements <G_{0L, RL}> = sum_c x_c gp, the
  average with the partner element at -R, and the windowed Bloch sum per l.

The chains run on the GPU through the C ABI; this module only sets up targets and weights and sums the results.
"""
from __future__ import annotations

import numpy as np

from .chains import ChainSpec, chains_proj

__all__ = ["spectral_kpath", "spectral_window", "spectral_unfold", "augn_basis", "spectral_dressing", "spectral_structure_ok",
           "spectral_origin_classes", "spectral_targets", "spectral_elements", "spectral_sum", "spectral_sum_origins",
           "bloch_spectral"]

ORB_L = np.array([0, 1, 1, 1, 2, 2, 2, 2, 2])


def spectral_kpath(kpts, nk: int):
    """k points along the corners kpts (3, nc) (units 2 pi / alat): nk points per segment, every corner once.  Returns
    (kv (3, n), dist (n) the path length, icorner (nc) 0-based indices of the corners)."""
    kpts = np.asarray(kpts, dtype=float).reshape(3, -1)
    nc = kpts.shape[1]
    ns = max(nc - 1, 0)
    n = ns * nk + 1
    kv = np.zeros((3, n))
    dist = np.zeros(n)
    icorner = np.zeros(nc, dtype=np.int64)
    kv[:, 0] = kpts[:, 0]
    q = 0
    for j in range(ns):
        for i in range(1, nk + 1):
            q += 1
            kv[:, q] = kpts[:, j] + (kpts[:, j + 1] - kpts[:, j]) * i / nk
            dist[q] = dist[q - 1] + np.linalg.norm(kv[:, q] - kv[:, q - 1])
        icorner[j + 1] = q
    return kv, dist, icorner


def spectral_window(kind: str, r: float, rmax: float) -> float:
    """Weight of a displacement of length r in the Fourier sum: 'ball' -- the overlap of two balls of diameter rmax at
    distance r over the volume of one, (1 - r/rmax)^2 (1 + r/(2 rmax)), whose lattice Fourier series is non-negative;
    'sharp' -- 1 up to rmax."""
    d = r / rmax
    if d > 1.0 + 1.0e-12:
        return 0.0
    if kind == "sharp":
        return 1.0
    d = min(d, 1.0)
    return (1.0 - d) ** 2 * (1.0 + 0.5 * d)


def spectral_unfold(disp, v, k) -> float:
    """sum_t cos(2 pi k . d_t) v_t: the unfolded Bloch sum of real-space values v (nt) at displacements disp (3, nt)."""
    disp = np.asarray(disp, dtype=float).reshape(3, -1)
    return float(np.sum(np.cos(2.0 * np.pi * (np.asarray(k, float) @ disp)) * np.asarray(v, dtype=float)))


def augn_basis(conc) -> np.ndarray:
    """phi (ns, ns): row l is the l-th orthonormal function of the species in <f, g> = sum_s x_s f(s) g(s), phi_0 = 1
    (Gram-Schmidt on the species indicators, twice for stability)."""
    conc = np.asarray(conc, dtype=float)
    ns = conc.shape[0]
    phi = np.zeros((ns, ns))
    phi[0] = 1.0
    for l in range(1, ns):
        phi[l] = 0.0
        phi[l, l - 1] = 1.0
        for _ in range(2):
            for m in range(l):
                phi[l] -= np.sum(conc * phi[m] * phi[l]) * phi[m]
        phi[l] /= np.sqrt(np.sum(conc * phi[l] ** 2))
    return phi


def spectral_dressing(dc, dl, spc, conc, frozen: bool, nsm: int | None = None) -> np.ndarray:
    """Dressing weights tau (9, nsm): tau(l, k) = sum_s x_s T_s(l) phi_k(s), T_s(l) = (dc(l) / dl(l, spc_s))^1/2, for a
    target site whose class holds species spc (1-based) at concentrations conc; states beyond the species of non-zero
    weight get zero; frozen: the target is the frozen centre (tau = 1 on the reference state)."""
    dc = np.asarray(dc, dtype=float)
    dl = np.asarray(dl, dtype=float)
    spc = np.asarray(spc, dtype=np.int64)
    conc = np.asarray(conc, dtype=float)
    nsm = len(conc) if nsm is None else nsm
    tau = np.zeros((9, nsm))
    if frozen:
        tau[:, 0] = 1.0
        return tau
    sup = np.nonzero(conc > 0.0)[0]
    phi = augn_basis(conc[sup])
    for k in range(len(sup)):
        for j, s in enumerate(sup):
            tau[:, k] += conc[s] * np.sqrt(dc / dl[:, spc[s] - 1]) * phi[k, j]
    return tau


def spectral_structure_ok(s) -> bool:
    """True if every sublattice of the structure is a single orbit of its space group (labels kept): one set of
    component potentials per sublattice needs every site of it equivalent to its first site."""
    from .crystal import space_group
    ops = space_group(s)
    for kap in range(1, s.nlabel + 1):
        sites = np.nonzero(s.label == kap)[0]
        if sites.size == 0:
            continue
        b0 = int(sites[0])
        reach = {int(o.perm[b0]) for o in ops}
        if any(int(b) not in reach for b in sites):
            return False
    return True


def spectral_origin_classes(s, ops=None):
    """Basis sites grouped by pure translations (rot = +I) and inversions (rot = -I) of the space group, sublattice by
    sublattice.  Returns bclass (nb, 1-based class), orig_b (1-based representative basis sites), orig_sign (nb: +1 when a
    translation maps the site onto its representative, -1 when an inversion does) and orig_w (site fraction per class)."""
    from .crystal import space_group
    ops = space_group(s) if ops is None else ops
    nb = s.nb
    bclass = np.zeros(nb, dtype=np.int64)
    sign = np.ones(nb, dtype=np.int64)
    orig = []
    eye = np.eye(3)
    for kap in range(1, s.nlabel + 1):
        for b in range(nb):
            if s.label[b] != kap or bclass[b]:
                continue
            orig.append(b + 1)
            bclass[b] = len(orig)
            for want, sg in ((eye, 1), (-eye, -1)):
                for b2 in range(b + 1, nb):
                    if s.label[b2] != kap or bclass[b2]:
                        continue
                    if any(o.perm[b2] == b and np.max(np.abs(o.rot - want)) < 1e-7 for o in ops):
                        bclass[b2], sign[b2] = len(orig), sg
    w = np.array([np.sum(bclass == g) / nb for g in range(1, len(orig) + 1)])
    return bclass, np.array(orig, dtype=np.int64), sign, w


def spectral_targets(cg, bclass, orig_sign, rmax: float) -> dict:
    """Targets of one origin class (spectral_final, src/asr_class_scf.f90:1562-1586): the sites of the origin's crystal
    graph ``cg`` (``crystal.crystal_graph`` started on the origin's representative basis site) within rmax (alat) of the
    origin, in cluster order.  bclass (nb, 1-based) and orig_sign (nb) come from ``spectral_origin_classes``.  Returns
    dict(tsite (nt,) 1-based graph sites for ``asr_op_build_targets``, tdisp (3, nt), tbase (nt,) the 0-based origin class
    of each target's basis site, tsign (nt,), t0 the index of the origin among the targets)."""
    disp = np.asarray(cg.disp, dtype=float)
    r2 = 4.0 * np.sum(disp * disp, axis=0)
    sel = np.nonzero(r2 <= 4.0 * rmax * rmax + 1.0e-9)[0]
    if sel.size == 0 or sel[0] != 0:
        raise ValueError("spectral_targets: the origin is not a spectral target")
    basis = np.asarray(cg.basis)[sel]
    return dict(tsite=(sel + 1).astype(np.int32), tdisp=disp[:, sel].copy(),
                tbase=(np.asarray(bclass)[basis] - 1).astype(np.int64), tsign=np.asarray(orig_sign)[basis].astype(float),
                t0=0)


def spectral_elements(op, tnode, tgop, t0: int, comps, conc, eds, z, nsteps: int, tail: str = "hull", precision: str = "fp64",
                      project: bool = True, spc=None):
    """The averaged elements of one origin class (spectral_worker, src/asr_class_scf.f90:1862-1910): for every central
    species comps[c] (1-based, concentration conc[c], edc parameters eds[c] from ``synthetic.edc_params``), start orbital
    o = 1..9 and energy, one projected chain on the device; gdg(o, t, j) = sum_c x_c gp(o, t) and gdg4 the same from the
    chains cut four steps earlier.  op: the D2h-reduced operator built with the targets (tnode, tgop (nsm, nt)); t0 the
    index of the origin among the targets.  Returns (gdg, gdg4), each (9, nt, ne)."""
    tnode = np.asarray(tnode)
    nsm, nt = tnode.shape
    spc = np.asarray(comps if spc is None else spc, dtype=np.int64)
    z = np.atleast_1d(np.asarray(z, dtype=np.complex128))
    ne = z.shape[0]
    gdg = np.zeros((9, nt, ne), np.complex128)
    gdg4 = np.zeros((9, nt, ne), np.complex128)
    for ci, cen in enumerate(comps):
        ed = eds[ci]
        tw = np.zeros((9, nsm, nt))
        for t in range(nt):
            tw[:, :, t] = spectral_dressing(ed["dc"], ed["dl"], spc, conc, t == t0, nsm)
        specs = [ChainSpec(c=ed["c"], d=ed["d"], o=ed["o"], e=ed["e"], pa=ed["pa"], pb=ed["pb"], frozen_sp=int(cen),
                           start_orb=l0, nlev=nsteps) for l0 in range(1, 10)]
        r = chains_proj(op, specs, z, tnode, tgop, tw, tail, precision, project)
        for o in range(9):
            gdg[o] += conc[ci] * r["gp"][o, :, :, o]
            gdg4[o] += conc[ci] * r["gp4"][o, :, :, o]
    return gdg, gdg4


def spectral_sum(gdg, tdisp, kv, rmax: float, window: str = "ball"):
    """Symmetrise with the partner element at -R (the element itself where no partner exists) and sum the windowed
    Bloch series per l (src/asr_class_scf.f90:1690-1745): A (ne, nk, 3) = sum_R w(|R|) cos(2 pi k . R)
    (-1/pi) Im sum_{L in l} <G_{0L, RL}>.  gdg (9, nt, ne); tdisp (3, nt) alat; kv (3, nk) units 2 pi / alat."""
    tdisp = np.asarray(tdisp, dtype=float)
    nt = tdisp.shape[1]
    mir = np.arange(nt)
    for t in range(nt):
        hit = np.nonzero(np.all(np.abs(tdisp + tdisp[:, t:t + 1]) < 1e-9, axis=0))[0]
        if hit.size:
            mir[t] = hit[0]
    gsym = 0.5 * (gdg + gdg[:, mir])
    w = np.array([spectral_window(window, float(np.linalg.norm(tdisp[:, t])), rmax) for t in range(nt)])
    kv = np.asarray(kv, dtype=float).reshape(3, -1)
    phase = np.cos(2.0 * np.pi * (kv.T @ tdisp))                              # (nk, nt)
    A = np.zeros((gdg.shape[2], kv.shape[1], 3))
    for l in range(3):
        v = -np.imag(np.sum(gsym[ORB_L == l], axis=0)) / np.pi                # (nt, ne)
        A[:, :, l] = (phase @ (v * w[:, None])).T
    return A, gsym


def spectral_sum_origins(gdg: list, tdisp: list, tbase: list, tsign: list, orig_w, kv, rmax: float, window: str = "ball"):
    """A(k, E) summed over origin classes u with weights orig_w[u] (spectral_final, src/asr_class_scf.f90:1588-1601
    partners, :1693-1701 symmetrisation, :1725-1746 the weighted Bloch sum).  gdg[u] (9, nt_u, ne) are the elements of
    origin u, tdisp[u] (3, nt_u) the target displacements (alat), tbase[u] (nt_u, 0-based) the origin class of each
    target's basis site and tsign[u] (nt_u) the sign of the operation that maps that site onto its class representative.
    The partner of target t of origin u is the target j of origin u2 = tbase[u][t] with tbase[u2][j] == u and
    tdisp[u2][:, j] = -tsign[u][t] tdisp[u][:, t]; without one it is target t of origin u2.  Every element whose partner is
    not itself is averaged with it.  Returns (A (ne, nk, 3) per orbital l, parts (norig, ne, nk) the part of each origin
    summed over l, the symmetrised elements)."""
    nor = len(gdg)
    mir = []
    for u in range(nor):
        mu = []
        for t in range(tdisp[u].shape[1]):
            u2 = int(tbase[u][t])
            hit = [j for j in range(tdisp[u2].shape[1]) if int(tbase[u2][j]) == u
                   and np.max(np.abs(tdisp[u2][:, j] + tsign[u][t] * tdisp[u][:, t])) < 1e-9]
            mu.append((u2, hit[0] if hit else t))
        mir.append(mu)
    sym = []
    for u in range(nor):
        g = np.array(gdg[u], copy=True)
        for t, (u2, j) in enumerate(mir[u]):
            if (u2, j) != (u, t):
                g[:, t] = 0.5 * (gdg[u][:, t] + gdg[u2][:, j])
        sym.append(g)
    kv = np.asarray(kv, dtype=float).reshape(3, -1)
    ne = sym[0].shape[2]
    A = np.zeros((ne, kv.shape[1], 3))
    parts = np.zeros((nor, ne, kv.shape[1]))
    for u in range(nor):
        w = np.array([spectral_window(window, float(np.linalg.norm(tdisp[u][:, t])), rmax) for t in range(tdisp[u].shape[1])])
        phase = np.cos(2.0 * np.pi * (kv.T @ tdisp[u]))
        for l in range(3):
            v = -np.imag(np.sum(sym[u][ORB_L == l], axis=0)) / np.pi
            a = orig_w[u] * (phase @ (v * w[:, None])).T
            A[:, :, l] += a
            parts[u] += a
    return A, parts, sym


def bloch_spectral(op, tnode, tgop, tdisp, t0: int, comps, conc, eds, z, kv, nsteps: int, rmax: float, window: str = "ball",
                   tail: str = "hull", precision: str = "fp64", project: bool = True, spc=None):
    """A(k, E) of one origin class on a Bravais sublattice (spectral_final, src/asr_class_scf.f90:1600-1760):
    ``spectral_elements`` then ``spectral_sum``.  Returns (A (ne, nk, 3), gsym (9, nt, ne), spread4 = the largest
    off-site |gdg - gdg4| over the largest off-site |gdg|, the reference's step-spread diagnostic)."""
    gdg, gdg4 = spectral_elements(op, tnode, tgop, t0, comps, conc, eds, z, nsteps, tail, precision, project, spc)
    nt = gdg.shape[1]
    off = np.arange(nt) != t0
    spread4 = 0.0
    if off.any():
        spread4 = float(np.max(np.abs(gdg[:, off] - gdg4[:, off])) / max(np.max(np.abs(gdg[:, off])), 1e-300))
    A, gsym = spectral_sum(gdg, tdisp, kv, rmax, window)
    return A, gsym, spread4
