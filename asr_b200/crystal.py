"""Structure clusters and their symmetry: the operator inputs of a sublattice, found from the structure alone.

Host-side restatement of the set-up that feeds ``build_augcls_operator`` in the reference's ``class_scf``
(src/asr_class_scf.f90:342-391):

* ``Structure`` / ``prototype_structure`` -- ``structure_t`` (src/asr_crystal.f90:15-60) and the named prototypes of
  src/asr_prototypes.f90:19-65 (sc, bcc, fcc, b2, hex, hcp, nias): primitive vectors as columns in alat units,
  fractional basis positions wrapped into [0, 1), sublattice labels;
* ``space_group`` -- every {m | t} with m integer in lattice coordinates (entries -2..2, |det m| = 1, m^T G m = G) that
  maps each site onto a site with its label (src/asr_crystal_symmetry.f90:50-116); the identity first;
* ``site_ops``, ``basis_orbits``, ``translation_types``, ``is_monomial``, ``orbital_matrix``, ``orbital_groups``,
  ``reduction_ops`` -- src/asr_crystal_symmetry.f90:118-254: the site group of a basis site, the orbital groups of a
  site group (one start orbital per group, its size the weight; cubic sites give s | p | t2g | e_g), and the monomial
  reduction group under which every representative is one dimensional;
* ``crystal_graph`` / ``graph_site`` / ``graph_site_ops`` / ``structure_cluster`` -- src/asr_crystal_graph.f90:60-245: the
  ball of radius 2 levels b_max about the start site (no periodic box), one union list of bond slots sorted by length
  then x, y, z, neighbour entries 0 (no such bond) and -1 (outside the ball), and the site operations in canonical
  order (monomial first, by axis permutation and row signs);
* ``sublattice_inputs`` -- the per-sublattice block of class_scf: flippable sites, classes, the class-preserving site
  group, its orbital groups and reduction group, giving (graph, cls, perm, dmat, flippable, start orbitals, weights);
* ``decoration_build`` / ``decoration_classes`` / ``decoration_structure`` -- src/asr_sublattice.f90:26-116: sublattices
  given by Wyckoff positions of a decoration cell of ``period`` conventional cubes of an sc / bcc / fcc graph with a
  centering (P, I, F), as classes of graph sites or as a crystal structure.

Everything here runs once per set-up on the host (integer and small dense work); the device build consumes its output.
"""
from __future__ import annotations

import functools
from dataclasses import dataclass, field

import numpy as np

from .lattices import Graph, orbital_rep

__all__ = ["Structure", "prototype_structure", "SymOp", "space_group", "site_ops", "basis_orbits", "translation_types",
           "is_monomial", "orbital_matrix", "orbital_groups", "reduction_ops", "CrystalGraph", "crystal_graph", "graph_site",
           "graph_site_ops", "structure_cluster", "graph_distances", "sublattice_inputs", "Decoration", "decoration_build",
           "decoration_classes", "decoration_structure", "GEO_TOL", "RTOL"]

GEO_TOL = 1.0e-6     # fractional-coordinate tolerance (src/asr_crystal.f90:13)
RTOL = 1.0e-9        # distance tolerance in alat units (src/asr_crystal_graph.f90:36)
OTOL = 1.0e-9        # orbital-matrix entries within this of an integer are that integer
# tie-break order of the start-orbital representatives: s, p_z, d_3z2, d_xy, d_x2-y2, p_y, p_x, d_yz, d_xz (1-based)
PREF = (1, 3, 7, 5, 9, 2, 4, 6, 8)
# axis permutations in the order of the canonical site-operation key (as the cubic operation table)
AXPERM = ((1, 2, 3), (1, 3, 2), (2, 1, 3), (2, 3, 1), (3, 1, 2), (3, 2, 1))


def inv3(a: np.ndarray) -> np.ndarray:
    """Inverse of a 3 x 3 matrix by its adjugate: exact on the half-integer cells of the prototypes."""
    a = np.asarray(a, dtype=float)
    c = np.empty((3, 3))
    for i in range(3):
        for j in range(3):
            r = [k for k in range(3) if k != i]
            s = [k for k in range(3) if k != j]
            c[i, j] = (-1) ** (i + j) * (a[r[0], s[0]] * a[r[1], s[1]] - a[r[0], s[1]] * a[r[1], s[0]])
    det = float(np.sum(a[0, :] * c[0, :]))
    return c.T / det


def det3(a) -> float:
    a = np.asarray(a, dtype=float)
    return float(a[0, 0] * (a[1, 1] * a[2, 2] - a[1, 2] * a[2, 1]) - a[0, 1] * (a[1, 0] * a[2, 2] - a[1, 2] * a[2, 0])
                 + a[0, 2] * (a[1, 0] * a[2, 1] - a[1, 1] * a[2, 0]))


def same_frac(f1, f2) -> bool:
    d = np.asarray(f1, float) - np.asarray(f2, float)
    return bool(np.all(np.abs(d - np.rint(d)) < GEO_TOL))


# --------------------------------------------------------------------------------------------------------- structures
@dataclass
class Structure:
    """Primitive vectors ``avec`` (3, 3) as columns (alat units), fractional positions ``frac`` (3, nb) wrapped into
    [0, 1), positive sublattice labels ``label`` (nb)."""
    avec: np.ndarray
    frac: np.ndarray
    label: np.ndarray
    bvec: np.ndarray = field(init=False)     # dual vectors as columns, b_i . a_j = delta_ij (no 2 pi)
    tau: np.ndarray = field(init=False)      # Cartesian positions (3, nb)

    def __post_init__(self):
        self.avec = np.asarray(self.avec, dtype=float).reshape(3, 3)
        frac = np.asarray(self.frac, dtype=float).reshape(3, -1)
        self.label = np.asarray(self.label, dtype=np.int64).reshape(-1)
        if frac.shape[1] < 1 or self.label.shape[0] != frac.shape[1]:
            raise ValueError("Structure: frac must be (3, nb) and label (nb) with nb >= 1")
        if abs(det3(self.avec)) < GEO_TOL:
            raise ValueError("Structure: the primitive vectors are linearly dependent")
        if np.any(self.label < 1):
            raise ValueError("Structure: labels must be positive")
        self.frac = frac - np.floor(frac + GEO_TOL)
        self.bvec = inv3(self.avec).T
        self.tau = self.avec @ self.frac
        for b in range(self.nb):
            for c in range(b + 1, self.nb):
                if same_frac(self.frac[:, b], self.frac[:, c]):
                    raise ValueError("Structure: two basis sites coincide")

    @property
    def nb(self) -> int:
        return int(self.frac.shape[1])

    @property
    def nlabel(self) -> int:
        return int(np.max(self.label))


def _hexagonal(ca: float) -> np.ndarray:
    return np.array([[1.0, -0.5, 0.0], [0.0, np.sqrt(3.0) / 2.0, 0.0], [0.0, 0.0, ca]])


def prototype_structure(name: str, c_over_a: float | None = None) -> Structure:
    """The named prototypes (src/asr_prototypes.f90:19-65): the cells and basis sites are those of the reference so that
    site, slot and operation orders agree."""
    h, t1, t2, q1, q3 = 0.5, 1.0 / 3.0, 2.0 / 3.0, 0.25, 0.75
    if name == "sc":
        return Structure(np.eye(3), np.zeros((3, 1)), [1])
    if name == "bcc":
        return Structure(np.array([[-h, h, h], [h, -h, h], [h, h, -h]]), np.zeros((3, 1)), [1])
    if name == "fcc":
        return Structure(np.array([[0.0, h, h], [h, 0.0, h], [h, h, 0.0]]), np.zeros((3, 1)), [1])
    if name == "b2":
        return Structure(np.eye(3), np.array([[0.0, h], [0.0, h], [0.0, h]]), [1, 2])
    if name == "hex":
        if c_over_a is None:
            raise ValueError("prototype hex: c_over_a is required")
        return Structure(_hexagonal(c_over_a), np.zeros((3, 1)), [1])
    if name == "hcp":
        ca = np.sqrt(8.0 / 3.0) if c_over_a is None else c_over_a
        return Structure(_hexagonal(ca), np.array([[0.0, t1], [0.0, t2], [0.0, h]]), [1, 1])
    if name == "nias":
        if c_over_a is None:
            raise ValueError("prototype nias: c_over_a is required")
        return Structure(_hexagonal(c_over_a), np.array([[0.0, 0.0, t1, t2], [0.0, 0.0, t2, t1], [0.0, h, q1, q3]]),
                         [1, 1, 2, 2])
    raise ValueError(f"unknown prototype {name!r} (known: sc bcc fcc b2 hex hcp nias)")


# --------------------------------------------------------------------------------------------------------- symmetry
@dataclass
class SymOp:
    """{m | t}: m integer rotation in lattice coordinates, rot its Cartesian form, t fractional translation in [0, 1);
    basis site b goes to perm[b] (0-based) with m frac_b + t = frac_perm[b] + shift[:, b]."""
    m: np.ndarray
    rot: np.ndarray
    t: np.ndarray
    perm: np.ndarray
    shift: np.ndarray


def _metric_rotations(g: np.ndarray) -> np.ndarray:
    """Every integer matrix with entries -2..2, |det| = 1 and m^T g m = g, in the search order of the reference (code
    0 .. 5^9 - 1, digit j of the code -> m[j % 3, j // 3])."""
    code = np.arange(5 ** 9, dtype=np.int64)
    dig = np.empty((code.size, 9), dtype=np.int8)
    k = code.copy()
    for j in range(9):
        dig[:, j] = (k % 5) - 2
        k //= 5
    m = np.zeros((code.size, 3, 3), dtype=np.int8)
    for j in range(9):
        m[:, j % 3, j // 3] = dig[:, j]
    mi = m.astype(np.int64)
    det = (mi[:, 0, 0] * (mi[:, 1, 1] * mi[:, 2, 2] - mi[:, 1, 2] * mi[:, 2, 1])
           - mi[:, 0, 1] * (mi[:, 1, 0] * mi[:, 2, 2] - mi[:, 1, 2] * mi[:, 2, 0])
           + mi[:, 0, 2] * (mi[:, 1, 0] * mi[:, 2, 1] - mi[:, 1, 1] * mi[:, 2, 0]))
    cand = mi[np.abs(det) == 1].astype(float)
    mg = np.einsum("nki,kl,nlj->nij", cand, g, cand)
    ok = np.max(np.abs(mg - g[None]).reshape(len(cand), 9), axis=1) <= 1.0e-8
    return cand[ok].astype(np.int64)


def space_group(s: Structure) -> list[SymOp]:
    """All operations {m | t} that map the structure onto itself, labels included; operation 0 is the identity
    (src/asr_crystal_symmetry.f90:50-116)."""
    g = s.avec.T @ s.avec
    ainv = inv3(s.avec)
    # every operation must carry some site onto a site of the same label; trying the translations only from one site of
    # the rarest label keeps the candidate list shortest (ties: the lowest label number, then the first such site)
    i0, nlab = 0, s.nb + 1
    for lab in range(1, s.nlabel + 1):
        n = int(np.sum(s.label == lab))
        if 0 < n < nlab:
            nlab, i0 = n, int(np.argmax(s.label == lab))
    ops: list[SymOp] = []
    for m in _metric_rotations(g):
        rm = m.astype(float)
        for j in range(s.nb):
            if s.label[j] != s.label[i0]:
                continue
            t = s.frac[:, j] - rm @ s.frac[:, i0]
            t = t - np.floor(t + GEO_TOL)
            perm = np.zeros(s.nb, dtype=np.int64)
            shift = np.zeros((3, s.nb), dtype=np.int64)
            ok = True
            for b in range(s.nb):
                fb = rm @ s.frac[:, b] + t
                hit = -1
                for c in range(s.nb):
                    if s.label[c] == s.label[b] and same_frac(fb, s.frac[:, c]):
                        hit = c
                        break
                if hit < 0:
                    ok = False
                    break
                perm[b] = hit
                shift[:, b] = np.rint(fb - s.frac[:, hit]).astype(np.int64)
            if not ok:
                continue
            if any(np.array_equal(o.m, m) and same_frac(o.t, t) for o in ops):
                continue
            ops.append(SymOp(m=m.copy(), rot=s.avec @ rm @ ainv, t=t, perm=perm, shift=shift))
    ident = [k for k, o in enumerate(ops) if np.array_equal(o.m, np.eye(3, dtype=np.int64)) and np.all(np.abs(o.t) < GEO_TOL)]
    if not ident:
        raise RuntimeError("space_group: the identity was not found")
    k = ident[0]
    # the identity goes first by exchanging two entries (not by a shift of the list), so that the site groups and the
    # canonical representatives built from this order see the operations in the order the search found them
    ops[0], ops[k] = ops[k], ops[0]
    return ops


def site_ops(ops: list[SymOp], b: int) -> np.ndarray:
    """0-based indices of the site group of basis site b (0-based): the operations with perm[b] = b."""
    return np.array([k for k, o in enumerate(ops) if o.perm[b] == b], dtype=np.int64)


def basis_orbits(ops: list[SymOp], nb: int):
    """Space-group orbits of the basis sites: orbit (nb) in 1..norbit numbered by first site, and norbit."""
    orbit = np.zeros(nb, dtype=np.int64)
    norbit = 0
    for b in range(nb):
        if orbit[b]:
            continue
        norbit += 1
        for o in ops:
            orbit[o.perm[b]] = norbit
    return orbit, norbit


def translation_types(s: Structure):
    """Basis sites b, c share a type when frac_c - frac_b maps every site onto a site (labels ignored): the geometry,
    so the structure constants, seen from both is the same.  Returns typ (nb) in 1..ntyp and ntyp."""
    typ = np.zeros(s.nb, dtype=np.int64)
    ntyp = 0
    for b in range(s.nb):
        if typ[b]:
            continue
        ntyp += 1
        typ[b] = ntyp
        for c in range(b + 1, s.nb):
            if typ[c]:
                continue
            sh = s.frac[:, c] - s.frac[:, b]
            if all(any(same_frac(s.frac[:, d] + sh, s.frac[:, e]) for e in range(s.nb)) for d in range(s.nb)):
                typ[c] = ntyp
    return typ, ntyp


def is_monomial(rot: np.ndarray) -> bool:
    """A signed permutation: one entry +-1 per row and column, zeros elsewhere."""
    r = np.asarray(rot, dtype=float)
    if not np.all((np.abs(r) < GEO_TOL) | (np.abs(np.abs(r) - 1.0) < GEO_TOL)):
        return False
    big = np.abs(r) > 0.5
    return bool(np.all(big.sum(axis=1) == 1) and np.all(big.sum(axis=0) == 1))


def orbital_matrix(rot: np.ndarray) -> np.ndarray:
    """d (9, 9) with Y_k(rot p) = sum_j d(k, j) Y_j(p) for any rotation (least squares on a fixed point set)."""
    return np.ascontiguousarray(orbital_rep(np.asarray(rot, dtype=float).reshape(3, 3, 1))[:, :, 0])


def orbital_groups(d: np.ndarray, mono):
    """Orbital groups of a site group (src/asr_crystal_symmetry.f90:208-238).

    d (9, 9, nop) orbital matrices, mono (nop) monomial flags.  Two orbitals share a group when the twirl
    (1/|G|) sum_g d(:, L, g) d(:, L, g)^T is the same matrix: then every matrix that commutes with the group has equal
    diagonal entries on them.  Returns grp (9, values 1..ngrp numbered by first orbital), ngrp, rep (ngrp, 1-based: the
    orbital of the group with the largest monomial little group, ties in PREF order) and weight (ngrp, group sizes)."""
    d = np.asarray(d, dtype=float)
    mono = np.asarray(mono, dtype=bool)
    nop = d.shape[2]
    u = np.einsum("klg,jlg->lkj", d, d) / nop           # u[l] = mean_g d(:, l, g) d(:, l, g)^T
    grp = np.zeros(9, dtype=np.int64)
    ngrp = 0
    for l in range(9):
        for l2 in range(l):
            if np.max(np.abs(u[l] - u[l2])) < 1.0e-8:
                grp[l] = grp[l2]
                break
        if grp[l] == 0:
            ngrp += 1
            grp[l] = ngrp
    rep = np.zeros(ngrp, dtype=np.int64)
    weight = np.zeros(ngrp, dtype=np.int64)
    for k in range(1, ngrp + 1):
        weight[k - 1] = int(np.sum(grp == k))
        best = -1
        for p in PREF:
            if grp[p - 1] != k:
                continue
            nlit = int(np.sum(mono & (np.abs(np.abs(d[p - 1, p - 1, :]) - 1.0) < OTOL)))
            if nlit > best:
                best, rep[k - 1] = nlit, p
    return grp, ngrp, rep, weight


def reduction_ops(d: np.ndarray, mono, reps) -> np.ndarray:
    """0-based indices of the monomial operations under which every representative orbital (1-based) is one dimensional."""
    d = np.asarray(d, dtype=float)
    keep = np.asarray(mono, dtype=bool).copy()
    for r in reps:
        keep &= np.abs(np.abs(d[r - 1, r - 1, :]) - 1.0) < OTOL
    return np.nonzero(keep)[0]


# --------------------------------------------------------------------------------------------------------- the graph
def _sort_keys(key: np.ndarray) -> np.ndarray:
    """Stable order of the columns of key (rows compared first to last, entries within RTOL equal)."""
    cols = [key[:, i] for i in range(key.shape[1])]

    def cmp(a, b):
        for x, y in zip(cols[a], cols[b]):
            if x < y - RTOL:
                return -1
            if x > y + RTOL:
                return 1
        return 0
    return np.array(sorted(range(len(cols)), key=functools.cmp_to_key(cmp)), dtype=np.int64)


def _cells(s: Structure, r: float):
    nmax = [int(np.ceil(r * np.linalg.norm(s.bvec[:, i]))) + 1 for i in range(3)]
    # n1 fastest, then n2, then n3 (the loop order of the reference)
    n3, n2, n1 = np.meshgrid(*[np.arange(-nmax[i], nmax[i] + 1) for i in (2, 1, 0)], indexing="ij")
    return np.stack([n1.ravel(), n2.ravel(), n3.ravel()]).astype(np.int64)


def structure_cluster(s: Structure, b: int, rmax: float):
    """Every crystal site within rmax (alat units) of basis site b (0-based): vec (3, n) Cartesian, relative to b, the
    origin first, then by distance, ties by z, then y, then x; cb (n) basis site (0-based) and cn (3, n) cell of each."""
    cells = _cells(s, rmax)
    tv, tc, tn = [], [], []
    for c in range(s.nb):
        v = s.avec @ (cells + (s.frac[:, c] - s.frac[:, b])[:, None])
        keep = np.sqrt(np.sum(v * v, axis=0)) <= rmax + RTOL
        tv.append(v[:, keep])
        tc.append(np.full(int(keep.sum()), c, dtype=np.int64))
        tn.append(cells[:, keep])
    tv, tc, tn = np.concatenate(tv, axis=1), np.concatenate(tc), np.concatenate(tn, axis=1)
    key = np.vstack([np.sum(tv * tv, axis=0), tv[2], tv[1], tv[0]])
    order = _sort_keys(key)
    vec = tv[:, order]
    if np.sum(vec[:, 0] ** 2) > 0.0:
        raise RuntimeError("structure_cluster: the origin is not first")
    return vec, tc[order], tn[:, order]


@dataclass
class CrystalGraph:
    """``crystal_graph_t`` (src/asr_crystal_graph.f90:38-54).  Sites are 1-based in ``g``; ``basis`` and ``b0`` are
    0-based basis indices; ``btgt`` (nslot, nb) holds 1-based basis sites (0: no such bond)."""
    g: Graph
    n: int
    nslot: int
    nb: int
    b0: int
    norbit: int
    levels: int
    radius: float
    bmax: float
    nbox: np.ndarray
    cell: np.ndarray
    basis: np.ndarray
    orbit: np.ndarray
    bvec: np.ndarray
    btgt: np.ndarray
    bdn: np.ndarray
    disp: np.ndarray
    index: np.ndarray


def graph_site(cg: CrystalGraph, n, b: int) -> int:
    """1-based site of crystal site (cell n, basis b 0-based); 0 outside the cluster."""
    n = np.asarray(n, dtype=np.int64)
    if np.any(np.abs(n) > cg.nbox):
        return 0
    return int(cg.index[n[0] + cg.nbox[0], n[1] + cg.nbox[1], n[2] + cg.nbox[2], b])


def crystal_graph(s: Structure, ops: list[SymOp], rcl: float, levels: int, start: int = 0,
                  rmin: float | None = None) -> CrystalGraph:
    """Graph of structure s with every bond up to rcl (alat units) on the ball of radius max(2 levels b_max, rmin) about
    basis site ``start`` (0-based) (src/asr_crystal_graph.f90:60-168)."""
    if not 0 <= start < s.nb:
        raise ValueError("crystal_graph: start is not a basis site")
    if levels < 0:
        raise ValueError("crystal_graph: levels must not be negative")
    cells = _cells(s, rcl)
    tv, tb, tt, tdn = [], [], [], []
    for b in range(s.nb):
        for c in range(s.nb):
            f = cells + (s.frac[:, c] - s.frac[:, b])[:, None]
            v = s.avec @ f
            keep = np.sqrt(np.sum(v * v, axis=0)) <= rcl + RTOL
            if c == b:
                keep &= np.any(cells != 0, axis=0)
            for i in np.nonzero(keep)[0]:
                tv.append(v[:, i])
                tb.append(b)
                tt.append(c)
                tdn.append(cells[:, i])
    if not tv:
        raise ValueError("crystal_graph: no bond within rcl")
    # union of the bond vectors (first occurrence), sorted by length, then x, y, z
    uniq: list[np.ndarray] = []
    slot_of = np.zeros(len(tv), dtype=np.int64)
    for i, v in enumerate(tv):
        for j, u in enumerate(uniq):
            if np.max(np.abs(u - v)) < GEO_TOL:
                slot_of[i] = j
                break
        else:
            slot_of[i] = len(uniq)
            uniq.append(v)
    ns = len(uniq)
    key = np.array([[np.sum(v * v), v[0], v[1], v[2]] for v in uniq]).T
    order = _sort_keys(key)
    lab = np.empty(ns, dtype=np.int64)
    lab[order] = np.arange(ns)
    bvec = key[1:4, order].copy()
    btgt = np.zeros((ns, s.nb), dtype=np.int64)
    bdn = np.zeros((3, ns, s.nb), dtype=np.int64)
    for i in range(len(tv)):
        k = lab[slot_of[i]]
        btgt[k, tb[i]] = tt[i] + 1
        bdn[:, k, tb[i]] = tdn[i]
    bmax = float(np.max(np.linalg.norm(bvec, axis=0)))
    radius = 2.0 * levels * bmax
    if rmin is not None:
        radius = max(radius, float(rmin))
    disp, basis, cell = structure_cluster(s, start, radius)
    n = disp.shape[1]
    nbox = np.max(np.abs(cell), axis=1) + 1
    index = np.zeros((2 * nbox[0] + 1, 2 * nbox[1] + 1, 2 * nbox[2] + 1, s.nb), dtype=np.int64)
    index[cell[0] + nbox[0], cell[1] + nbox[1], cell[2] + nbox[2], basis] = np.arange(1, n + 1)
    cg = CrystalGraph(g=None, n=n, nslot=ns, nb=s.nb, b0=start, norbit=0, levels=levels, radius=radius, bmax=bmax,
                      nbox=nbox, cell=cell, basis=basis, orbit=None, bvec=bvec, btgt=btgt, bdn=bdn, disp=disp, index=index)
    # neighbour lists: slot k of site i is the site at r_i + bvec[:, k]; 0 no such bond, -1 outside the ball
    nbr = np.zeros((n, ns), dtype=np.int64)
    has = btgt[:, basis].T > 0                                           # (n, ns)
    tgt = btgt[:, basis].T - 1
    dest = cell[:, :, None] + np.transpose(bdn[:, :, basis], (0, 2, 1))   # (3, n, ns)
    inbox = np.all(np.abs(dest) <= nbox[:, None, None], axis=0)
    dc = np.clip(dest + nbox[:, None, None], 0, (2 * nbox)[:, None, None])
    site = index[dc[0], dc[1], dc[2], np.maximum(tgt, 0)]
    site = np.where(inbox, site, 0)
    nbr[has] = np.where(site[has] > 0, site[has], -1)
    cg.g = Graph(n=n, nbr_ptr=(1 + ns * np.arange(n + 1)).astype(np.int32), nbr=nbr.reshape(-1).astype(np.int32))
    orb, cg.norbit = basis_orbits(ops, s.nb)
    cg.orbit = orb[basis]
    return cg


def _op_key(rot: np.ndarray, k: int) -> int:
    if not is_monomial(rot):
        return 1000 + k
    pp = tuple(int(np.argmax(np.abs(rot[i, :]))) + 1 for i in range(3))
    sgn = sum(1 << i for i in range(3) if rot[i, pp[i] - 1] < 0.0)
    return 8 * AXPERM.index(pp) + sgn


def graph_site_ops(cg: CrystalGraph, s: Structure, ops: list[SymOp]):
    """The space-group operations that fix the start site, in canonical order (src/asr_crystal_graph.f90:180-206):
    perm (n, nk) Fortran order with 1-based site images, rot (3, 3, nk), idx (nk) 0-based indices into ops."""
    if s.nb != cg.nb:
        raise ValueError("graph_site_ops: the graph belongs to another structure")
    b0 = cg.b0
    cand = [k for k, o in enumerate(ops) if o.perm[b0] == b0]
    keys = [_op_key(ops[k].rot, k + 1) for k in cand]
    order = sorted(range(len(cand)), key=lambda i: keys[i])
    nk = len(cand)
    perm = np.zeros((cg.n, nk), dtype=np.int32, order="F")
    rot = np.zeros((3, 3, nk), order="F")
    idx = np.zeros(nk, dtype=np.int64)
    for i, oi in enumerate(order):
        k = cand[oi]
        o = ops[k]
        idx[i] = k
        rot[:, :, i] = o.rot
        n2 = o.m @ cg.cell + o.shift[:, cg.basis] - o.shift[:, b0][:, None]
        bb = o.perm[cg.basis]
        inbox = np.all(np.abs(n2) <= cg.nbox[:, None], axis=0)
        dc = np.clip(n2 + cg.nbox[:, None], 0, (2 * cg.nbox)[:, None])
        perm[:, i] = np.where(inbox, cg.index[dc[0], dc[1], dc[2], bb], 0)
    if np.any(perm == 0):
        raise RuntimeError("graph_site_ops: an operation maps a site out of the cluster")
    if not np.array_equal(perm[:, 0], np.arange(1, cg.n + 1)):
        raise RuntimeError("graph_site_ops: operation 1 is not the identity")
    if np.any(perm[0, :] != 1):
        raise RuntimeError("graph_site_ops: an operation moves the start site")
    return perm, rot, idx


def graph_distances(g: Graph, start: int = 1) -> np.ndarray:
    """Hop distances from site ``start`` (1-based) by breadth-first search; entries <= 0 are not bonds; -1 unreached
    (src/asr_augspace.f90:119-135)."""
    nbr_ptr = np.asarray(g.nbr_ptr)
    nbr = np.asarray(g.nbr)
    dist = -np.ones(g.n, dtype=np.int64)
    dist[start - 1] = 0
    front = [start]
    d = 0
    while front:
        d += 1
        nxt = []
        for r in front:
            for j in nbr[nbr_ptr[r - 1] - 1:nbr_ptr[r] - 1]:
                if j > 0 and dist[j - 1] < 0:
                    dist[j - 1] = d
                    nxt.append(int(j))
        front = nxt
    return dist


# --------------------------------------------------------------------------------------------------------- sublattices
def sublattice_inputs(s: Structure, ops: list[SymOp], kap: int, rcl: float, levels: int, flip_radius: int = 99,
                      rmin: float | None = None, cls_override=None, group: str = "reduction") -> dict:
    """Operator inputs of sublattice ``kap`` (1-based label), the per-sublattice block of src/asr_class_scf.f90:342-391:
    the ball about the first basis site with that label, flippable sites (graph distance <= flip_radius, not the start),
    classes = labels of the sites, the class-preserving site group and its orbital groups (start orbitals ``reps`` with
    weights), and the reduction group (``perm`` (n, nred), ``dmat`` (9, 9, nred)).  ``cls_override`` (n) replaces the
    classes (a short-range-order shell decoration, for instance) before the group is taken.  ``group="diagonal"``
    reduces by the diagonal operations of the class-preserving group instead (D2h on cubic sites: all nine orbitals
    one dimensional, as the spectral path does, src/asr_class_scf.f90:1613-1619); ``group="identity"`` not at all."""
    b0 = int(np.argmax(s.label == kap))
    if s.label[b0] != kap:
        raise ValueError(f"sublattice_inputs: no basis site carries label {kap}")
    cg = crystal_graph(s, ops, rcl, levels, start=b0, rmin=rmin)
    dist = graph_distances(cg.g, 1)
    flip = (dist <= flip_radius).astype(np.int32)
    flip[0] = 0
    cls = s.label[cg.basis].astype(np.int32) if cls_override is None else np.asarray(cls_override, dtype=np.int32)
    typ, _ = translation_types(s)
    perm, rot, _ = graph_site_ops(cg, s, ops)
    keep = [k for k in range(perm.shape[1]) if np.array_equal(cls[perm[:, k] - 1], cls)]
    if not keep or keep[0] != 0:
        raise RuntimeError("sublattice_inputs: the identity does not keep the classes")
    dgo = np.zeros((9, 9, len(keep)), order="F")
    mono = np.zeros(len(keep), dtype=bool)
    for i, k in enumerate(keep):
        dgo[:, :, i] = orbital_matrix(rot[:, :, k])
        mono[i] = is_monomial(rot[:, :, k])
    grp, ngrp, rep, wgt = orbital_groups(dgo, mono)
    if group == "reduction":
        red = reduction_ops(dgo, mono, rep)
    elif group == "diagonal":
        red = np.array([i for i, k in enumerate(keep) if np.array_equal(np.abs(rot[:, :, k]), np.eye(3))], dtype=np.int64)
    elif group == "identity":
        red = np.zeros(1, dtype=np.int64)
    else:
        raise ValueError(f"sublattice_inputs: unknown group {group!r}")
    return dict(cg=cg, graph=cg.g, cls=cls, flippable=flip, stype=typ[cg.basis].astype(np.int32),
                perm=np.asfortranarray(perm[:, [keep[r] for r in red]]), dmat=np.asfortranarray(dgo[:, :, red]),
                site_group=len(keep), orbital_group=grp, reps=rep, weights=wgt, maxlevel=levels)


# --------------------------------------------------------------------------------------------------------- decorations
def _on_graph(kind: str, h) -> bool:
    h = np.asarray(h, dtype=np.int64)
    if kind == "sc":
        return bool(np.all(h % 2 == 0))
    if kind == "bcc":
        return bool(h[0] % 2 == h[1] % 2 == h[2] % 2)
    if kind == "fcc":
        return bool(int(np.sum(h)) % 2 == 0)
    return False


@dataclass
class Decoration:
    """Sublattices of an sc / bcc / fcc graph in a cell of ``period`` conventional cubes (edge m = 2 period half-lattice
    units): ``tab`` (m, m, m) the sublattice of every graph point of the cell (0: not a site), ``pts`` (3, nsite) the sites
    in the order z, y, x (x fastest), ``pcls`` their sublattices, ``rep`` (3, ncls) the first site of each, ``frac`` the
    site fractions."""
    lattice: str
    period: int
    m: int
    ncls: int
    tab: np.ndarray
    pts: np.ndarray
    pcls: np.ndarray
    rep: np.ndarray
    frac: np.ndarray


def decoration_build(lattice: str, period: int, centering: str, pos, owner, ncls: int) -> Decoration:
    """Sublattices from Wyckoff positions pos (3, k) (fractions of the decoration cell) with owners (k, 1-based) and the
    centering translations P, I or F.  Every graph site of the cell must belong to exactly one sublattice (ValueError)."""
    tr = {"P": [[0, 0, 0]], "I": [[0, 0, 0], [0.5, 0.5, 0.5]],
          "F": [[0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0]]}.get(centering)
    if tr is None:
        raise ValueError("centering must be 'P', 'I' or 'F'")
    m = 2 * period
    pos = np.asarray(pos, dtype=float).reshape(3, -1)
    owner = np.asarray(owner, dtype=np.int64)
    tab = np.zeros((m, m, m), dtype=np.int64)
    for k in range(pos.shape[1]):
        for t in tr:
            f = np.mod(pos[:, k] + np.asarray(t, float), 1.0) * m
            h = np.mod(np.rint(f).astype(np.int64), m)
            if np.max(np.abs(f - np.rint(f))) > 1e-6 or not _on_graph(lattice, h):
                raise ValueError("a sublattice position is not a site of the graph lattice")
            if tab[h[0], h[1], h[2]] not in (0, owner[k]):
                raise ValueError("two sublattices share a site")
            tab[h[0], h[1], h[2]] = owner[k]
    pts, pcls = [], []
    for l in range(m):
        for j in range(m):
            for i in range(m):
                if not _on_graph(lattice, (i, j, l)):
                    continue
                if tab[i, j, l] == 0:
                    raise ValueError("a site of the decoration cell belongs to no sublattice")
                pts.append((i, j, l))
                pcls.append(int(tab[i, j, l]))
    pts = np.array(pts, dtype=np.int64).T
    pcls = np.array(pcls, dtype=np.int64)
    rep = -np.ones((3, ncls), dtype=np.int64)
    frac = np.zeros(ncls)
    for q in range(pts.shape[1]):
        c = pcls[q] - 1
        if rep[0, c] < 0:
            rep[:, c] = pts[:, q]
        frac[c] += 1.0
    if np.any(frac == 0.0):
        raise ValueError("a sublattice has no site")
    return Decoration(lattice=lattice, period=period, m=m, ncls=ncls, tab=tab, pts=pts, pcls=pcls, rep=rep,
                      frac=frac / pts.shape[1])


def decoration_classes(dec: Decoration, coord: np.ndarray, mg: int, origin: int) -> np.ndarray:
    """Classes (1-based) of the graph sites coord (3, n) of a periodic supercell of edge mg half-lattice units, with the
    representative site of sublattice ``origin`` (1-based) moved to the graph origin."""
    if mg % dec.m:
        raise ValueError("decoration_classes: the supercell is not a multiple of the decoration cell")
    h = np.mod(np.asarray(coord, dtype=np.int64) + dec.rep[:, origin - 1][:, None], dec.m)
    cls = dec.tab[h[0], h[1], h[2]]
    if np.any(cls == 0):
        raise ValueError("decoration_classes: graph site outside the decoration")
    return cls.astype(np.int32)


def decoration_structure(dec: Decoration) -> Structure:
    """The decoration as a crystal structure: the cell of ``period`` cubes (alat units), every graph site of the cell a
    basis site in the order of ``pts``, labelled by its sublattice."""
    return Structure(np.eye(3) * dec.period, dec.pts.astype(float) / dec.m, dec.pcls)
