"""Seeded synthetic alloys for the recursion hot path.

The reference takes its bond blocks from screened LMTO structure constants (``src/asr_lmto_alloy.f90:38-77``) and its
species parameters from the SCF (``src/asr_lmto_ham.f90``).  The workloads here replace both with seeded stand-ins of the
same shapes:

* bond blocks: two-centre Slater-Koster blocks (Slater & Koster, Phys. Rev. 94, 1498 (1954), Table I) for s, p, d in the
  reference's real-harmonic order s | y z x | xy yz 3z2-r2 xz x2-y2, nearest plus next-nearest neighbours.  They obey
  S(-v) = S(v)^T and S(gv) = D(g) S(v) D(g)^T for every cubic operation, the two properties the group-reduced operator
  needs; the on-site block is diagonal per l with a cubic e_g / t2g split;
* species parameters per (species, l): c_l in U[-0.6, 0.2] Ry, d_l in U[0.05, 0.4], Delta_l in U[0.5, 1.5] (relative
  band-width scale of the energy-dependent transform), all from ``numpy.random.default_rng(seed)``.

Parameter maps onto the operator's (c, d, o, e) of ``class_alloy_t`` (``src/asr_augcls.f90:36-43``):

* plain mode: c = c_l, d = d_l, o = 0, e = 0, so H = c + d S d (Delta_l unused);
* edc mode (``src/asr_edc.f90:41-71`` with E_nu = 0 and d_l in the role of sqrt(D_c)): for central species c,
  c_s = (Delta_c / Delta_s) c_l,s, d = d_l,c for every species (uniform), o = 0, e = 0, and the energy-dependent diagonal
  e_s(z) = z pa_s + pb_s with pa_s = 1 - Delta_c / Delta_s, pb_s = 0.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import lattices as lat

__all__ = ["sk_block", "sk_blocks", "ClassModel", "plain_params", "edc_params", "SpeciesParams", "draw_species",
           "cubic_case"]

ORB_L = np.array([0, 1, 1, 1, 2, 2, 2, 2, 2])
S3 = np.sqrt(3.0)
P3 = ("x", "y", "z")


def _sk_pair(a: str, b: str, c: dict, v: dict) -> float:
    """E_ab(v) for orbital a at the origin and b at v (unit vector with cosines c['x'], c['y'], c['z'])."""
    l, m, n = c["x"], c["y"], c["z"]
    if a == "s" and b == "s":
        return v["sss"]
    if a == "s" and b in P3:
        return c[b] * v["sps"]
    if a in P3 and b in P3:
        if a == b:
            return c[a] ** 2 * v["pps"] + (1 - c[a] ** 2) * v["ppp"]
        return c[a] * c[b] * (v["pps"] - v["ppp"])
    if a == "s":
        if b == "x2y2":
            return 0.5 * S3 * (l * l - m * m) * v["sds"]
        if b == "z2":
            return (n * n - 0.5 * (l * l + m * m)) * v["sds"]
        p, q = b[0], b[1]
        return S3 * c[p] * c[q] * v["sds"]
    if a in P3:
        if b == "x2y2":
            if a == "x":
                return 0.5 * S3 * l * (l * l - m * m) * v["pds"] + l * (1 - l * l + m * m) * v["pdp"]
            if a == "y":
                return 0.5 * S3 * m * (l * l - m * m) * v["pds"] - m * (1 + l * l - m * m) * v["pdp"]
            return 0.5 * S3 * n * (l * l - m * m) * v["pds"] - n * (l * l - m * m) * v["pdp"]
        if b == "z2":
            if a in ("x", "y"):
                return c[a] * (n * n - 0.5 * (l * l + m * m)) * v["pds"] - S3 * c[a] * n * n * v["pdp"]
            return n * (n * n - 0.5 * (l * l + m * m)) * v["pds"] + S3 * n * (l * l + m * m) * v["pdp"]
        p, q = b[0], b[1]
        if a == p or a == q:
            o = q if a == p else p
            return S3 * c[a] ** 2 * c[o] * v["pds"] + c[o] * (1 - 2 * c[a] ** 2) * v["pdp"]
        return S3 * c["x"] * c["y"] * c["z"] * v["pds"] - 2 * c["x"] * c["y"] * c["z"] * v["pdp"]
    # d-d
    eg = ("z2", "x2y2")
    if a not in eg and b not in eg:
        ap, aq = a[0], a[1]
        bp, bq = b[0], b[1]
        if {ap, aq} == {bp, bq}:
            k = ({"x", "y", "z"} - {ap, aq}).pop()
            return (3 * c[ap] ** 2 * c[aq] ** 2 * v["dds"] + (c[ap] ** 2 + c[aq] ** 2 - 4 * c[ap] ** 2 * c[aq] ** 2) * v["ddp"]
                    + (c[k] ** 2 + c[ap] ** 2 * c[aq] ** 2) * v["ddd"])
        shared = ({ap, aq} & {bp, bq}).pop()
        x1 = ({ap, aq} - {shared}).pop()
        x2 = ({bp, bq} - {shared}).pop()
        cs = c[shared]
        return (3 * c[x1] * cs * cs * c[x2] * v["dds"] + c[x1] * c[x2] * (1 - 4 * cs * cs) * v["ddp"]
                + c[x1] * c[x2] * (cs * cs - 1) * v["ddd"])
    if a in eg and b not in eg:
        return _sk_pair(b, a, c, v)   # d-d pairs are symmetric under exchange (parity +1)
    if a not in eg and b == "x2y2":
        d2 = l * l - m * m
        if a == "xy":
            return 1.5 * l * m * d2 * v["dds"] + 2 * l * m * (m * m - l * l) * v["ddp"] + 0.5 * l * m * d2 * v["ddd"]
        if a == "yz":
            return 1.5 * m * n * d2 * v["dds"] - m * n * (1 + 2 * d2) * v["ddp"] + m * n * (1 + 0.5 * d2) * v["ddd"]
        return 1.5 * n * l * d2 * v["dds"] + n * l * (1 - 2 * d2) * v["ddp"] - n * l * (1 - 0.5 * d2) * v["ddd"]
    if a not in eg and b == "z2":
        w = n * n - 0.5 * (l * l + m * m)
        if a == "xy":
            return S3 * l * m * w * v["dds"] - 2 * S3 * l * m * n * n * v["ddp"] + 0.5 * S3 * l * m * (1 + n * n) * v["ddd"]
        p, q = a[0], a[1]
        return (S3 * c[p] * c[q] * w * v["dds"] + S3 * c[p] * c[q] * (l * l + m * m - n * n) * v["ddp"]
                - 0.5 * S3 * c[p] * c[q] * (l * l + m * m) * v["ddd"])
    d2 = l * l - m * m
    if a == "x2y2" and b == "x2y2":
        return 0.75 * d2 * d2 * v["dds"] + (l * l + m * m - d2 * d2) * v["ddp"] + (n * n + 0.25 * d2 * d2) * v["ddd"]
    if a == "z2" and b == "z2":
        w = n * n - 0.5 * (l * l + m * m)
        return w * w * v["dds"] + 3 * n * n * (l * l + m * m) * v["ddp"] + 0.75 * (l * l + m * m) ** 2 * v["ddd"]
    w = n * n - 0.5 * (l * l + m * m)
    return 0.5 * S3 * d2 * w * v["dds"] + S3 * n * n * (m * m - l * l) * v["ddp"] + 0.25 * S3 * (1 + n * n) * d2 * v["ddd"]


_ORBS = ["s", "y", "z", "x", "xy", "yz", "z2", "xz", "x2y2"]
_ORBS_SK = ["s", "y", "z", "x", "xy", "yz", "z2", "zx", "x2y2"]


def sk_block(vec, ints: dict) -> np.ndarray:
    """9 x 9 block B[a, b] = E_ab(v) for the bond vector ``vec`` (orbital a at R, b at R + v)."""
    vec = np.asarray(vec, dtype=float)
    u = vec / np.linalg.norm(vec)
    c = {"x": u[0], "y": u[1], "z": u[2]}
    key = {o: k for o, k in zip(_ORBS, _ORBS_SK)}
    B = np.zeros((9, 9))
    for i, a in enumerate(_ORBS):
        for j, b in enumerate(_ORBS):
            if j < i:
                continue
            e = _sk_pair(key[a], key[b], c, ints)
            B[i, j] = e
            B[j, i] = e * (-1.0) ** (ORB_L[i] + ORB_L[j])
    return B


_INT_NAMES = ["sss", "sps", "pps", "ppp", "sds", "pds", "pdp", "dds", "ddp", "ddd"]
_INT_SIGN = np.array([-1, 1, 1, -1, -1, -1, 1, -1, 1, -1], dtype=float)


def draw_two_centre(rng: np.random.Generator, scale: float) -> dict:
    mag = rng.uniform(0.3, 1.0, size=len(_INT_NAMES))
    return {k: float(s * m * scale) for k, s, m in zip(_INT_NAMES, _INT_SIGN, mag)}


def sk_blocks(bvec: np.ndarray, seed: int, shells=None):
    """Bond blocks block(9, 9, nslot) (Fortran order) for the slots ``bvec`` (3, nslot) plus the on-site block0(9, 9).

    One set of two-centre integrals per shell (|v|^2), the NNN shell scaled by 0.4; block0 = diag per l with an
    e_g / t2g split."""
    rng = np.random.default_rng(seed)
    r2 = np.sum(bvec.astype(np.int64) ** 2, axis=0)
    shells = sorted(set(int(x) for x in r2))
    ints = {s: draw_two_centre(rng, 1.0 if i == 0 else 0.4) for i, s in enumerate(shells)}
    ns = bvec.shape[1]
    block = np.zeros((9, 9, ns), order="F")
    for k in range(ns):
        block[:, :, k] = sk_block(bvec[:, k], ints[int(r2[k])])
    on = rng.uniform(-0.2, 0.2, size=4)
    block0 = np.diag([on[0], on[1], on[1], on[1], on[2], on[2], on[3], on[2], on[3]]).copy(order="F")
    return block, block0


@dataclass
class ClassModel:
    """``class_alloy_t`` (src/asr_augcls.f90:36-43) without the species parameters: classes, species and blocks."""
    nsp: int
    nsc: np.ndarray            # (ncls,)
    spc: np.ndarray            # (ldspc, ncls) Fortran, 1-based species
    conc: np.ndarray           # (ldspc, ncls) Fortran
    block: np.ndarray          # (9, 9, nslot, ntype) Fortran
    block0: np.ndarray         # (9, 9, ntype) Fortran

    @property
    def ncls(self) -> int:
        return int(self.nsc.shape[0])

    @staticmethod
    def single_class(nsp: int, conc, block, block0) -> "ClassModel":
        conc = np.asarray(conc, dtype=float)
        spc = np.asfortranarray(np.arange(1, nsp + 1, dtype=np.int32).reshape(nsp, 1))
        return ClassModel(nsp=nsp, nsc=np.array([nsp], dtype=np.int32), spc=spc,
                          conc=np.asfortranarray(conc.reshape(nsp, 1)),
                          block=np.asfortranarray(block.reshape(9, 9, -1, 1)),
                          block0=np.asfortranarray(block0.reshape(9, 9, 1)))


@dataclass
class SpeciesParams:
    """Per-species, per-l draws: c, d, Delta (nsp, 3) for l = s, p, d."""
    c: np.ndarray
    d: np.ndarray
    delta: np.ndarray
    enu: np.ndarray = field(default=None)

    def per_orbital(self, x: np.ndarray) -> np.ndarray:
        """(nsp, 3) per l -> (9, nsp) Fortran per orbital."""
        return np.asfortranarray(x[:, ORB_L].T)


def draw_species(nsp: int, seed: int) -> SpeciesParams:
    rng = np.random.default_rng(seed)
    c = rng.uniform(-0.6, 0.2, size=(nsp, 3))
    d = rng.uniform(0.05, 0.4, size=(nsp, 3))
    delta = rng.uniform(0.5, 1.5, size=(nsp, 3))
    return SpeciesParams(c=c, d=d, delta=delta, enu=np.zeros((nsp, 3)))


def draw_o(nsp: int, seed: int, scale: float = 0.15) -> np.ndarray:
    """o_l of every species and l (nsp, 3), U[-scale, scale] from the seed (the o of the alpha representation that
    edc_setup scales to o_s = o_l D_s / D_c, src/asr_edc.f90:66)."""
    rng = np.random.default_rng(1000 + seed)
    return rng.uniform(-scale, scale, size=(nsp, 3))


def edc_params_o(sp: SpeciesParams, ol: np.ndarray, central: int):
    """``edc_params`` with the o of edc_setup: o(l, s) = o_l,s D_s / D_c (src/asr_edc.f90:66), (9, nsp) Fortran."""
    ed = edc_params(sp, central)
    o = sp.per_orbital(ol)
    de = ed["dl"]
    ed["o"] = np.asfortranarray(o * de / ed["dc"][:, None])
    return ed


def plain_params(sp: SpeciesParams):
    """(c, d, o, e) each (9, nsp) Fortran: H = c + d S d."""
    c = sp.per_orbital(sp.c)
    d = sp.per_orbital(sp.d)
    z = np.zeros_like(c, order="F")
    return c, d, z.copy(order="F"), z.copy(order="F")


def edc_params(sp: SpeciesParams, central: int):
    """edc form for central species ``central`` (1-based): (c, d, o, e, pa, pb) each (9, nsp), plus (dc, del, enu)."""
    c = sp.per_orbital(sp.c)
    d = sp.per_orbital(sp.d)
    de = sp.per_orbital(sp.delta)
    en = sp.per_orbital(sp.enu)
    dc = de[:, central - 1].copy()
    cc = np.asfortranarray(dc[:, None] / de * c)
    dd = np.asfortranarray(np.repeat(d[:, central - 1:central], d.shape[1], axis=1))
    o = np.zeros_like(cc, order="F")
    e = np.zeros_like(cc, order="F")
    pa = np.asfortranarray(1.0 - dc[:, None] / de)
    pb = np.asfortranarray(dc[:, None] * en / de)
    return dict(c=cc, d=dd, o=o, e=e, pa=pa, pb=pb, dc=dc, dl=np.asfortranarray(de), enu=np.asfortranarray(en))


def ed3_params(sp: SpeciesParams, central: int, o=None, p=None):
    """Route ed3 (``ed3_setup``, src/asr_edc.f90's sibling src/asr_ed3.f90:57-79) for central species ``central``: with
    D_s = Delta_l,s, g_s = (D_c / D_s) c_l,s (c as C - E_nu), d = d_l of the central species in the role of D_c^1/2 (as
    in the edc mapping), and the alpha-representation o_s, p_s per (species, l) (``o``, ``p`` (nsp, 3); default 0).
    Returns the group dict of ``chains.ed3_blocks`` (start_orb and nlev to be added)."""
    nsp = sp.c.shape[0]
    o = np.zeros((nsp, 3)) if o is None else np.asarray(o, float)
    p = np.zeros((nsp, 3)) if p is None else np.asarray(p, float)
    c, d, de, en = (sp.per_orbital(x) for x in (sp.c, sp.d, sp.delta, sp.enu))
    dc = de[:, central - 1].copy()
    return dict(g=np.asfortranarray(dc[:, None] / de * c), d=np.asfortranarray(np.repeat(d[:, central - 1:central], nsp, axis=1)),
                dc=dc, dl=np.asfortranarray(de), enu=np.asfortranarray(en), o=sp.per_orbital(o), p=sp.per_orbital(p),
                central=central)


def cubic_case(kind: str, l: int, nsp: int, conc, seed: int, group: str = "d2h", r2max: int | None = None):
    """A one-class cubic alloy: graph, group (perm, dmat), model with Slater-Koster blocks.

    ``group``: 'd2h' (all nine orbitals one dimensional), 'd4h' (class_ops), 'identity' (unreduced)."""
    if r2max is None:
        r2max = {"bcc": 4, "fcc": 4, "sc": 8}[kind]   # NN + NNN (bcc 8 + 6, fcc 12 + 6, sc 6 + 12)
    g, coord, bvec = lat.periodic_graph_shells(kind, l, r2max)
    cls = np.ones(g.n, dtype=np.int32)
    if group == "d2h":
        perm, mats = lat.d2h_ops(coord, 2 * l, cls)
        dmat = lat.orbital_rep(mats)
    elif group == "d4h":
        perm, mats = lat.class_ops(coord, 2 * l, cls)
        dmat = lat.orbital_rep(mats)
    elif group == "identity":
        perm, dmat = lat.identity_group(g.n)
    else:
        raise ValueError(group)
    block, block0 = sk_blocks(bvec, seed)
    mdl = ClassModel.single_class(nsp, conc, block, block0)
    return dict(graph=g, coord=coord, bvec=bvec, cls=cls, perm=np.asfortranarray(perm, dtype=np.int32),
                dmat=np.asfortranarray(dmat), model=mdl)


def batched_ternary_workload():
    """The batched, uneven-depth configuration: fcc ternary Fe0.66Ni0.14Cr0.20-like random alloy on a 5^3-cell periodic
    cluster (NN + NNN Slater-Koster blocks, 18 slots), one site class, D2h reduction (the operator is built from start
    site 1 to 3 levels at rank 1, the start site not flippable); 2 spins x 3 central species x 9 start orbitals = 54 chain
    groups in the edc form (``edc_params``) with depths drawn from U{16..28} (seed 1); energies: the 48-point
    Gauss-Legendre semicircle over [-1.2, 0.3] (the node rule of contour_nodes, src/asr_contour.f90:17-34) followed by
    4096 real-axis energies on [-1.5, 1.0] + 0.005i.  Returns (case, flippable, groups, z), groups as dicts of ed, cen,
    l0, nlev in the order (spin, central species, start orbital)."""
    case = cubic_case("fcc", 5, 3, [0.66, 0.14, 0.20], seed=1, group="d2h")
    fl = np.ones(case["graph"].n, np.int32)
    fl[0] = 0
    rng = np.random.default_rng(1)
    depths = rng.integers(16, 29, size=54)
    groups = []
    for spin in range(2):
        sp = draw_species(3, seed=1 + spin)
        for cen in (1, 2, 3):
            ed = edc_params(sp, cen)
            for l0 in range(1, 10):
                groups.append(dict(ed=ed, cen=cen, l0=l0, nlev=int(depths[len(groups)]), spin=spin))
    ebot, ef = -1.2, 0.3
    x, _ = np.polynomial.legendre.leggauss(48)
    th = 0.5 * np.pi * (1.0 - x)
    zc = 0.5 * (ebot + ef) + 0.5 * (ef - ebot) * np.exp(1j * th)
    zr = np.linspace(-1.5, 1.0, 4096) + 0.005j
    return case, fl, groups, np.concatenate([zc, zr])


# L2_1 (Heusler-like) decoration of bcc: four fcc sublattices.  Sites of the bcc grid have i, j, k all even or all odd
# (half-lattice units); even sites split by (i + j + k) / 2 mod 2, odd sites by (i + j + k - 3) / 2 mod 2.
HEUSLER_SHIFT = ((0, 0, 0), (2, 0, 0), (1, 1, 1), (3, 1, 1))   # a site of sublattice 1..4 relative to sublattice 1


def heusler_sublattice(coord: np.ndarray) -> np.ndarray:
    """Sublattice 1..4 of every bcc site (3, n)."""
    s = coord.sum(axis=0)
    odd = (coord[0] % 2).astype(np.int64)
    half = np.where(odd == 1, (s - 3) // 2, s // 2) % 2
    return (1 + 2 * odd + half).astype(np.int32)


def heusler_case(l: int = 4, seed: int = 3, sublattice: int = 1, maxlevel: int = 3, maxrank: int = 1):
    """L2_1 four-sublattice bcc cell with sublattices 1-3 ordered (species 1, 2, 3) and sublattice 4 disordered
    (species 4 and 5 at 0.6 / 0.4, Cr0.6Fe0.4-like); NN + NNN Slater-Koster blocks.  The site classes are shifted so
    that site 1 (the origin, the start of the recursion) lies on ``sublattice``; the group is the class-preserving
    diagonal subgroup (D2 here: all nine orbitals one dimensional)."""
    if l % 2:
        raise ValueError("heusler_case: l must be even for a periodic L2_1 decoration")
    g, coord, bvec = lat.periodic_graph_shells("bcc", l, 4)
    shift = np.asarray(HEUSLER_SHIFT[sublattice - 1], dtype=np.int64)[:, None]
    cls = heusler_sublattice(coord + shift)
    perm, mats = lat.d2h_ops(coord, 2 * l, cls)
    dmat = lat.orbital_rep(mats)
    block, block0 = sk_blocks(bvec, seed)
    nsc = np.array([1, 1, 1, 2], dtype=np.int32)
    spc = np.asfortranarray(np.array([[1, 0], [2, 0], [3, 0], [4, 5]], dtype=np.int32).T)
    conc = np.asfortranarray(np.array([[1.0, 0.0], [1.0, 0.0], [1.0, 0.0], [0.6, 0.4]]).T)
    mdl = ClassModel(nsp=5, nsc=nsc, spc=spc, conc=conc, block=np.asfortranarray(block.reshape(9, 9, -1, 1)),
                     block0=np.asfortranarray(block0.reshape(9, 9, 1)))
    fl = np.ones(g.n, np.int32)
    fl[0] = 0
    return dict(graph=g, coord=coord, bvec=bvec, cls=cls, perm=np.asfortranarray(perm, dtype=np.int32),
                dmat=np.asfortranarray(dmat), model=mdl, maxlevel=maxlevel, maxrank=maxrank, flippable=fl,
                sublattice=sublattice)


# The operator inputs of the reference's shipped examples (example/*.toml): bcc graph (NN + NNN, the structure-constant
# range 1.2 a_bcc) on a periodic cluster large enough for the closure, class-preserving operations with the z axis kept
# (the monomial reduction group under which the start orbitals are one dimensional), the start site not flippable.
# The augmented-space node counts of these inputs are printed by the reference ("nodes / sublattice" of
# example/reference/*/asr.out).
EXAMPLES = {
    # name: (lattice, cluster l, levels, classes of the sublattices, species per class, concentrations per class)
    "cuzn_alloy": ("bcc", 8, 4, ("a2",), ((1, 2),), ((0.5, 0.5),)),
    "fe66ni14cr20_fcc": ("fcc", 8, 3, ("fcc",), ((1, 2, 3),), ((0.66, 0.14, 0.20),)),
    "cuzn_b2": ("bcc", 12, 4, ("b2_a", "b2_b"), ((1,), (2,)), ((1.0,), (1.0,))),
    "co2fe04cr06al_l21": ("bcc", 8, 4, ("l21_8c", "l21_4a", "l21_4b"), ((1,), (2,), (3, 4)), ((1.0,), (1.0,), (0.4, 0.6))),
}
_EXAMPLE_SHIFT = {"a2": (0, 0, 0), "fcc": (0, 0, 0), "b2_a": (0, 0, 0), "b2_b": (1, 1, 1),
                  "l21_8c": (1, 1, 1), "l21_4a": (0, 0, 0), "l21_4b": (2, 0, 0)}


def _example_classes(kind: str, coord: np.ndarray, shift) -> np.ndarray:
    c = coord + np.asarray(shift, dtype=np.int64)[:, None]
    if kind in ("a2", "fcc"):
        return np.ones(coord.shape[1], np.int32)
    odd = (c[0] % 2).astype(np.int64)
    if kind.startswith("b2"):
        return (1 + odd).astype(np.int32)          # 1: cube corners, 2: cube centres
    half = (c.sum(axis=0) // 2) % 2
    return np.where(odd == 1, 1, np.where(half == 0, 2, 3)).astype(np.int32)   # 1: 8c, 2: 4a, 3: 4b


def example_case(name: str, sublattice: int = 1, seed: int = 0, l: int | None = None):
    """Operator inputs of the reference example ``name`` with the start site on ``sublattice`` (1-based): the cluster is
    shifted so that site 1 lies on that sublattice and every site keeps the class of its sublattice in the example's
    class list; returns the case dict of ``cubic_case`` plus maxlevel.
    ``l`` overrides the periodic cluster (the examples' own: the supercell their published runs used)."""
    kind, l0, levels, cnames, spcs, concs = EXAMPLES[name]
    l = l0 if l is None else l
    g, coord, bvec = lat.periodic_graph_shells(kind, l, 4)
    cname = cnames[sublattice - 1]
    cls = _example_classes(cname, coord, _EXAMPLE_SHIFT[cname])
    # the shift puts site 1 on the start sublattice; the classes keep the example's labels (B2: 1 = cube corners a,
    # 2 = cube centres b)
    perm, mats = lat.class_ops(coord, 2 * l, cls)
    dmat = lat.orbital_rep(mats)
    block, block0 = sk_blocks(bvec, seed)
    ncls = len(cnames)
    ld = max(len(s) for s in spcs)
    spc = np.zeros((ld, ncls), np.int32, order="F")
    conc = np.zeros((ld, ncls), order="F")
    for k in range(ncls):
        spc[: len(spcs[k]), k] = spcs[k]
        conc[: len(concs[k]), k] = concs[k]
    nsp = int(max(max(s) for s in spcs))
    mdl = ClassModel(nsp=nsp, nsc=np.array([len(s) for s in spcs], np.int32), spc=spc, conc=conc,
                     block=np.asfortranarray(block.reshape(9, 9, -1, 1)), block0=np.asfortranarray(block0.reshape(9, 9, 1)))
    fl = np.ones(g.n, np.int32)
    fl[0] = 0
    return dict(graph=g, coord=coord, bvec=bvec, cls=cls, perm=np.asfortranarray(perm, dtype=np.int32), dmat=np.asfortranarray(dmat),
                model=mdl, maxlevel=levels, maxrank=1, flippable=fl)


def structure_blocks(bvec: np.ndarray, seed: int, ntype: int = 1):
    """Bond blocks for float bond vectors (alat units): one set of two-centre integrals per shell of equal length, the
    shells after the first scaled by 0.4; the same blocks for every translation type.  block (9, 9, nslot, ntype),
    block0 (9, 9, ntype), Fortran order."""
    rng = np.random.default_rng(seed)
    r2 = np.round(np.sum(np.asarray(bvec, float) ** 2, axis=0), 6)
    shells = sorted(set(float(x) for x in r2))
    ints = {s: draw_two_centre(rng, 1.0 if i == 0 else 0.4) for i, s in enumerate(shells)}
    ns = bvec.shape[1]
    block = np.zeros((9, 9, ns, ntype), order="F")
    for k in range(ns):
        block[:, :, k, :] = sk_block(bvec[:, k], ints[float(r2[k])])[:, :, None]
    on = rng.uniform(-0.2, 0.2, size=4)
    b0 = np.diag([on[0], on[1], on[1], on[1], on[2], on[2], on[3], on[2], on[3]])
    block0 = np.asfortranarray(np.repeat(b0[:, :, None], ntype, axis=2))
    return block, block0


# the structures of the reference examples as their inputs give them: graph lattice, period of the decoration cell in
# conventional cubes, centering, and the Wyckoff positions (fractions of the decoration cell) of each sublattice, in the
# order of the examples' sublattices; with the recursion levels of each example
EXAMPLE_DECORATIONS = {
    "cuzn_alloy": ("bcc", 1, "I", [[(0.0, 0.0, 0.0)]], 4),
    "fe66ni14cr20_fcc": ("fcc", 1, "F", [[(0.0, 0.0, 0.0)]], 3),
    "cuzn_b2": ("bcc", 1, "P", [[(0.0, 0.0, 0.0)], [(0.5, 0.5, 0.5)]], 4),
    "co2fe04cr06al_l21": ("bcc", 2, "F", [[(0.25, 0.25, 0.25), (0.75, 0.75, 0.75)], [(0.0, 0.0, 0.0)], [(0.5, 0.5, 0.5)]], 4),
}


def example_structure(name: str):
    """The Structure of reference example ``name``: its decoration cell (``crystal.decoration_build``) as the cell, every
    graph site of the cell a basis site labelled by its sublattice."""
    from . import crystal as X
    lattice, period, centering, subl, _ = EXAMPLE_DECORATIONS[name]
    pos = np.array([p for sl in subl for p in sl], dtype=float).T
    owner = [k + 1 for k, sl in enumerate(subl) for _ in sl]
    dec = X.decoration_build(lattice, period, centering, pos, owner, len(subl))
    return X.decoration_structure(dec)


def structure_case(name: str, sublattice: int = 1, seed: int = 0, rcl: float = 1.2, levels: int | None = None,
                   group: str = "reduction"):
    """Operator inputs of reference example ``name`` built from its structure alone (crystal.sublattice_inputs): the
    ball about the start site, the class-preserving site group, its start orbitals and weights, and the reduction group.
    Returns the keys of ``example_case`` plus reps, weights, stype and the crystal graph."""
    from . import crystal as X
    lev = EXAMPLE_DECORATIONS[name][4]
    levels = lev if levels is None else levels
    spcs, concs = EXAMPLES[name][4], EXAMPLES[name][5]
    s = example_structure(name)
    ops = X.space_group(s)
    inp = X.sublattice_inputs(s, ops, sublattice, rcl, levels, group=group)
    _, ntype = X.translation_types(s)
    block, block0 = structure_blocks(inp["cg"].bvec, seed, ntype)
    ncls = len(spcs)
    ld = max(len(x) for x in spcs)
    spc = np.zeros((ld, ncls), np.int32, order="F")
    conc = np.zeros((ld, ncls), order="F")
    for k in range(ncls):
        spc[: len(spcs[k]), k] = spcs[k]
        conc[: len(concs[k]), k] = concs[k]
    nsp = int(max(max(x) for x in spcs))
    mdl = ClassModel(nsp=nsp, nsc=np.array([len(x) for x in spcs], np.int32), spc=spc, conc=conc, block=block, block0=block0)
    return dict(graph=inp["graph"], cls=inp["cls"], perm=inp["perm"], dmat=inp["dmat"], model=mdl, maxlevel=levels, maxrank=1,
                flippable=inp["flippable"], stype=inp["stype"], reps=inp["reps"], weights=inp["weights"], cg=inp["cg"],
                site_group=inp["site_group"])
