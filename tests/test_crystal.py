"""Structure clusters and their symmetry (asr_b200.crystal) against the reference's own expectations:
test/test_crystal_symmetry.f90 (space-group and site-group orders, monomial operations, orbital groups, representatives,
reduction-group orders for seven prototypes) and test/test_crystal_graph.f90 (cubic slots in the order of the periodic
shell graphs, the ball of radius 2 levels b_max, the 48 site operations in cubic-table order, slot / size / operation
consistency, B2 = bcc site by site, hcp and NiAs shells, rmin and levels 0)."""
import numpy as np
import pytest

from asr_b200 import crystal as X
from asr_b200 import lattices as lat

CUBIC_GRP = [1, 2, 2, 2, 3, 3, 4, 3, 4]      # s | p y z x | xy yz 3z2 xz x2-y2
HEX_GRP = [1, 2, 3, 2, 4, 5, 6, 5, 4]        # s | p_xy, p_z | d_xy,x2-y2 | d_yz,xz | d_3z2
CA_IDEAL = 1.632993161855452


@pytest.mark.parametrize("name,ca,nsg,nsite,nmono,ngrp,nred,grp_ref,rep_ref", [
    ("sc", None, 48, [48], [48], 4, 16, CUBIC_GRP, [1, 3, 5, 7]),
    ("bcc", None, 48, [48], [48], 4, 16, CUBIC_GRP, [1, 3, 5, 7]),
    ("fcc", None, 48, [48], [48], 4, 16, CUBIC_GRP, [1, 3, 5, 7]),
    ("b2", None, 48, [48, 48], [48, 48], 4, 16, CUBIC_GRP, [1, 3, 5, 7]),
    ("hex", 1.6, 24, [24], [8], 6, 8, HEX_GRP, None),
    ("hcp", None, 24, [12, 12], [4, 4], 6, 4, HEX_GRP, None),
    ("nias", 1.617, 24, [12, 12, 12, 12], [4, 4, 4, 4], 6, 4, HEX_GRP, None),
])
def test_prototype_symmetry(name, ca, nsg, nsite, nmono, ngrp, nred, grp_ref, rep_ref):
    s = X.prototype_structure(name, ca)
    ops = X.space_group(s)
    assert len(ops) == nsg
    assert np.array_equal(ops[0].m, np.eye(3, dtype=np.int64)) and np.allclose(ops[0].t, 0.0)
    # the integer action on the basis sites equals the Cartesian one
    for o in ops:
        for b in range(s.nb):
            r = o.rot @ s.tau[:, b] + s.avec @ o.t - s.tau[:, o.perm[b]] - s.avec @ o.shift[:, b]
            assert np.max(np.abs(r)) < 1e-10
    for b in range(s.nb):
        idx = X.site_ops(ops, b)
        assert len(idx) == nsite[b]
        d = np.stack([X.orbital_matrix(ops[k].rot) for k in idx], axis=2)
        mono = np.array([X.is_monomial(ops[k].rot) for k in idx])
        for k in range(d.shape[2]):
            assert np.max(np.abs(d[:, :, k].T @ d[:, :, k] - np.eye(9))) < 1e-10
        assert mono.sum() == nmono[b]
        grp, ng, rep, wgt = X.orbital_groups(d, mono)
        assert ng == ngrp and list(grp) == grp_ref and wgt.sum() == 9
        if rep_ref is not None:
            assert list(rep) == rep_ref
        assert len(X.reduction_ops(d, mono, rep)) == nred


def _lattice_ball(kind, radius):
    """Cubic lattice points within radius (alat) in half-lattice integers, ordered by r^2, then z, y, x."""
    m = int(2 * radius) + 2
    r = np.arange(-m, m + 1)
    i, j, k = np.meshgrid(r, r, r, indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    on = {"sc": (i % 2 == 0) & (j % 2 == 0) & (k % 2 == 0), "bcc": (i % 2 == j % 2) & (j % 2 == k % 2),
          "fcc": (i + j + k) % 2 == 0}[kind]
    r2 = i * i + j * j + k * k
    on &= r2 <= int(np.floor(4 * radius * radius + 1e-9))
    i, j, k, r2 = i[on], j[on], k[on], r2[on]
    o = np.lexsort((i, j, k, r2))
    return np.stack([i[o], j[o], k[o]])


def _find_slot(cg, v):
    for k in range(cg.nslot):
        if np.max(np.abs(cg.bvec[:, k] - v)) < 1e-9:
            return k
    return -1


def _nbr(cg):
    return np.asarray(cg.g.nbr).reshape(cg.n, cg.nslot)


def _slot_checks(s, cg):
    nbr = _nbr(cg)
    for k in range(cg.nslot):
        for b in range(cg.nb):
            if cg.btgt[k, b]:
                v = s.avec @ (cg.bdn[:, k, b] + s.frac[:, cg.btgt[k, b] - 1] - s.frac[:, b])
                assert np.max(np.abs(v - cg.bvec[:, k])) < 1e-12
    back = [_find_slot(cg, -cg.bvec[:, k]) for k in range(cg.nslot)]
    for i in range(cg.n):
        b = cg.basis[i]
        assert X.graph_site(cg, cg.cell[:, i], b) == i + 1
        v = s.avec @ (cg.cell[:, i] + s.frac[:, b] - s.frac[:, cg.b0])
        assert np.max(np.abs(v - cg.disp[:, i])) < 1e-12
        for k in range(cg.nslot):
            j = nbr[i, k]
            assert (j == 0) == (cg.btgt[k, b] == 0)
            if j == 0:
                continue
            t = X.graph_site(cg, cg.cell[:, i] + cg.bdn[:, k, b], cg.btgt[k, b] - 1)
            if j == -1:
                assert t == 0 and np.linalg.norm(cg.disp[:, i] + cg.bvec[:, k]) > cg.radius + X.RTOL
                continue
            assert j == t and cg.basis[j - 1] == cg.btgt[k, b] - 1
            assert np.max(np.abs(cg.disp[:, j - 1] - cg.disp[:, i] - cg.bvec[:, k])) < 1e-12
            assert back[k] >= 0 and nbr[j - 1, back[k]] == i + 1


def _size_checks(cg):
    dist = X.graph_distances(cg.g, 1)
    nbr = _nbr(cg)
    inner = (dist >= 0) & (dist <= 2 * cg.levels - 1)
    assert np.all(nbr[inner] >= 0)
    assert np.any(nbr == -1)


def _op_checks(s, cg, ops):
    perm, rot, _ = X.graph_site_ops(cg, s, ops)
    nbr = _nbr(cg)
    for g in range(perm.shape[1]):
        kmap = np.array([_find_slot(cg, rot[:, :, g] @ cg.bvec[:, k]) for k in range(cg.nslot)])
        assert np.all(kmap >= 0)
        p = perm[:, g] - 1
        assert np.max(np.abs(cg.disp[:, p] - rot[:, :, g] @ cg.disp)) < 1e-12
        j = nbr
        j2 = nbr[p][:, kmap]
        want = np.where(j <= 0, j, perm[np.maximum(j, 1) - 1, g])
        assert np.array_equal(j2, want)
    assert np.all(perm[0, :] == 1)


@pytest.mark.parametrize("kind,rcl,levels", [("sc", 1.2, 3), ("bcc", 1.2, 2), ("bcc", 1.45, 2), ("fcc", 1.2, 2), ("fcc", 0.75, 3)])
def test_cubic_graph(kind, rcl, levels):
    s = X.prototype_structure(kind)
    ops = X.space_group(s)
    cg = X.crystal_graph(s, ops, rcl, levels)
    _, _, bv = lat.periodic_graph_shells(kind, 4, int((2.0 * rcl) ** 2 + 1e-9))
    assert cg.nslot == bv.shape[1]
    assert np.array_equal(cg.bvec, 0.5 * bv)
    assert abs(cg.radius - 2.0 * levels * np.max(np.linalg.norm(cg.bvec, axis=0))) < 1e-14
    ball = _lattice_ball(kind, cg.radius)
    assert ball.shape[1] == cg.n and np.array_equal(0.5 * ball, cg.disp)
    assert np.all(np.asarray(cg.g.nbr) != 0)
    g2, coord = lat.periodic_graph(kind, 2)
    _, m48 = lat.cubic_site_perms(coord, 4)
    perm, rot, _ = X.graph_site_ops(cg, s, ops)
    assert perm.shape[1] == 48 and np.array_equal(rot, m48.astype(float))
    _slot_checks(s, cg)
    _size_checks(cg)
    _op_checks(s, cg, ops)


def test_b2_graph_is_the_bcc_graph():
    sb = X.prototype_structure("bcc")
    opsb = X.space_group(sb)
    cgb = X.crystal_graph(sb, opsb, 1.2, 2)
    permb, _, _ = X.graph_site_ops(cgb, sb, opsb)
    s = X.prototype_structure("b2")
    ops = X.space_group(s)
    for b0 in (0, 1):
        cg = X.crystal_graph(s, ops, 1.2, 2, start=b0)
        assert cg.n == cgb.n and np.array_equal(cg.disp, cgb.disp) and np.array_equal(cg.g.nbr, cgb.g.nbr)
        assert np.array_equal(cg.basis, (np.rint(2.0 * cg.disp[0]).astype(np.int64) + b0) % 2)
        assert cg.norbit == 2
        perm, _, _ = X.graph_site_ops(cg, s, ops)
        assert perm.shape[1] == 48 and np.array_equal(perm, permb)
        _slot_checks(s, cg)
        _size_checks(cg)
        _op_checks(s, cg, ops)


@pytest.mark.parametrize("ca,nshell,nsecond", [(CA_IDEAL, 12, 0), (1.7, 6, 6)])
def test_hcp_graph(ca, nshell, nsecond):
    s = X.prototype_structure("hcp", ca)
    ops = X.space_group(s)
    cg = X.crystal_graph(s, ops, 1.05, 2)
    assert cg.norbit == 1
    length = np.linalg.norm(cg.bvec, axis=0)
    for b in range(2):
        have = cg.btgt[:, b] > 0
        d1 = length[have].min()
        n1 = int(np.sum(have & (np.abs(length - d1) < 1e-9)))
        assert (n1, int(have.sum()) - n1) == (nshell, nsecond)
    assert cg.nslot == 18 and np.all(np.sum(cg.btgt > 0, axis=0) == 12)
    perm, rot, _ = X.graph_site_ops(cg, s, ops)
    mono = [X.is_monomial(rot[:, :, i]) for i in range(rot.shape[2])]
    assert perm.shape[1] == 12 and sum(mono) == 4 and all(mono[:4])
    _slot_checks(s, cg)
    _size_checks(cg)
    _op_checks(s, cg, ops)


def test_nias_graph():
    s = X.prototype_structure("nias", 1.617)
    ops = X.space_group(s)
    for b in range(4):
        cg = X.crystal_graph(s, ops, 0.9, 2, start=b)
        assert cg.norbit == 2
        have = cg.btgt[:, b] > 0
        length = np.linalg.norm(cg.bvec, axis=0)
        dmin = length[have].min()
        lab = s.label[np.maximum(cg.btgt[:, b] - 1, 0)]
        other = have & (lab != s.label[b])
        same = have & (lab == s.label[b])
        nte = int(np.sum(other & (np.abs(length - dmin) < 1e-9)))
        counts = (nte, int(same.sum()), int(other.sum()) - nte)
        assert counts == ((6, 2, 0) if s.label[b] == 1 else (6, 0, 0))
        perm, _, _ = X.graph_site_ops(cg, s, ops)
        assert perm.shape[1] == 12
        _slot_checks(s, cg)
        _size_checks(cg)
        _op_checks(s, cg, ops)


def test_rmin_and_levels_zero():
    s = X.prototype_structure("fcc")
    ops = X.space_group(s)
    cg = X.crystal_graph(s, ops, 0.75, 1, rmin=3.1)
    assert abs(cg.radius - 3.1) < 1e-14 and cg.n == _lattice_ball("fcc", 3.1).shape[1]
    cg = X.crystal_graph(s, ops, 0.75, 0)
    assert cg.n == 1 and np.all(np.asarray(cg.g.nbr) == -1)


def test_sublattice_inputs_of_the_l21_cell():
    """The L2_1 cell from its decoration: the 8c site group is T_d (24 operations, class-preserving), the 4a and 4b site
    groups O_h (48); four start orbitals s, p_z, d_xy, d_3z2 with weights 1, 3, 3, 2 on each, reduction groups of
    order 8 (8c) and 16 (4a, 4b)."""
    from asr_b200 import synthetic as S
    s = S.example_structure("co2fe04cr06al_l21")
    ops = X.space_group(s)
    assert s.nb == 16               # the decoration cell of the example: 2^3 conventional bcc cubes, 16 sites
    assert len(ops) == 48 * 4       # Fm-3m on that cell: 48 point operations x 4 centring translations
    for kap, nsite, nred in ((1, 24, 8), (2, 48, 16), (3, 48, 16)):
        inp = X.sublattice_inputs(s, ops, kap, 1.2, 1)
        assert inp["site_group"] == nsite and inp["perm"].shape[1] == nred
        assert list(inp["reps"]) == [1, 3, 5, 7] and list(inp["weights"]) == [1, 3, 3, 2]
        assert inp["cls"][0] == kap and inp["flippable"][0] == 0


def test_decorations():
    """Decoration cells (src/asr_sublattice.f90:39-116): the L2_1 cell of its example (16 sites, fractions 1/2, 1/4, 1/4),
    classes of a periodic supercell with the origin moved to a sublattice, and the input errors."""
    d = X.decoration_build("bcc", 2, "F", np.array([[0.25, 0.75, 0.0, 0.5]] * 3), [1, 1, 2, 3], 3)
    assert d.pts.shape[1] == 16 and np.allclose(d.frac, [0.5, 0.25, 0.25])
    g, coord, _ = lat.periodic_graph_shells("bcc", 4, 4)
    for origin in (1, 2, 3):
        cls = X.decoration_classes(d, coord, 8, origin)
        assert cls[0] == origin and np.allclose(np.bincount(cls)[1:] / cls.size, d.frac)
    with pytest.raises(ValueError, match="share a site"):
        X.decoration_build("bcc", 1, "P", np.array([[0.0, 0.0], [0.0, 0.0], [0.0, 0.0]]), [1, 2], 2)
    with pytest.raises(ValueError, match="no sublattice"):
        X.decoration_build("bcc", 1, "P", np.zeros((3, 1)), [1], 1)
    with pytest.raises(ValueError, match="centering"):
        X.decoration_build("bcc", 1, "C", np.zeros((3, 1)), [1], 1)


@pytest.mark.parametrize("kind,sub", [("bcc", 1), ("fcc", 1)])
def test_decoration_and_primitive_cells_give_the_same_operator_inputs(kind, sub):
    """A sublattice's operator inputs do not depend on the cell the structure is written in: the conventional cube with
    its centring sites and the primitive cell give the same ball, classes, group and start orbitals."""
    d = X.decoration_build(kind, 1, "I" if kind == "bcc" else "F", np.zeros((3, 1)), [1], 1)
    sd, sp = X.decoration_structure(d), X.prototype_structure(kind)
    a = X.sublattice_inputs(sd, X.space_group(sd), sub, 1.2, 2)
    b = X.sublattice_inputs(sp, X.space_group(sp), sub, 1.2, 2)
    for k in ("cls", "perm", "dmat", "flippable", "stype", "reps", "weights"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
    assert np.array_equal(a["graph"].nbr, b["graph"].nbr)
