"""Effective pair interactions: the pair group, the symmetry-adapted start vectors and the chain trace formula of the
oracle (epi_setup, epi_start, epi_blocks, epi_integrand restated) against the exact configuration average of
Tr[G dH/dlambda] over the random sites of a 16-site cell (dense matrices, no recursion), after the reference's
test/test_epi.f90 parts (G) and (D)."""
import numpy as np
import pytest

from asr_b200 import epi as EP
from asr_b200 import lattices as lat
from oracle.oracle import OracleOp
from tests import epi_case as E

Z = 0.12 + 0.3j
LAM = 0.35


def test_pair_group_and_adapted_vectors():
    c = E.cell()
    mdl, cls, fl = E.chain_model(c)
    perm, mats = EP.epi_pair_ops(c["coord"], E.MG, cls)
    assert perm.shape[1] == 2                      # the two random sites are related by the mirror x <-> y
    vec, chi, lo = EP.epi_adapted(lat.orbital_rep(mats))
    assert np.max(np.abs(vec.T @ vec - np.eye(9))) < 1e-13
    d = lat.orbital_rep(mats)
    for a in range(9):
        for g in range(d.shape[2]):
            assert np.max(np.abs(d[:, :, g] @ vec[:, a] - chi[g, a] * vec[:, a])) < 1e-12
    assert int(np.sum(chi[1] > 0)) == 6 and list(lo) == [1, 2, 2, 2, 5, 5, 5, 5, 5]


def test_exchange_skip_mirror():
    u = np.arange(9.0).reshape(3, 3)
    v = EP.epi_exchange(u)
    assert np.allclose(v, v.T) and np.all(np.diag(v) == 0) and v[0, 1] == u[0, 0] + u[1, 1] - u[0, 1] - u[1, 0]
    assert EP.epi_skip(True, True, 3, 2) and not EP.epi_skip(True, True, 3, 1) and not EP.epi_skip(True, True, 2, 3)
    assert not EP.epi_skip(False, True, 3, 2) and not EP.epi_skip(True, False, 3, 2)
    m = EP.epi_mirror(u)
    assert m[2, 1] == u[1, 2] and np.all(m[:, 0] == u[:, 0]) and np.all(m[1] == u[1])


@pytest.mark.parametrize("group", ["pair", "identity"])
def test_oracle_chain_trace_equals_the_exact_configuration_average(group):
    c = E.cell()
    par = E.species()
    mdl, cls, fl = E.chain_model(c)
    if group == "pair":
        perm, mats = EP.epi_pair_ops(c["coord"], E.MG, cls)
        d = lat.orbital_rep(mats)
    else:
        perm, d = lat.identity_group(c["graph"].n)
    op = OracleOp(c["graph"], mdl, cls, perm, d, 1, 8, 2, fl)
    if group == "identity":
        assert op.nn == 9 * c["graph"].n           # 16 sites x 9 configurations of the random pair: complete
    vec, chi, lo = EP.epi_adapted(d)
    pt = EP.epi_path(par[0], par[1], LAM)
    params, ed = EP.epi_setup(par, pt)
    for sj in (2, 3):
        ref = E.exact_trace(c, par, 1, 2, LAM, sj, Z)
        op.set_params(*params)
        op.unfreeze()
        op.freeze_any(1, 4)
        op.freeze_any(c["jp"], sj)
        tr = 0.0
        for ia in range(9):
            op.set_chi(chi[: op.nop, ia])
            x, _ = op.epi_blocks(ed, vec[:, ia], Z, 100, tail="none")
            tr += EP.epi_integrand(pt, int(lo[ia]), Z, x)
        # epi_integrand leaves out the constant -2 kappa: it equals the exact trace plus 2 sum_L kappa_L
        assert abs(tr - ref) / abs(ref) < 1e-8, (sj, tr, ref)


def test_pair_lists_on_periodic_cubic_cells():
    """Part (G) of the reference's test: pair types, multiplicities, lengths, pair-group orders; a shell that does not fit
    into the cell is refused; B2 partners on the other and the own sublattice."""
    c = E.cell()
    cls = np.ones(c["graph"].n, np.int64)
    pairs = EP.epi_pair_list(c["coord"], E.MG, cls, 1)
    assert len(pairs) == 1 and (pairs[0].mult, pairs[0].r2, pairs[0].nop) == (8, 3, 2)
    with pytest.raises(ValueError, match="does not fit"):
        EP.epi_pair_list(c["coord"], E.MG, cls, 2)
    gf, cf = lat.periodic_graph("fcc", 2)
    pairs = EP.epi_pair_list(cf, 4, np.ones(gf.n, np.int64), 1)
    assert len(pairs) == 1 and (pairs[0].mult, pairs[0].nop) == (12, 4)
    g3, c3 = lat.periodic_graph("bcc", 3)
    pairs = EP.epi_pair_list(c3, 6, np.ones(g3.n, np.int64), 3)
    assert [p.mult for p in pairs] == [8, 6, 12] and [p.r2 for p in pairs] == [3, 4, 8] and [p.nop for p in pairs] == [2, 4, 4]
    pairs = EP.epi_pair_list(c3, 6, 1 + c3[0] % 2, 2)
    assert [p.cls2 for p in pairs] == [2, 1]


def test_pair_lists_on_site_clusters():
    """hcp (ideal): two pair types in the first shell, 6 + 6 sites at distance a; NiAs from an anion: cations, then
    out-of-plane and in-plane anions, 6 each, at the expected lengths; adapted vectors of the pair group orthonormal."""
    from asr_b200 import crystal as X
    s = X.prototype_structure("hcp")
    ops = X.space_group(s)
    cg = X.crystal_graph(s, ops, 1.1, 2, start=0)
    perm, rot, _ = X.graph_site_ops(cg, s, ops)
    pairs = EP.epi_pair_list_c(cg.disp, perm, rot, s.label[cg.basis], 1)
    assert len(pairs) == 2 and [p.mult for p in pairs] == [6, 6]
    assert max(abs(np.linalg.norm(p.rvec) - 1.0) for p in pairs) < 1e-10
    s = X.prototype_structure("nias", 1.62)
    ops = X.space_group(s)
    cg = X.crystal_graph(s, ops, 1.1, 2, start=2)
    perm, rot, _ = X.graph_site_ops(cg, s, ops)
    cls = s.label[cg.basis].astype(np.int64)
    pairs = EP.epi_pair_list_c(cg.disp, perm, rot, cls, 3)
    assert len(pairs) == 3 and [p.cls2 for p in pairs] == [1, 2, 2] and [p.mult for p in pairs] == [6, 6, 6]
    assert abs(np.linalg.norm(pairs[1].rvec) - np.sqrt(1.0 / 3.0 + (0.5 * 1.62) ** 2)) < 1e-10
    assert abs(np.linalg.norm(pairs[2].rvec) - 1.0) < 1e-10
    cls[pairs[1].site - 1] = 3
    idx = EP.epi_pair_ops_c(perm, rot, cls)
    pd = np.stack([X.orbital_matrix(rot[:, :, k]) for k in idx], axis=2)
    vec, _, _ = EP.epi_adapted(pd)
    assert np.max(np.abs(vec.T @ vec - np.eye(9))) < 1e-13
