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
        op.freeze_site(1, 4)
        op.freeze_site(c["jp"], sj)
        tr = 0.0
        for ia in range(9):
            op.set_chi(chi[: op.nop, ia])
            x, _ = op.epi_blocks(ed, vec[:, ia], Z, 100, tail="none")
            tr += EP.epi_integrand(pt, int(lo[ia]), Z, x)
        # epi_integrand leaves out the constant -2 kappa: it equals the exact trace plus 2 sum_L kappa_L
        assert abs(tr - ref) / abs(ref) < 1e-8, (sj, tr, ref)
