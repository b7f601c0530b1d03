"""The oracle's chains against dense linear algebra (no recursion on the other side), after the reference's
test/test_recursion_dense.f90 (plain Lanczos + continued fraction = the dense spectral sum; the second moment) and
test/test_augcls_project.f90 (edc chains on the group-reduced operator = the dense inverse of the unreduced one)."""
import numpy as np
import pytest

from asr_b200 import synthetic as S
from tests import cases as K
from oracle import oracle as O


def _fraction(a, b, n, z):
    g = 0.0
    for k in range(n - 1, -1, -1):
        g = 1.0 / (z - a[k] - (b[k] ** 2 * g if k < n - 1 else 0.0))
    return g


def _dense(op, nd):
    h = np.zeros((nd, nd))
    for k in range(nd):
        x = np.zeros(nd)
        x[k] = 1.0
        h[:, k] = op.apply(x)
    return h


@pytest.mark.parametrize("l0", [1, 3, 7])
def test_plain_lanczos_equals_the_dense_spectral_sum(l0):
    """An ordered 8-site periodic sc cell (one species, identity group): the node set is the sites, the chain closes, and
    the fraction equals sum_n |<0 l0|n>|^2 / (z - E_n) (1e-9); a_1^2 + b_1^2 = (H^2)_00 (1e-12)."""
    case = S.cubic_case("sc", 2, 1, [1.0], seed=3, group="identity")
    fl = np.zeros(case["graph"].n, np.int32)
    op = O.OracleOp(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, 6, 0, fl)
    assert op.nn == case["graph"].n
    c, d, o, e = S.plain_params(S.draw_species(1, 3))
    op.set_params(c, d, o, e)
    op.set_start(l0)
    h = _dense(op, op.dim)
    assert np.max(np.abs(h - h.T)) < 1e-13
    ev, vec = np.linalg.eigh(h)
    v0 = np.zeros(op.dim)
    v0[l0 - 1] = 1.0
    a, b, n = op.lanczos(v0, op.dim + 5)
    small = np.nonzero(np.abs(b[:n]) < 1e-8 * np.max(np.abs(b[:n])))[0]
    assert small.size                                    # the invariant subspace of the start vector is exhausted
    n = int(small[0]) + 1                                # the chain up to the first vanishing b (no reorthogonalisation)
    assert abs(a[0] ** 2 + b[0] ** 2 - (h @ h)[l0 - 1, l0 - 1]) < 1e-12
    w = vec[l0 - 1] ** 2
    for z in (0.1 + 0.2j, -0.7 + 0.05j, 1.3 + 0.4j):
        ref = np.sum(w / (z - ev))
        assert abs(_fraction(a, b, n, z) - ref) < 1e-9 * abs(ref)


def test_reduced_edc_chain_equals_the_dense_unreduced_inverse():
    """A random bcc binary on the 16-site periodic cell, levels 2, rank 1, start frozen: the edc chain (tail none) on the
    D4h-reduced operator (58 nodes) equals <e|(z - H(z))^-1|e> from a dense solve with the unreduced operator (256 nodes)."""
    red = S.cubic_case("bcc", 2, 2, [0.5, 0.5], seed=0, group="d4h")
    unr = S.cubic_case("bcc", 2, 2, [0.5, 0.5], seed=0, group="identity")
    fl = np.ones(red["graph"].n, np.int32)
    fl[0] = 0
    opr = O.OracleOp(red["graph"], red["model"], red["cls"], red["perm"], red["dmat"], 1, 2, 1, fl)
    opu = O.OracleOp(unr["graph"], unr["model"], unr["cls"], unr["perm"], unr["dmat"], 1, 2, 1, fl)
    assert (opr.nn, opu.nn) == (58, 256)
    ed = S.edc_params(S.draw_species(2, 6), 2)
    for op in (opr, opu):
        op.set_params(ed["c"], ed["d"], ed["o"], ed["e"])
        op.freeze_site(1, 2)
    hu = _dense(opu, opu.dim)
    worst = 0.0
    for l0 in (1, 5, 7):
        opr.set_start(l0)
        for z in (0.05 + 0.3j, -0.4 + 0.1j):
            ep = np.asfortranarray(z - ed["dc"][:, None] * (z - ed["enu"]) / ed["dl"])
            xu = np.zeros((opu.dim, opu.dim), np.complex128)
            for k in range(opu.dim):
                u = np.zeros(opu.dim, np.complex128)
                u[k] = 1.0
                xu[:, k] = opu.rand_c(ep, u)
            rhs = np.zeros(opu.dim, np.complex128)
            rhs[l0 - 1] = 1.0
            gd = np.linalg.solve(z * np.eye(opu.dim) - hu - xu, rhs)[l0 - 1]
            gc = opr.edc_green(ed, z, l0, 600, tail="none")[0]
            worst = max(worst, abs(gc - gd) / abs(gd))
    assert worst < 1e-9, worst


def test_threaded_node_loops_give_the_same_bits():
    """The oracle's node loops on several host threads (oracle.apply_threads) give the serial chain bit for bit."""
    case = K.cubic("bcc", 3, 2, (0.5, 0.5), group="d2h", maxlevel=2)
    oop = O.OracleOp(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, case["maxlevel"],
                     case["maxrank"], case["flippable"])
    c, d, o, e = S.plain_params(S.draw_species(2, 0))
    oop.set_params(c, d, o + 0.01, e + 0.02)
    oop.set_start(1)
    v0 = np.zeros(oop.dim)
    v0[0] = 1.0
    ref = oop.lanczos(v0, 10)
    with O.apply_threads(4):
        got = oop.lanczos(v0, 10)
    assert O.lib().orc_apply_threads() == 1
    assert np.array_equal(ref[0], got[0]) and np.array_equal(ref[1], got[1]) and ref[2] == got[2]
