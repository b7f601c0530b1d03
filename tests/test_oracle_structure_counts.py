"""Operator inputs from the structure alone (crystal.sublattice_inputs: ball cluster, class-preserving site group,
orbital groups, reduction group) through the oracle's build_augcls_operator.

* Node counts: the ball about the start site holds no image of any site, so its node set is the one of a periodic
  cluster large enough that nothing wraps within the closure; both constructions give the same counts.  (The published
  counts of the examples, 17515 / 15827 / 8648 / 4639 / 4516 / 197, came from the 8^3 / 12^3 periodic supercells of the
  release that wrote them and are pinned by test_oracle_golden_counts.)
* Start orbitals: chains from the representatives under the reduction group have the recursion coefficients of the
  chains from every orbital of their group under the diagonal (D2h) group: the weights are exact."""
import numpy as np
import pytest

from asr_b200 import synthetic as S
from oracle.oracle import OracleOp

# (example, sublattice, node count of the ball / an unwrapped periodic cluster)
BALL = [("cuzn_alloy", 1, 21579), ("fe66ni14cr20_fcc", 1, 16270), ("cuzn_b2", 1, 215), ("cuzn_b2", 2, 215),
        ("co2fe04cr06al_l21", 1, 10771), ("co2fe04cr06al_l21", 2, 5814), ("co2fe04cr06al_l21", 3, 5578)]


def _oracle(c):
    return OracleOp(c["graph"], c["model"], c["cls"], c["perm"], c["dmat"], 1, c["maxlevel"], c["maxrank"], c["flippable"],
                    c.get("stype"))


@pytest.mark.parametrize("name,sub,count", BALL)
def test_structure_node_counts(name, sub, count):
    c = S.structure_case(name, sub)
    assert list(c["reps"]) == [1, 3, 5, 7] and list(c["weights"]) == [1, 3, 3, 2]
    assert _oracle(c).nn == count


@pytest.mark.parametrize("name,sub", [("cuzn_b2", 2), ("co2fe04cr06al_l21", 3)])
def test_ball_equals_an_unwrapped_periodic_cluster(name, sub):
    ball = _oracle(S.structure_case(name, sub)).nn
    periodic = _oracle(S.example_case(name, sub, l=16)).nn
    assert ball == periodic == dict(((n, s), k) for n, s, k in BALL)[(name, sub)]


@pytest.mark.parametrize("name,sub", [("cuzn_alloy", 1), ("co2fe04cr06al_l21", 1)])
def test_representatives_carry_their_orbital_groups(name, sub):
    red = S.structure_case(name, sub, levels=2)
    diag = S.structure_case(name, sub, levels=2, group="diagonal")
    assert red["perm"].shape[1] > diag["perm"].shape[1] >= 1
    nsp = red["model"].nsp
    c, d, o, e = S.plain_params(S.draw_species(nsp, 5))
    ops = {}
    for key, case in (("red", red), ("diag", diag)):
        op = _oracle(case)
        op.set_params(c, d, o, e)
        ops[key] = op
    grp = np.array([1, 2, 2, 2, 3, 3, 4, 3, 4])
    reps = list(red["reps"])
    depth = 10
    coef = {}
    for key, starts in (("red", reps), ("diag", range(1, 10))):
        for l0 in starts:
            ops[key].set_start(l0)
            v0 = np.zeros(ops[key].dim)
            v0[l0 - 1] = 1.0
            a, b, n = ops[key].lanczos(v0, depth)
            coef[key, l0] = (np.asarray(a[:n]), np.asarray(b[:n]))
    for l0 in range(1, 10):
        ar, br = coef["red", reps[grp[l0 - 1] - 1]]
        ad, bd = coef["diag", l0]
        assert len(ar) == len(ad) == depth
        assert np.max(np.abs(ar - ad)) < 1e-9 * np.max(np.abs(ar)) and np.max(np.abs(br[:-1] - bd[:-1])) < 1e-9 * np.max(np.abs(br))


def test_ball_and_periodic_box_give_the_same_chains():
    """The ball about the start site and an unwrapped periodic box give the same recursion (the reference's cluster vs
    box check): plain chains from s, p_z, d_3z2 on the B2 sublattice a, 8 levels, coefficients to 1e-10 (deeper levels
    differ by the rounding that the two node orders amplify in a chain without reorthogonalisation)."""
    ball = S.structure_case("cuzn_b2", 1)
    box = S.example_case("cuzn_b2", 1, l=16)
    c, d, o, e = S.plain_params(S.draw_species(2, 7))
    ops = []
    for case in (ball, box):
        op = _oracle(case)
        op.set_params(c, d, o, e)
        ops.append(op)
    assert ops[0].nn == ops[1].nn
    for l0 in (1, 3, 7):
        coef = []
        for op in ops:
            op.set_start(l0)
            v0 = np.zeros(op.dim)
            v0[l0 - 1] = 1.0
            a, b, n = op.lanczos(v0, 8)
            coef.append((a[:n], b[:n]))
        assert np.max(np.abs(coef[0][0] - coef[1][0])) < 1e-10 and np.max(np.abs(coef[0][1] - coef[1][1])) < 1e-10


def test_chain_greens_is_independent_of_the_thread_count():
    """The oracle's task-parallel chain_greens gives bit-identical Green functions with 1 and 4 threads (the reference's
    thread-count test)."""
    case = S.structure_case("cuzn_b2", 2)
    op = _oracle(case)
    sp = S.draw_species(2, 3)
    groups = []
    for cen in (1, 2):
        ed = S.edc_params(sp, cen)
        groups.append(dict(c=ed["c"], d=ed["d"], o=ed["o"], e=ed["e"], dc=ed["dc"], dl=ed["dl"], enu=ed["enu"]))
    z = np.linspace(-0.8, 0.4, 12) + 0.05j
    nlev = np.full((2, 2), 16, np.int32)
    g1, _ = op.chain_greens(groups, [0, 0], [1, 3], nlev, z, 4, nthreads=1)
    g4, _ = op.chain_greens(groups, [0, 0], [1, 3], nlev, z, 4, nthreads=4)
    assert np.array_equal(g1, g4)
