"""The device operator build on the reference's shipped examples: the production node counts of example/reference/*/
asr.out ("nodes / sublattice") and tables bit-exact against the oracle; the same examples from their structures alone
(ball cluster, class-preserving site group, reduction group), and chains from the start-orbital representatives."""
import numpy as np
import pytest

from asr_b200 import augcls as A
from asr_b200 import chains as CH
from asr_b200 import synthetic as S
from oracle.oracle import OracleOp
from tests.test_gpu_parity import TABLE_KEYS
from tests.test_oracle_golden_counts import GOLDEN
from tests.test_oracle_structure_counts import BALL

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,sub,count", GOLDEN)
def test_device_build_reproduces_the_example_node_sets(name, sub, count):
    c = S.example_case(name, sub)
    args = (c["graph"], c["model"], c["cls"], c["perm"], c["dmat"], 1, c["maxlevel"])
    gop = A.build_augcls_operator(*args, maxrank=c["maxrank"], flippable=c["flippable"])
    assert gop.nn == count
    oop = OracleOp(*args, c["maxrank"], c["flippable"])
    tg, to = gop.tables(), oop.tables()
    for k in TABLE_KEYS:
        assert np.array_equal(tg[k], to[k]), (name, sub, k)


@pytest.mark.parametrize("name,sub,count", BALL)
def test_device_build_on_structure_inputs(name, sub, count):
    """The ball cluster and reduction group from the structure alone: node count and tables against the oracle."""
    c = S.structure_case(name, sub)
    args = (c["graph"], c["model"], c["cls"], c["perm"], c["dmat"], 1, c["maxlevel"])
    gop = A.build_augcls_operator(*args, maxrank=c["maxrank"], flippable=c["flippable"], stype=c["stype"])
    assert gop.nn == count
    oop = OracleOp(*args, c["maxrank"], c["flippable"], c["stype"])
    tg, to = gop.tables(), oop.tables()
    for k in TABLE_KEYS:
        assert np.array_equal(tg[k], to[k]), (name, sub, k)


def test_device_chains_from_representatives_weight_their_groups():
    """Plain chains on the device: the representative of each orbital group under the reduction group has the
    coefficients of every orbital of its group under the diagonal group (1e-9)."""
    red = S.structure_case("cuzn_alloy", 1, levels=3)
    diag = S.structure_case("cuzn_alloy", 1, levels=3, group="diagonal")
    cpar, d, o, e = S.plain_params(S.draw_species(2, 5))
    grp = np.array([1, 2, 2, 2, 3, 3, 4, 3, 4])
    out = {}
    for key, c in (("red", red), ("diag", diag)):
        op = A.build_augcls_operator(c["graph"], c["model"], c["cls"], c["perm"], c["dmat"], 1, c["maxlevel"],
                                     maxrank=1, flippable=c["flippable"], stype=c["stype"])
        starts = list(red["reps"]) if key == "red" else list(range(1, 10))
        specs = [CH.ChainSpec(c=cpar, d=d, o=o, e=e, start_orb=l0, nlev=14) for l0 in starts]
        r = CH.chains_run(op, specs, np.array([0.1j]), mode="plain", tail="none", coefs=True)
        out[key] = {l0: (r["a"][:, 0, q], r["b"][:, 0, q]) for q, l0 in enumerate(starts)}
    for l0 in range(1, 10):
        ar, br = out["red"][int(red["reps"][grp[l0 - 1] - 1])]
        ad, bd = out["diag"][l0]
        assert np.max(np.abs(ar - ad)) < 1e-9 * np.max(np.abs(ar)), l0
        assert np.max(np.abs(br[:-1] - bd[:-1])) < 1e-9 * np.max(np.abs(br)), l0
