"""Golden node counts of the reference's shipped examples ("nodes / sublattice" in example/reference/*/asr.out): the
oracle's restatement of build_augcls_operator (src/asr_augcls.f90:596-823) on the examples' graphs and reduction groups
gives the reference's production node sets."""
import pytest

from asr_b200 import synthetic as S
from oracle.oracle import OracleOp

GOLDEN = [("cuzn_alloy", 1, 17515), ("fe66ni14cr20_fcc", 1, 15827), ("cuzn_b2", 1, 197), ("cuzn_b2", 2, 197),
          ("co2fe04cr06al_l21", 1, 8648), ("co2fe04cr06al_l21", 2, 4639), ("co2fe04cr06al_l21", 3, 4516)]


@pytest.mark.parametrize("name,sub,count", GOLDEN)
def test_example_node_counts(name, sub, count):
    c = S.example_case(name, sub)
    op = OracleOp(c["graph"], c["model"], c["cls"], c["perm"], c["dmat"], 1, c["maxlevel"], c["maxrank"], c["flippable"])
    assert op.nn == count
