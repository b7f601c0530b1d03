"""The device operator build on the reference's shipped examples: the production node counts of example/reference/*/
asr.out ("nodes / sublattice") and tables bit-exact against the oracle."""
import numpy as np
import pytest

from asr_b200 import augcls as A
from asr_b200 import synthetic as S
from oracle.oracle import OracleOp
from tests.test_gpu_parity import TABLE_KEYS
from tests.test_oracle_golden_counts import GOLDEN

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
