"""The oracle's freeze semantics (src/asr_augcls.f90:129-161): augcls_freeze_site checks the start site's class,
augcls_freeze_any accepts any species index and counts the nodes on the site; both refuse a flippable site."""
import pytest

from oracle import oracle as O
from tests import cases as K
from tests import freeze_case as F


def _op(case):
    return O.OracleOp(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, case["maxlevel"],
                      case["maxrank"], case["flippable"])


def test_freeze_site_refuses_a_species_outside_the_start_class():
    op = _op(F.three_species_case())
    op.freeze_site(1, 2)
    with pytest.raises(RuntimeError, match="not in the class"):
        op.freeze_site(1, 3)
    with pytest.raises(RuntimeError, match="out of range"):
        op.freeze_site(1, 4)


def test_freeze_any_counts_the_nodes_of_the_site():
    case = F.three_species_case()
    op = _op(case)
    nodes_on_start = int((op.tables()["site"] == 1).sum())
    assert nodes_on_start >= 1
    assert op.freeze_any(1, 3) == nodes_on_start        # a species outside the start site's class is accepted
    with pytest.raises(RuntimeError, match="out of range"):
        op.freeze_any(1, 0)


def test_freeze_refuses_a_flippable_site():
    case = K.cubic("bcc", 3, 2, (0.5, 0.5), group="d4h", maxlevel=2, maxrank=1)
    op = _op(case)
    with pytest.raises(RuntimeError, match="flippable"):
        op.freeze_any(2, 1)
    with pytest.raises(RuntimeError, match="flippable"):
        op.freeze_site(2, 1)
