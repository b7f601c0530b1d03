"""The device node order (reverse Cuthill-McKee of the hop graph, start node first) is invisible at the interfaces: the
exported tables equal those of the build numbering bit for bit, the drop-in operator application gives the same vectors,
and the chains the same Green functions (rounding of the reduction order only)."""
import os

import numpy as np
import pytest

from asr_b200 import augcls as A
from asr_b200 import chains as CH
from asr_b200 import synthetic as S
from tests import cases as K

pytestmark = pytest.mark.gpu


def _build(case, order):
    old = os.environ.get("ASR_NODE_ORDER")
    try:
        if order == "build":
            os.environ["ASR_NODE_ORDER"] = "build"
        else:
            os.environ.pop("ASR_NODE_ORDER", None)
        return A.build_augcls_operator(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1,
                                       case["maxlevel"], maxrank=case["maxrank"], flippable=case["flippable"])
    finally:
        if old is None:
            os.environ.pop("ASR_NODE_ORDER", None)
        else:
            os.environ["ASR_NODE_ORDER"] = old


def test_node_order_is_invisible():
    case = K.cubic("fcc", 3, 3, (0.66, 0.14, 0.2), group="d2h", maxlevel=3, maxrank=1)
    op_b, op_r = _build(case, "build"), _build(case, "rcm")
    tb, tr = op_b.tables(), op_r.tables()
    for k in tb:
        assert np.array_equal(tb[k], tr[k]), k
    sp = S.draw_species(3, 4)
    ed = S.edc_params(sp, 2)
    for op in (op_b, op_r):
        op.set_params(ed["c"], ed["d"], ed["o"], ed["e"])
    rng = np.random.default_rng(0)
    x = rng.standard_normal((op_b.dim, 3))
    assert np.max(np.abs(op_b.apply(x) - op_r.apply(x))) < 1e-12 * np.max(np.abs(op_b.apply(x)))
    specs = [CH.ChainSpec(c=ed["c"], d=ed["d"], o=ed["o"], e=ed["e"], pa=ed["pa"], pb=ed["pb"], frozen_sp=2, start_orb=l0, nlev=20)
             for l0 in (1, 3, 6, 9)]
    z = np.linspace(-1.0, 0.5, 40) + 0.02j
    gb = CH.chains_run(op_b, specs, z, "edc", 0.0, "hull", "fp64")["g"]
    gr = CH.chains_run(op_r, specs, z, "edc", 0.0, "hull", "fp64")["g"]
    assert np.max(np.abs(gb - gr) / np.abs(gb)) < 1e-11
