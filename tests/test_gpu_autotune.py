"""The batch-shape autotuner (asr_autotune): the chosen shape is one of the candidates, later automatic calls use it,
and the chains give the same results (to the rounding of the per-block partial sums) before and after."""
import numpy as np
import pytest

from asr_b200 import augcls as A
from asr_b200 import chains as CH
from asr_b200 import synthetic as S
from tests import cases as K

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_autotune_keeps_results(precision):
    case = K.cubic("fcc", 3, 3, (0.66, 0.14, 0.2), group="d2h", maxlevel=3, maxrank=1)
    op = A.build_augcls_operator(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, case["maxlevel"],
                                 maxrank=case["maxrank"], flippable=case["flippable"])
    sp = S.draw_species(3, 2)
    specs = []
    for cen in (1, 2, 3):
        ed = S.edc_params(sp, cen)
        for l0 in (1, 4, 7):
            specs.append(CH.ChainSpec(c=ed["c"], d=ed["d"], o=ed["o"], e=ed["e"], pa=ed["pa"], pb=ed["pb"], frozen_sp=cen,
                                      start_orb=l0, nlev=16))
    z = np.linspace(-1.0, 0.5, 80) + 0.02j
    g0 = CH.chains_run(op, specs, z, "edc", 0.0, "hull", precision)["g"]
    tune = CH.autotune(op, specs, z, precision, levels=6)
    assert tune["tiles_per_batch"] in (4, 8, 16, 32) and tune["nodes_per_warp"] in (1, 2, 4, 8)
    assert all(t > 0 for t in tune["ms_npw"])
    g1 = CH.chains_run(op, specs, z, "edc", 0.0, "hull", precision)["g"]
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert np.max(np.abs(g1 - g0) / np.abs(g0)) < tol
