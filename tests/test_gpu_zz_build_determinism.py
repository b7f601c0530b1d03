"""The device analogue of the reference's thread test (test/test_augcls_threads.f90:64-86) on its case, a random bcc
binary with flippable sites, class operations, levels 4, rank 2 (65,972 nodes here): (B) two device builds give the
same node set and every table bit for bit, equal to the oracle's (the parallel closure claims each new node by the
smallest candidate position, so the numbering does not depend on the schedule); (C) the edc chains from orbital 5 with
the start site frozen, depth 24, hull tail, no depth test, give bitwise the same G on repeated calls (fixed-order
reductions, no floating-point atomics) and the oracle's G.  Also: the step kernel's two link-gather instantiations give
the same bits."""
import numpy as np
import pytest

import asr_b200 as A
from asr_b200 import synthetic as S
from oracle import oracle as O
from tests import cases as K

pytestmark = pytest.mark.gpu

TABLE_KEYS = ("flipr", "flipg", "hopr", "hopg", "lst", "site", "ncl", "level", "norb", "sq", "stab_ptr", "stab")


def test_repeated_device_builds_and_chains_are_identical():
    case = K.cubic("bcc", 4, 2, (0.5, 0.5), seed=5, group="d4h", maxlevel=4, maxrank=2)
    args = (case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, case["maxlevel"])
    g1 = A.build_augcls_operator(*args, maxrank=case["maxrank"], flippable=case["flippable"])
    g2 = A.build_augcls_operator(*args, maxrank=case["maxrank"], flippable=case["flippable"])
    oop = O.OracleOp(*args, case["maxrank"], case["flippable"])
    assert g1.nn == g2.nn == oop.nn > 1000
    t1, t2, to = g1.tables(), g2.tables(), oop.tables()
    for k in TABLE_KEYS:
        assert np.array_equal(t1[k], t2[k]) and np.array_equal(t1[k], to[k]), k
    ed = S.edc_params(S.draw_species(2, 5), 1)
    zs = np.array([-0.3 + 0.05j, 0.1 + 0.01j, 0.4 + 0.2j])
    for op in (g1, oop):
        op.set_params(ed["c"], ed["d"], ed["o"], ed["e"])
        op.freeze_site(1, 1)
        op.set_start(5)
    ga, ma, _, _ = A.edc_green_blk(g1, ed, zs, 5, 24, depth_tol=0.0, tail="hull", precision="fp64")
    gb, mb, _, _ = A.edc_green_blk(g1, ed, zs, 5, 24, depth_tol=0.0, tail="hull", precision="fp64")
    assert np.array_equal(ma, mb) and np.array_equal(ga, gb)
    go, mo, _, _ = oop.edc_green_blk(ed, zs, 5, 24, depth_tol=0.0, tail="hull")
    assert np.array_equal(ma, mo)
    assert np.max(np.abs(ga - go) / np.abs(go)) < 1e-8


@pytest.mark.parametrize("group", ["d2h", "d4h"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_fixed_offset_link_gathers_give_the_same_bits(group, precision):
    """The step kernel with fixed-offset link gathers (identity and sign-only orbital operations read their rows without
    index decoding) gives the same Green functions bit for bit as the general kernel at the same batch shape: D2h links
    are identities or sign changes, D4h links also permute orbitals (the general path inside the same kernel)."""
    from asr_b200 import chains as CH
    case = K.cubic("fcc", 3, 3, (0.66, 0.14, 0.2), group=group, maxlevel=3, maxrank=1)
    op = A.build_augcls_operator(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, case["maxlevel"],
                                 maxrank=case["maxrank"], flippable=case["flippable"])
    sp = S.draw_species(3, 2)
    specs = []
    for cen in (1, 2, 3):
        ed = S.edc_params(sp, cen)
        for l0 in (1, 3, 7):
            specs.append(CH.ChainSpec(c=ed["c"], d=ed["d"], o=ed["o"], e=ed["e"], pa=ed["pa"], pb=ed["pb"], frozen_sp=cen,
                                      start_orb=l0, nlev=14))
    z = np.linspace(-1.0, 0.5, 70) + 0.02j
    out = {}
    for link in ("general", "fixed-offset"):
        A.set_tuning(op, precision, 16 if precision == "fp64" else 8, 4, link)
        assert A.tuning(op, precision)["link_gather"] == link
        out[link] = CH.chains_run(op, specs, z, "edc", 0.0, "hull", precision)["g"]
    assert np.array_equal(out["general"], out["fixed-offset"])
