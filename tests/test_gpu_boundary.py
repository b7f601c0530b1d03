"""Boundary entry points against the oracle, through the C-ABI: augcls_hp_c (src/asr_augcls.f90:301-320), the freeze pair
augcls_freeze_site / augcls_freeze_any (:129-161) and dos_final (src/asr_class_scf.f90:1912-1931)."""
import numpy as np
import pytest

import asr_b200 as A
from asr_b200 import synthetic as S
from oracle import oracle as O
from tests import cases as K
from tests import freeze_case as F

pytestmark = pytest.mark.gpu


def _both(case):
    return K.build_both(case, A.build_augcls_operator, O.OracleOp)


def test_hp_c_matches_oracle():
    case = K.cubic("fcc", 3, 3, (0.66, 0.14, 0.2), group="d2h", maxlevel=2, maxrank=1)
    gop, oop = _both(case)
    c, d, o, e = K.general_params(3)
    for op in (gop, oop):
        op.set_params(c, d, o, e)
    rng = np.random.default_rng(7)
    x = rng.uniform(-0.5, 0.5, (gop.dim, 3)) + 1j * rng.uniform(-0.5, 0.5, (gop.dim, 3))
    yg = gop.hp_c(x)
    for j in range(3):
        yo = oop.hp_c(x[:, j])
        assert np.max(np.abs(yg[:, j] - yo)) <= 1e-12 * np.max(np.abs(yo))


def test_freeze_site_and_freeze_any_follow_the_oracle():
    case = F.three_species_case()
    gop, oop = _both(case)
    c, d, o, e = F.params3()
    for op in (gop, oop):
        op.set_params(c, d, o, e)
    # freeze_site: species 3 is outside the start site's class, species 0 and 4 out of range
    for op in (gop, oop):
        with pytest.raises((A.AsrError, RuntimeError), match="not in the class"):
            op.freeze_site(1, 3)
        for sp in (0, 4):
            with pytest.raises((A.AsrError, RuntimeError), match="out of range"):
                op.freeze_site(1, sp)
            with pytest.raises((A.AsrError, RuntimeError), match="out of range"):
                op.freeze_any(1, sp)
        with pytest.raises((A.AsrError, RuntimeError), match="flippable"):
            op.freeze_any(2, 1)
    # freeze_any accepts it and counts the nodes of the site; the operator then equals the oracle's
    assert gop.freeze_any(1, 3) == oop.freeze_any(1, 3) >= 1
    x = np.random.default_rng(3).uniform(-0.5, 0.5, gop.dim)
    yg, yo = gop.apply(x), oop.apply(x)
    assert np.max(np.abs(yg - yo)) <= 1e-12 * np.max(np.abs(yo))
    # freeze_site within the class, after the previous freeze (repeated freezes reuse the host tables)
    for op in (gop, oop):
        op.unfreeze()
        op.freeze_site(1, 2)
    yg, yo = gop.apply(x), oop.apply(x)
    assert np.max(np.abs(yg - yo)) <= 1e-12 * np.max(np.abs(yo))


def test_dos_final_matches_oracle():
    """edos(ie, l, comp, spin) of 2 spins x 3 components x 9 start orbitals (D2h: every orbital one dimensional, with
    the weights of an orbital grouping given per orbital) on the fcc ternary cluster."""
    case = K.cubic("fcc", 3, 3, (0.66, 0.14, 0.2), group="d2h", maxlevel=2, maxrank=1)
    gop, oop = _both(case)
    lorb = S.ORB_L.tolist()
    worb = [1.0, 1.0, 2.0, 1.0, 1.0, 1.0, 3.0, 1.0, 2.0]
    nlev = 16
    specs, comp, spin, lq, wq, groups, gcomp, pcomp, pspin = [], [], [], [], [], [], [], [], []
    for sp_ in (1, 2):
        sp = S.draw_species(3, 10 + sp_)
        for cen in (1, 2, 3):
            ed = S.edc_params(sp, cen)
            groups.append(dict(c=ed["c"], d=ed["d"], o=ed["o"], e=ed["e"], dc=ed["dc"], dl=ed["dl"], enu=ed["enu"]))
            gcomp.append(cen)
            pcomp.append(cen)
            pspin.append(sp_)
            for l0 in range(1, 10):
                specs.append(A.ChainSpec(c=ed["c"], d=ed["d"], o=ed["o"], e=ed["e"], pa=ed["pa"], pb=ed["pb"], frozen_sp=cen,
                                         start_orb=l0, nlev=nlev))
                comp.append(cen)
                spin.append(sp_)
                lq.append(lorb[l0 - 1])
                wq.append(worb[l0 - 1])
    emin, emax, eta, ndos = -1.4, 0.8, 0.01, 60
    e, edos = A.dos_final(gop, specs, comp, spin, lq, wq, 3, 2, emin, emax, eta, ndos)
    nlevq = np.full((6, 9), nlev, np.int32)
    eo, edos_o = O.dos_final(oop, groups, gcomp, list(range(1, 10)), nlevq, lorb, worb, pcomp, pspin, 3, 2, emin, emax, eta,
                             ndos)
    assert np.max(np.abs(e - eo)) < 1e-15
    assert edos.shape == (ndos, 3, 3, 2)
    assert np.max(np.abs(edos - edos_o)) <= 1e-8 * np.max(np.abs(edos_o))
    assert np.min(edos_o) > -1e-10      # a DOS: non-negative


def test_held_workspace_forward_gives_the_same_bits():
    """asr_ctx_hold_workspace on the batched chain runs: the kept vector slab, reused by the next calls, gives the bits of
    the allocating call."""
    case = S.cubic_case("bcc", 3, 2, [0.5, 0.5], seed=0, group="d4h")
    fl = np.ones(case["graph"].n, np.int32)
    fl[0] = 0
    op = A.build_augcls_operator(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, 2, maxrank=1,
                                 flippable=fl)
    specs = []
    for cen in (1, 2):
        ed = S.edc_params(S.draw_species(2, cen), cen)
        for l0 in (1, 3, 5):
            specs.append(A.ChainSpec(c=ed["c"], d=ed["d"], o=ed["o"], e=ed["e"], pa=ed["pa"], pb=ed["pb"], frozen_sp=cen,
                                     start_orb=l0, nlev=14))
    z = np.linspace(-0.6, 0.4, 40) + 0.02j
    ref = A.chains_run(op, specs, z, "edc", 0.0, "hull", "fp64")["g"]
    op.ctx.hold_workspace(True)
    try:
        for zz in (z, z, z[:7]):
            g = A.chains_run(op, specs, zz, "edc", 0.0, "hull", "fp64")["g"]
            assert np.array_equal(g, ref[: zz.size])
    finally:
        op.ctx.hold_workspace(False)
