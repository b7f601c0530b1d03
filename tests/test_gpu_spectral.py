"""Projected chains on the device (asr_chains_proj, edc_green_proj of src/asr_edc.f90:174-232) and the target links of
the device build (asr_op_build_targets, src/asr_augcls.f90:808-820) against the oracle, on the readout case of the
reference's test_spectral.f90 (random bcc binary, levels 2, rank 1, targets: origin + two shells)."""
import numpy as np
import pytest

from asr_b200 import augcls as A
from asr_b200 import chains as CH
from asr_b200 import spectral as SP
from oracle.oracle import OracleOp
from tests.spectral_case import CONC, readout_inputs

pytestmark = pytest.mark.gpu

ZS = np.array([0.35 + 0.08j, -0.2 + 0.03j, 0.6 + 0.01j, -0.45 + 0.15j])


@pytest.fixture(scope="module")
def both():
    r = readout_inputs()
    dev, orc = {}, {}
    for key, (perm, dmat) in r["groups"].items():
        args = (r["graph"], r["model"], r["cls"], perm, dmat, 1, 2)
        dev[key] = A.build_augcls_operator(*args, maxrank=1, flippable=r["flippable"], tsite=r["tsite"])
        op = OracleOp(*args, 1, r["flippable"], tsite=r["tsite"])
        ed = r["ed"]
        op.set_params(ed["c"], ed["d"], ed["o"], ed["e"])
        op.freeze_site(1, 1)
        orc[key] = op
    return r, dev, orc


def test_target_links_bit_exact(both):
    r, dev, orc = both
    for key in dev:
        op, tnode, tgop = dev[key]
        assert op.nn == orc[key].nn
        assert np.array_equal(tnode, orc[key].tnode), key
        found = tnode > 0
        assert np.array_equal(tgop[found], orc[key].tgop[found]), key


def _specs(ed, nlev, starts):
    return [CH.ChainSpec(c=ed["c"], d=ed["d"], o=ed["o"], e=ed["e"], pa=ed["pa"], pb=ed["pb"], frozen_sp=1, start_orb=l0,
                         nlev=nlev) for l0 in starts]


@pytest.mark.parametrize("nlev,tail", [(8, "none"), (24, "none"), (24, "hull"), (16, "avg2")])
def test_projections_match_the_oracle(both, nlev, tail):
    r, dev, orc = both
    ed, tw = r["ed"], r["tw"]
    op, tnode, tgop = dev["d2h"]
    res = CH.chains_proj(op, _specs(ed, nlev, range(1, 10)), ZS, tnode, tgop, tw, tail)
    worst = 0.0
    for q, l0 in enumerate(range(1, 10)):
        o = orc["d2h"]
        o.set_start(l0)
        for j, z in enumerate(ZS):
            g, gp, gp4, m = o.edc_green_proj(ed, z, l0, nlev, o.tnode, o.tgop, tw, tail=tail)
            assert res["m"][j, q] == m
            scale = max(np.max(np.abs(gp)), abs(g))
            worst = max(worst, abs(res["g"][j, q] - g) / scale, np.max(np.abs(res["gp"][:, :, j, q] - gp)) / scale,
                        np.max(np.abs(res["gp4"][:, :, j, q] - gp4)) / scale)
    assert worst < 1e-10, worst


def test_device_projections_in_three_bases(both):
    """The same Krylov process in three bases on the device: D2h and D4h projections equal the unreduced ones."""
    r, dev, _ = both
    ed, tw, t0 = r["ed"], r["tw"], r["t0"]
    d4 = r["groups"]["d4h"][1]
    out = {}
    for key in ("identity", "d2h", "d4h"):
        op, tnode, tgop = dev[key]
        starts = [l0 for l0 in range(1, 10)
                  if key != "d4h" or np.all(np.abs(np.abs(d4[l0 - 1, l0 - 1, :]) - 1.0) < 1e-9)]
        res = CH.chains_proj(op, _specs(ed, 8, starts), ZS[:1], tnode, tgop, tw, "none")
        out[key] = {l0: (res["g"][0, q], res["gp"][:, :, 0, q]) for q, l0 in enumerate(starts)}
    for key in ("d2h", "d4h"):
        for l0, (g, gp) in out[key].items():
            assert np.max(np.abs(gp - out["identity"][l0][1])) < 1e-11, (key, l0)
            assert abs(gp[l0 - 1, t0] - g) < 1e-13


def test_fp32_projections_close_to_fp64(both):
    r, dev, _ = both
    op, tnode, tgop = dev["d2h"]
    specs = _specs(r["ed"], 16, range(1, 10))
    r64 = CH.chains_proj(op, specs, ZS, tnode, tgop, r["tw"], "hull", "fp64")
    r32 = CH.chains_proj(op, specs, ZS, tnode, tgop, r["tw"], "hull", "fp32")
    assert np.max(np.abs(r32["gp"] - r64["gp"])) < 1e-4 * np.max(np.abs(r64["gp"]))


def test_spectral_elements_and_bloch_sum_against_the_oracle(both):
    """Averaged elements over the two central species on the device against the oracle's, then the windowed Bloch sum."""
    from asr_b200 import synthetic as S
    r, dev, orc = both
    op, tnode, tgop = dev["d2h"]
    sp = S.draw_species(2, 11)
    eds = [S.edc_params(sp, c) for c in (1, 2)]
    z = np.linspace(-0.6, 0.6, 7) + 0.02j
    gdg, gdg4 = SP.spectral_elements(op, tnode, tgop, r["t0"], [1, 2], list(CONC), eds, z, 12, tail="hull")
    ref = np.zeros_like(gdg)
    o = orc["d2h"]
    for ci, cen in enumerate((1, 2)):
        ed = eds[ci]
        o.set_params(ed["c"], ed["d"], ed["o"], ed["e"])
        o.unfreeze()
        o.freeze_site(1, cen)
        tw = np.zeros((9, 2, len(r["tsite"])))
        for t in range(len(r["tsite"])):
            tw[:, :, t] = SP.spectral_dressing(ed["dc"], ed["dl"], [1, 2], CONC, t == r["t0"])
        for l0 in range(1, 10):
            o.set_start(l0)
            for j, zz in enumerate(z):
                _, gp, _, _ = o.edc_green_proj(ed, zz, l0, 12, o.tnode, o.tgop, tw, tail="hull")
                ref[l0 - 1, :, j] += CONC[ci] * gp[l0 - 1]
    assert np.max(np.abs(gdg - ref)) < 1e-10 * np.max(np.abs(ref))
    kv, _, _ = SP.spectral_kpath(np.array([[0, 1, 0.5], [0, 0, 0.5], [0, 0, 0.5]], float), 6)
    a_dev, _ = SP.spectral_sum(gdg, r["tdisp"], kv, 1.0)
    a_ref, _ = SP.spectral_sum(ref, r["tdisp"], kv, 1.0)
    assert np.max(np.abs(a_dev - a_ref)) < 1e-10 * np.max(np.abs(a_ref))
    assert np.all(np.isfinite(a_dev))
