"""The oracle's operator and chains against exact answers: ring configuration averages (test_slow/test_augcls.f90:69-148),
group-reduced == unreduced chains (test_slow/test_augcls.f90 (B), test/test_augcls_project.f90), projector identities
(test/test_augcls_project.f90:166-187), block == single chains (test_slow/test_augcls_blk.f90)."""
import numpy as np
import pytest

from asr_b200 import synthetic as S
from oracle import oracle as O
from tests import toy_models as T

RCLS = [1, 2, 3, 2]


@pytest.mark.parametrize("ic", [1, 2, 3])
def test_ring_recursion_equals_exact_average(ic):
    g = T.ring_graph(4)
    mdl = T.three_classes()
    sp = T.species_lmto()
    ib = RCLS.index(ic)
    rcls = list(np.roll(RCLS, -ib))
    perm = np.asfortranarray(np.arange(1, 5, dtype=np.int32).reshape(4, 1))
    dmat = np.asfortranarray(np.eye(9).reshape(9, 9, 1))
    fl = np.array([0, 1, 1, 1], np.int32)
    err = 0.0
    for j in range(mdl.nsc[ic - 1]):
        cen = int(mdl.spc[j, ic - 1])
        ed = T.edc_setup(sp, cen)
        op = O.OracleOp(g, mdl, np.array(rcls, np.int32), perm, dmat, 1, 80, 0, fl)
        op.set_params(ed["c"], ed["d"], ed["o"], ed["e"])
        op.freeze_site(1, cen)
        for l0 in (1, 5, 9):
            op.set_start(l0)
            for kz in (1, 2, 3):
                z = complex(-0.3 + 0.3 * kz, 0.3)
                gre = op.edc_green(ed, z, l0, 400, tail="none")[0]
                gden, psum = T.exact_average(mdl, g, rcls, cen, sp, z, l0)
                assert abs(psum - 1.0) < 1e-12
                err = max(err, abs(gre - gden))
    assert err < 1e-6, err


@pytest.fixture(scope="module")
def bcc_pair():
    case = S.cubic_case("bcc", 3, 2, [0.5, 0.5], seed=0, group="d4h")
    caseu = S.cubic_case("bcc", 3, 2, [0.5, 0.5], seed=0, group="identity")
    fl = np.ones(case["graph"].n, np.int32)
    fl[0] = 0
    op = O.OracleOp(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, 2, 0, fl)
    opu = O.OracleOp(caseu["graph"], caseu["model"], caseu["cls"], caseu["perm"], caseu["dmat"], 1, 2, 0, fl)
    return case, op, opu


def test_reduced_chain_equals_unreduced(bcc_pair):
    case, op, opu = bcc_pair
    ed = S.edc_params(S.draw_species(2, 0), 1)
    for o_ in (op, opu):
        o_.set_params(ed["c"], ed["d"], ed["o"], ed["e"])
        o_.unfreeze()
        o_.freeze_site(1, 1)
    for l0 in (1, 5, 7, 9):
        op.set_start(l0)
        opu.set_start(l0)
        z = complex(-0.1, 0.05)
        g, a, b, m, _ = op.edc_green(ed, z, l0, 16)
        gu, au, bu, mu, _ = opu.edc_green(ed, z, l0, 16)
        assert m == mu
        assert np.max(np.abs(a - au) / np.abs(au)) < 1e-9
        assert abs(g - gu) / abs(gu) < 1e-10


def test_projector_is_idempotent_and_symmetric(bcc_pair):
    case, op, _ = bcc_pair
    op.set_start(1)
    rng = np.random.default_rng(2)
    x = rng.uniform(-0.5, 0.5, op.dim) + 1j * rng.uniform(-0.5, 0.5, op.dim)
    y = rng.uniform(-0.5, 0.5, op.dim) + 1j * rng.uniform(-0.5, 0.5, op.dim)
    px = op.project_c(x)
    py = op.project_c(y)
    leak = lambda v: np.linalg.norm(v - op.project_c(v)) / np.linalg.norm(v)
    assert leak(x) > 0.1
    assert leak(px) < 1e-14
    assert abs(np.sum(y * px) - np.sum(py * x)) / abs(np.sum(py * x)) < 1e-13


def test_block_chain_equals_single(bcc_pair):
    case, op, _ = bcc_pair
    ed = S.edc_params(S.draw_species(2, 0), 2)
    op.set_params(ed["c"], ed["d"], ed["o"], ed["e"])
    op.unfreeze()
    op.freeze_site(1, 2)
    op.set_start(5)
    zs = np.array([complex(-0.2, 0.03), complex(0.1, 0.02), complex(0.3, 0.1)])
    gb, mb, ab, bb = op.edc_green_blk(ed, zs, 5, 20, depth_tol=1e-6)
    for j, z in enumerate(zs):
        g, a, b, m, _ = op.edc_green(ed, z, 5, 20, depth_tol=1e-6)
        assert m == mb[j]
        assert abs(g - gb[j]) / abs(g) < 1e-11
