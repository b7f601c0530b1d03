"""GPU parity through the C-ABI against the oracle: node tables bit-exact; operator applications, chain coefficients and
Green functions within the tolerances of the reference's own tests (recursion coefficients 1e-9 relative, G 1e-8)."""
import numpy as np
import pytest

import asr_b200 as A
from asr_b200 import synthetic as S
from oracle import oracle as O
from tests import cases as K
from tests import toy_models as T

pytestmark = pytest.mark.gpu

TABLE_KEYS = ("flipr", "flipg", "hopr", "hopg", "lst", "site", "ncl", "level", "norb", "sq", "stab_ptr", "stab")

CASES = {
    "bcc_d2h_l2": lambda: K.cubic("bcc", 3, 2, (0.5, 0.5), group="d2h", maxlevel=2),
    "bcc_d4h_l3_r1": lambda: K.cubic("bcc", 3, 2, (0.5, 0.5), group="d4h", maxlevel=3, maxrank=1),
    "fcc_ternary_d2h_l2_r2": lambda: K.cubic("fcc", 3, 3, (0.66, 0.14, 0.2), group="d2h", maxlevel=2, maxrank=2),
    "bcc_identity_l2": lambda: K.cubic("bcc", 2, 2, (0.5, 0.5), group="identity", maxlevel=2),
    "bcc_flippable_start": lambda: K.cubic("bcc", 3, 2, (0.3, 0.7), group="d4h", maxlevel=2, start_flippable=True),
    "ring_three_classes": K.ring,
}


@pytest.fixture(scope="module", params=sorted(CASES))
def pair(request):
    case = CASES[request.param]()
    gop, oop = K.build_both(case, A.build_augcls_operator, O.OracleOp)
    return request.param, case, gop, oop


def test_tables_bit_exact(pair):
    name, case, gop, oop = pair
    assert gop.nn == oop.nn and gop.nslot == oop.nslot and gop.nstab == oop.nstab, name
    tg, to = gop.tables(), oop.tables()
    for k in TABLE_KEYS:
        assert np.array_equal(tg[k], to[k]), (name, k)


def _params(case, oop):
    return K.general_params(case["model"].nsp)


def test_apply_general_operator(pair):
    name, case, gop, oop = pair
    c, d, o, e = _params(case, oop)
    for op in (gop, oop):
        op.set_params(c, d, o, e)
    rng = np.random.default_rng(1)
    x = rng.uniform(-0.5, 0.5, (gop.dim, 3))
    yg = gop.apply(x)
    for j in range(3):
        yo = oop.apply(x[:, j])
        assert np.max(np.abs(yg[:, j] - yo)) <= 1e-12 * np.max(np.abs(yo)), name


def test_apply_with_frozen_start(pair):
    name, case, gop, oop = pair
    if case["flippable"][0]:
        pytest.skip("start site flippable")
    c, d, o, e = _params(case, oop)
    for op in (gop, oop):
        op.set_params(c, d, o, e)
        op.unfreeze()
        op.freeze_site(1, int(case["model"].spc[0, case["cls"][0] - 1]))
    x = np.random.default_rng(2).uniform(-0.5, 0.5, gop.dim)
    yg, yo = gop.apply(x), oop.apply(x)
    assert np.max(np.abs(yg - yo)) <= 1e-12 * np.max(np.abs(yo)), name
    for op in (gop, oop):
        op.unfreeze()


def test_rand_c_and_project(pair):
    name, case, gop, oop = pair
    nsp = case["model"].nsp
    rng = np.random.default_rng(4)
    par = rng.uniform(-1, 1, (9, nsp)) + 1j * rng.uniform(-1, 1, (9, nsp))
    x = rng.uniform(-0.5, 0.5, gop.dim) + 1j * rng.uniform(-0.5, 0.5, gop.dim)
    for op in (gop, oop):
        op.set_start(1)
    wg, wo = gop.rand_c(par, x), oop.rand_c(par, x)
    assert np.max(np.abs(wg - wo)) <= 1e-13 * np.max(np.abs(wo)), name
    pg, po = gop.project_c(x), oop.project_c(x)
    assert np.max(np.abs(pg - po)) <= 1e-14 * np.max(np.abs(po)), name


def _edc_compare(gop, oop, ed, zs, l0, nlev, depth_tol, tail, precision="fp64"):
    for op in (gop, oop):
        op.set_start(l0)
    g, m, a, b = A.edc_green_blk(gop, ed, zs, l0, nlev, depth_tol=depth_tol, tail=tail, precision=precision)
    go, mo, ao, bo = oop.edc_green_blk(ed, zs, l0, nlev, depth_tol=depth_tol, tail=tail)
    return g, m, a, b, go, mo, ao, bo


@pytest.mark.parametrize("tail", ["hull", "bp", "avg2", "none"])
def test_edc_chains_match_oracle(tail):
    case = K.cubic("bcc", 3, 2, (0.5, 0.5), group="d4h", maxlevel=3, maxrank=1)
    gop, oop = K.build_both(case, A.build_augcls_operator, O.OracleOp)
    ed = S.edc_params(S.draw_species(2, 0), 1)
    for op in (gop, oop):
        op.set_params(ed["c"], ed["d"], ed["o"], ed["e"])
        op.unfreeze()
        op.freeze_site(1, 1)
    zs = np.linspace(-0.6, 0.4, 40) + 0.02j
    g, m, a, b, go, mo, ao, bo = _edc_compare(gop, oop, ed, zs, 5, 20, 0.0, tail)
    assert np.array_equal(m, mo)
    for j in range(len(zs)):
        mj = m[j]
        assert np.max(np.abs(a[:mj, j] - ao[:mj, j]) / np.abs(ao[:mj, j])) < 1e-9
        assert np.max(np.abs(b[: mj - 1, j] - bo[: mj - 1, j]) / np.abs(bo[: mj - 1, j])) < 1e-9
    assert np.max(np.abs(g - go) / np.abs(go)) < 1e-8


def test_edc_general_operator_with_o_and_depth_tol():
    case = K.cubic("fcc", 3, 3, (0.66, 0.14, 0.2), group="d2h", maxlevel=2, maxrank=1)
    gop, oop = K.build_both(case, A.build_augcls_operator, O.OracleOp)
    sp = T.species_lmto(3, seed=9)
    ed = T.edc_setup(sp, 2)                 # o != 0, d uniform: the two-h path of blk_hamx
    for op in (gop, oop):
        op.set_params(ed["c"], ed["d"], ed["o"], ed["e"])
        op.unfreeze()
        op.freeze_site(1, 2)
    zs = np.linspace(-0.3, 0.3, 33) + 0.05j
    g, m, a, b, go, mo, ao, bo = _edc_compare(gop, oop, ed, zs, 3, 24, 1e-5, "hull")
    assert np.array_equal(m, mo)
    assert np.max(np.abs(g - go) / np.abs(go)) < 1e-8


def test_edc_depth_test_stops_where_the_oracle_stops():
    """The depth test |G_k - G_{k-4}| <= tol |G_k| (src/asr_edc.f90:121-127) near the real axis, where the stopping depth
    varies from energy to energy."""
    case = K.cubic("bcc", 3, 2, (0.5, 0.5), group="d4h", maxlevel=3, maxrank=1)
    gop, oop = K.build_both(case, A.build_augcls_operator, O.OracleOp)
    ed = S.edc_params(S.draw_species(2, 8), 1)
    for op in (gop, oop):
        op.set_params(ed["c"], ed["d"], ed["o"], ed["e"])
        op.unfreeze()
        op.freeze_site(1, 1)
    zs = np.linspace(-0.8, 0.4, 41) + 0.01j
    g, m, a, b, go, mo, ao, bo = _edc_compare(gop, oop, ed, zs, 1, 40, 1e-3, "hull")
    assert np.array_equal(m, mo)
    assert len(set(m.tolist())) > 1
    assert np.max(np.abs(g - go) / np.abs(go)) < 1e-8


def test_edc_fp32_matvec_error_is_bounded():
    case = K.cubic("bcc", 3, 2, (0.5, 0.5), group="d4h", maxlevel=3, maxrank=1)
    gop, oop = K.build_both(case, A.build_augcls_operator, O.OracleOp)
    ed = S.edc_params(S.draw_species(2, 0), 2)
    for op in (gop, oop):
        op.set_params(ed["c"], ed["d"], ed["o"], ed["e"])
        op.unfreeze()
        op.freeze_site(1, 2)
    zs = np.linspace(-0.6, 0.4, 32) + 0.02j
    g32, *_ = A.edc_green_blk(gop, ed, zs, 1, 20, precision="fp32")
    for op in (gop, oop):
        op.set_start(1)
    go, *_ = oop.edc_green_blk(ed, zs, 1, 20)
    err = np.max(np.abs(g32 - go)) / np.max(np.abs(go))
    assert err < 1e-4, err


def test_plain_lanczos_and_bp_dos_match_oracle():
    case = K.cubic("bcc", 3, 2, (0.5, 0.5), group="d2h", maxlevel=3, start_flippable=True)
    gop, oop = K.build_both(case, A.build_augcls_operator, O.OracleOp)
    c, d, o, e = S.plain_params(S.draw_species(2, 0))
    for op in (gop, oop):
        op.set_params(c, d, o, e)
    z = np.linspace(-1.2, 0.8, 200) + 0.005j
    specs = []
    for l0 in range(1, 10):
        gop.set_start(l0)
        oop.set_start(l0)
        a, b, n = A.lanczos(gop, l0, 12)
        v0 = np.zeros(oop.dim)
        v0[l0 - 1] = 1.0
        with O.apply_threads():   # 2.8 M nodes: the oracle's node loops on every host thread (the same bits)
            ao, bo, no = oop.lanczos(v0, 12)
        assert n == no
        assert np.max(np.abs(a[:n] - ao[:n]) / np.abs(ao[:n])) < 1e-9
        assert np.max(np.abs(b[:n] - bo[:n]) / np.abs(bo[:n])) < 1e-9
        specs.append(A.ChainSpec(c=c, d=d, o=o, e=e, start_orb=l0, nlev=12))
        gref, _ = O.terminated_green(ao, bo, no, z, "beer-pettifor")
        if l0 == 1:
            r = A.chains_run(gop, specs[:1], z, mode="plain", tail="bp")
            dos, dos_o = -r["g"][:, 0].imag / np.pi, -gref.imag / np.pi
            assert np.max(np.abs(dos - dos_o)) < 1e-8
    r = A.chains_run(gop, specs, z, mode="plain", tail="bp")
    assert r["g"].shape == (200, 9)


def test_cf_species_on_golden_chains(golden):
    for name in ("cr1", "cr2"):
        c = golden[name]
        a = np.array(c["re_a"]) + 1j * np.array(c["im_a"])
        b = np.array(c["re_b"]) + 1j * np.array(c["im_b"])
        z = complex(*golden["zc1" if name == "cr1" else "zc2"])
        zz = z + np.linspace(-0.05, 0.05, 11)
        for tail in ("none", "hull", "bp", "avg2"):
            g = A.cf_species(a, b, 24, zz.reshape(-1, 1), tail)[:, 0]
            go = np.array([O.cf_species(a, b, 24, zj, tail)[0] for zj in zz])
            assert np.max(np.abs(g - go) / np.abs(go)) < 1e-10, (name, tail)


def test_ring_recursion_on_gpu_equals_exact_average():
    case = K.ring()
    g = case["graph"]
    mdl = case["model"]
    sp = T.species_lmto()
    gop = A.build_augcls_operator(g, mdl, case["cls"], case["perm"], case["dmat"], 1, 80, flippable=case["flippable"])
    err = 0.0
    for cen in (1,):
        ed = T.edc_setup(sp, cen)
        gop.set_params(ed["c"], ed["d"], ed["o"], ed["e"])
        gop.unfreeze()
        gop.freeze_site(1, cen)
        zs = np.array([complex(-0.3 + 0.3 * kz, 0.3) for kz in (1, 2, 3)])
        for l0 in (1, 5, 9):
            gop.set_start(l0)
            gg, m, a, b = A.edc_green_blk(gop, ed, zs, l0, 128, tail="none")
            for j, z in enumerate(zs):
                gden, _ = T.exact_average(mdl, g, [1, 2, 3, 2], cen, sp, z, l0)
                err = max(err, abs(gg[j] - gden))
    assert err < 1e-6, err
