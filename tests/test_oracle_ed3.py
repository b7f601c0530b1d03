"""The oracle's route ed3 (src/asr_ed3.f90) on CPU: with o = p = 0 the secular matrix K' reduces to et - h', so the
|a> = |u> chain is the edc chain (src/asr_edc.f90:75-164) and G_11 equals edc_green's G; with o, p != 0 the two estimates
of q1 from the |a> and |v> chains agree to the residual of the fraction."""
import numpy as np

from asr_b200 import synthetic as S
from oracle.oracle import OracleOp
from tests import cases as K


def _op():
    case = K.cubic("bcc", 3, 2, (0.5, 0.5), group="d4h", maxlevel=3, maxrank=1)
    return OracleOp(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, case["maxlevel"], case["maxrank"],
                    case["flippable"])


def _prepare(op, e3, iv):
    z = np.zeros_like(e3["g"])
    op.set_params(e3["g"], e3["d"], z, z)
    op.unfreeze()
    op.freeze_site(1, e3["central"])
    op.set_start(iv)


def test_ed3_without_o_and_p_is_the_edc_chain():
    op = _op()
    sp = S.draw_species(2, 5)
    e3 = S.ed3_params(sp, 2)
    ed = S.edc_params(sp, 2)
    iv, nlev = 5, 14
    zs = np.linspace(-0.5, 0.3, 7) + 0.05j
    _prepare(op, e3, iv)
    bk, m, a, b, c = op.ed3_blocks(e3, zs, iv, nlev, tail="hull")
    g_edc = op.edc_green_blk(ed, zs, iv, nlev, tail="hull")[0]
    assert np.max(np.abs(bk[0] - g_edc) / np.abs(g_edc)) < 1e-12
    assert np.all(m == nlev)


def test_ed3_q1_estimates_agree_and_depth_test():
    op = _op()
    sp = S.draw_species(2, 6)
    rng = np.random.default_rng(6)
    e3 = S.ed3_params(sp, 1, o=rng.uniform(0.0, 0.15, (2, 3)), p=rng.uniform(0.0, 0.05, (2, 3)))
    iv = 1
    zs = np.linspace(-0.4, 0.2, 5) + 0.1j
    _prepare(op, e3, iv)
    bk, m, a, b, c = op.ed3_blocks(e3, zs, iv, 24, tail="hull")
    scale = np.max(np.abs(bk[:3]))
    assert np.max(np.abs(bk[3])) < 1e-2 * scale          # the two q1 estimates agree to the residual of the fraction
    bk2, m2, *_ = op.ed3_blocks(e3, zs, iv, 24, depth_tol=3e-3, tail="hull")
    assert np.all(m2 <= 24) and np.any(m2 < 24)
    assert np.max(np.abs(bk2[:3] - bk[:3])) < 1e-2 * scale
