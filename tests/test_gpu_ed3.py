"""Route ed3 (src/asr_ed3.f90) on the GPU against the oracle's restatement: chain coefficients a, b and projections c
of both chains (1e-9), depths, and the central blocks bk = (G_11, (hG)_11, (hGh)_11, q1 mismatch) (1e-8)."""
import numpy as np
import pytest

from asr_b200 import augcls as A
from asr_b200 import chains as CH
from asr_b200 import synthetic as S
from oracle.oracle import OracleOp
from tests import cases as K

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pair():
    case = K.cubic("bcc", 3, 2, (0.5, 0.5), group="d4h", maxlevel=3, maxrank=1)
    args = (case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, case["maxlevel"])
    return A.build_augcls_operator(*args, maxrank=case["maxrank"], flippable=case["flippable"]), OracleOp(*args, case["maxrank"],
                                                                                                        case["flippable"])


def _groups(seed=6):
    sp = S.draw_species(2, seed)
    rng = np.random.default_rng(seed)
    o, p = rng.uniform(0.0, 0.15, (2, 3)), rng.uniform(0.0, 0.05, (2, 3))
    out = []
    for central, orb, nlev in ((1, 1, 16), (2, 5, 12), (1, 3, 20)):
        g = S.ed3_params(sp, central, o, p)
        g.update(start_orb=orb, nlev=nlev)
        out.append(g)
    return out


def _oracle(oop, g, zs, depth_tol, tail):
    z9 = np.zeros_like(g["g"])
    oop.set_params(g["g"], g["d"], z9, z9)
    oop.unfreeze()
    oop.freeze_site(1, g["central"])
    oop.set_start(g["start_orb"])
    return oop.ed3_blocks(g, zs, g["start_orb"], g["nlev"], depth_tol=depth_tol, tail=tail)


@pytest.mark.parametrize("tail,depth_tol", [("hull", 0.0), ("none", 0.0), ("avg2", 0.0), ("bp", 0.0), ("hull", 3e-3)])
def test_ed3_matches_oracle(pair, tail, depth_tol):
    gop, oop = pair
    groups = _groups()
    zs = np.linspace(-0.45, 0.25, 9) + 0.08j
    r = CH.ed3_blocks(gop, groups, zs, depth_tol=depth_tol, tail=tail, coefs=True)
    for q, g in enumerate(groups):
        bk, m, a, b, c = _oracle(oop, g, zs, depth_tol, tail)
        assert np.array_equal(r["m"][:, :, q], m), q
        for j in range(len(zs)):
            for kd in range(2):
                mm = m[kd, j]
                ga, oa = r["a"][:mm, kd, j, q], a[j, kd, :mm]
                assert np.max(np.abs(ga - oa) / np.abs(oa)) < 1e-9
                gb_, ob = r["b"][:mm - 1, kd, j, q], b[j, kd, :mm - 1]
                assert np.max(np.abs(gb_ - ob) / np.abs(ob)) < 1e-9
                gc, oc = r["c"][:mm, kd, j, q], c[j, kd, :mm]
                assert np.max(np.abs(gc - oc)) < 1e-9 * np.max(np.abs(oc))
        scale = np.max(np.abs(bk[:3]))
        assert np.max(np.abs(r["bk"][:, :, q] - bk)) < 1e-8 * scale, q


def test_ed3_fp32_error_is_bounded(pair):
    gop, _ = pair
    groups = _groups(7)
    zs = np.linspace(-0.4, 0.2, 6) + 0.1j
    b64 = CH.ed3_blocks(gop, groups, zs, tail="hull")["bk"]
    b32 = CH.ed3_blocks(gop, groups, zs, tail="hull", precision="fp32")["bk"]
    assert np.max(np.abs(b32[:3] - b64[:3])) < 1e-4 * np.max(np.abs(b64[:3]))
