"""KPM on an explicit supercell through the C-ABI against the oracle's kpm_moments (src/reference/asr_kpm.f90:39-65) on the
same counter-based Rademacher vectors; FP64 moments agree to rounding, FP32-matvec moments within a stated bound; the
realisation operator (o != 0 included) equals the oracle's real_apply."""
import numpy as np
import pytest

from asr_b200 import kpm
from asr_b200 import synthetic as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cell():
    nbr, spc, bvec, _ = kpm.fcc_supercell(3, [0.66, 0.14, 0.20], -0.10, seed=4, sweeps=10)
    block, block0 = S.sk_blocks(bvec, 4)
    sp = S.draw_species(3, 4)
    c, d, o, e = S.plain_params(sp)
    return dict(nbr=nbr, spc=spc, block=block, block0=block0, c=c, d=d, o=o, e=e)


def test_supercell_apply_general(cell):
    rng = np.random.default_rng(0)
    o = np.asfortranarray(rng.uniform(-0.3, 0.3, (9, 3)))
    e = np.asfortranarray(rng.uniform(-0.1, 0.1, (9, 3)))
    sc = kpm.Supercell(cell["nbr"], cell["spc"], cell["c"], cell["d"], o, e, cell["block"], cell["block0"])
    x = rng.uniform(-0.5, 0.5, sc.dim)
    y = sc.apply(x)
    yo = O.real_apply(cell["nbr"], cell["spc"], cell["c"], cell["d"], o, e, cell["block"], cell["block0"], x)
    assert np.max(np.abs(y - yo)) <= 1e-12 * np.max(np.abs(yo))


@pytest.mark.parametrize("doubling", [False, True])
def test_kpm_moments_fp64_match_oracle(cell, doubling):
    sc = kpm.Supercell(cell["nbr"], cell["spc"], cell["c"], cell["d"], cell["o"], cell["e"], cell["block"], cell["block0"])
    cen, scl = -0.2, 2.5
    mu = sc.kpm_moments(cen, scl, 64, 4, seed=7, doubling=doubling)
    mo = O.kpm_moments(cell["nbr"], cell["spc"], cell["c"], cell["d"], cell["o"], cell["e"], cell["block"], cell["block0"], cen, scl,
                       64, 0, 4, 7)
    assert abs(mu[0] - 1.0) < 1e-15
    assert np.max(np.abs(mu - mo)) < 1e-11


def test_kpm_fp32_error_and_dos(cell):
    sc = kpm.Supercell(cell["nbr"], cell["spc"], cell["c"], cell["d"], cell["o"], cell["e"], cell["block"], cell["block0"])
    cen, scl = -0.2, 2.5
    m64 = sc.kpm_moments(cen, scl, 128, 8, seed=3)
    m32 = sc.kpm_moments(cen, scl, 128, 8, seed=3, precision="fp32")
    assert np.max(np.abs(m32 - m64)) < 1e-4
    e = np.linspace(-2.5, 2.0, 400)
    r64 = kpm.kpm_dos(m64, cen, scl, e)
    ro = O.kpm_dos(m64, cen, scl, e)
    assert np.max(np.abs(r64 - ro)) < 1e-12
    # the DOS integrates to 1 per orbital (states per orbital and unit energy)
    assert abs(np.trapezoid(r64, e) - 1.0) < 2e-2


def test_kpm_moments_general_operator(cell):
    # o != 0 and e != 0: the three-pass operator of real_apply inside the Chebyshev recursion
    rng = np.random.default_rng(5)
    o = np.asfortranarray(rng.uniform(-0.2, 0.2, (9, 3)))
    e = np.asfortranarray(rng.uniform(-0.1, 0.1, (9, 3)))
    sc = kpm.Supercell(cell["nbr"], cell["spc"], cell["c"], cell["d"], o, e, cell["block"], cell["block0"])
    cen, scl = -0.2, 3.0
    mu = sc.kpm_moments(cen, scl, 32, 2, seed=9, doubling=False)
    mo = O.kpm_moments(cell["nbr"], cell["spc"], cell["c"], cell["d"], o, e, cell["block"], cell["block0"], cen, scl, 32, 0, 2, 9)
    assert np.max(np.abs(mu - mo)) < 1e-11
