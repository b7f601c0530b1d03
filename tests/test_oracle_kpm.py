"""The oracle's KPM against exact diagonalisation (test/test_kpm.f90:19-43 pattern: moments of the exact spectrum) and
the SRO layout generator against its targets."""
import numpy as np

from asr_b200 import kpm
from asr_b200 import synthetic as S
from oracle import oracle as O


def test_kpm_moments_against_exact_spectrum():
    # small cell: the stochastic trace of T_n against the exact trace; tolerance from the vector count (test_kpm uses 2.5 %)
    nbr, spc, bvec, _ = kpm.fcc_supercell(2, [0.5, 0.5], None, seed=1, sweeps=1)
    block, block0 = S.sk_blocks(bvec, 1)
    c, d, o, e = S.plain_params(S.draw_species(2, 1))
    n = nbr.shape[1]
    H = np.zeros((9 * n, 9 * n))
    for j in range(9 * n):
        x = np.zeros(9 * n)
        x[j] = 1.0
        H[:, j] = O.real_apply(nbr, spc, c, d, o, e, block, block0, x)
    assert np.max(np.abs(H - H.T)) < 1e-12
    ev = np.linalg.eigvalsh(H)
    cen = 0.5 * (ev[0] + ev[-1])
    sc = 0.55 * (ev[-1] - ev[0])
    xs = (ev - cen) / sc
    exact = np.array([np.mean(np.cos(k * np.arccos(xs))) for k in range(40)])
    mu = O.kpm_moments(nbr, spc, c, d, o, e, block, block0, cen, sc, 40, 0, 60, 11)
    assert np.max(np.abs(mu - exact)) < 0.025


def test_sro_layout_hits_target():
    nbr, spc, bvec, a = kpm.fcc_supercell(8, [0.66, 0.14, 0.20], -0.10, seed=4, sweeps=30)
    counts = np.bincount(spc, minlength=4)[1:] / spc.shape[0]
    assert np.allclose(counts, [0.66, 0.14, 0.20], atol=1e-3)
    off = a[~np.eye(3, dtype=bool)]
    assert np.max(np.abs(off + 0.10)) < 5e-3
