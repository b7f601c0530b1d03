"""The oracle's continued fractions and terminators against asr's own known answers (test/test_terminators.f90) and
against scipy's LAPACK (the reference calls zgeev / dsterf)."""
import numpy as np
import pytest
import scipy.linalg as sla

from oracle import oracle as O


def _chain(d, name):
    c = d[name]
    return np.array(c["re_a"]) + 1j * np.array(c["im_a"]), np.array(c["re_b"]) + 1j * np.array(c["im_b"])


def _nevanlinna_ratio(golden, tail):
    # test/test_terminators.f90:157-163
    a1, b1 = _chain(golden, "cr1")
    a2, b2 = _chain(golden, "cr2")
    z1 = complex(*golden["zc1"])
    z2 = complex(*golden["zc2"])
    g1 = O.cf_species(a1, b1, 24, z1, tail)[0]
    g2 = O.cf_species(a2, b2, 24, z2, tail)[0]
    return abs(g2 - g1) / abs(z2 - z1) / (min(-g1.imag, -g2.imag) / z1.imag)


def test_golden_chain_hull_obeys_nevanlinna(golden):
    # test/test_terminators.f90:150-152: hull ratio < 1 (about 0.4)
    assert _nevanlinna_ratio(golden, "hull") < golden["expect"]["hull_ratio_below"]


def test_golden_chain_bp_breaks_nevanlinna(golden):
    # test/test_terminators.f90:153: the bp tail exceeds the bound on the same chains
    assert _nevanlinna_ratio(golden, "bp") > golden["expect"]["bp_ratio_above"]


def test_golden_chain_eigenvalues_match_lapack(golden):
    for name in ("cr1", "cr2"):
        a, b = _chain(golden, name)
        for m in (8, 12, 16, 20, 24):
            T = np.diag(a[:m]) + np.diag(b[: m - 1], 1) + np.diag(b[: m - 1], -1)
            ref = np.sort_complex(sla.eigvals(T))
            got = np.sort_complex(O.chain_eigvals(a[:m], b[:m]))
            scale = np.max(np.abs(ref))
            # match each reference eigenvalue to its nearest computed one
            err = max(np.min(np.abs(got - r)) for r in ref) / scale
            assert err < 1e-12, (name, m, err)


def test_random_chains_eigenvalue_extremes_match_lapack():
    rng = np.random.default_rng(7)
    for trial in range(200):
        m = int(rng.integers(2, 33))
        a = rng.uniform(-1, 1, m) + 1j * rng.uniform(-0.3, 0.3, m)
        b = rng.uniform(0.2, 1.0, m) + 1j * rng.uniform(-0.2, 0.2, m)
        T = np.diag(a) + np.diag(b[: m - 1], 1) + np.diag(b[: m - 1], -1)
        ref = sla.eigvals(T)
        got = O.chain_eigvals(a, b)
        for sel in (np.argmin, np.argmax):
            r = ref[sel(ref.real)]
            g = got[sel(got.real)]
            assert abs(r - g) <= 1e-11 * max(1.0, np.max(np.abs(ref))), (trial, r, g)


def test_bp_uniform_chain_converges():
    # test/test_terminators.f90:90-96: BP on a uniform chain recovers (0, 1) as depth grows
    a = np.zeros(60)
    b = np.ones(60)
    for n in (8, 24, 40, 56):
        ainf, binf, _, _ = O.bp_asymptote(a, b, n)
    assert abs(binf - 1.0) < 1e-2 and abs(ainf) < 1e-12


def test_cf_species_bp_equals_bp_asymptote(golden):
    # test/test_terminators.f90:127-143
    a = np.array(golden["chain6_a"])
    b = np.array(golden["chain6_b"])
    ainf, binf, _, _ = O.bp_asymptote(a, b, 6)
    d = 0.0
    for ie in range(9):
        z = complex(-2.4 + 0.6 * ie, 0.05)
        g1 = O.cf_species(a.astype(complex), b.astype(complex), 6, z, "bp")[0]
        g2 = 1.0 / (z - a[5] - O.sqrt_tail(z, ainf, binf))
        for k in range(4, -1, -1):
            g2 = 1.0 / (z - a[k] - b[k] ** 2 * g2)
        d = max(d, abs(g1 - g2))
    assert d <= 1e-10


def test_luchini_nex_interpolation():
    # test/test_terminators.f90:97-103
    a = np.zeros(60)
    b = np.ones(60)
    a[7] = 0.4
    b[7] = 1.4
    _, tp = O.terminated_green(a, b, 8, np.array([0.3 + 0.1j]), "sqrt-avg2", "luchini-nex", 4)
    assert int(tp[2]) == 12
    ta, tb = O.terminator_coefs(a, b, 8, 4, tp[0], tp[1])
    assert abs(ta[11] - (a[7] + 4.0 / 5.0 * (tp[0] - a[7]))) <= 1e-14
    assert abs(tb[9] - (b[7] + 2.0 / 5.0 * (tp[1] - b[7]))) <= 1e-14


def test_periodic_tail_identities():
    # test/test_terminators.f90:81-89
    z = complex(1.3, 0.2)
    g1 = O.periodic_g(z, [0.4], [1.7])
    g2 = O.sqrt_tail(z, 0.4, 1.7) / 1.7 ** 2
    assert abs(g1 - g2) <= 1e-13
    g1 = O.periodic_g(z, [0.5, -0.5], [1.2, 0.9])
    g2 = 1.0 / (z - 0.5 - 1.2 ** 2 / (z + 0.5 - 0.9 ** 2 * g1))
    assert abs(g1 - g2) <= 1e-13
    assert max(0.0, g1.imag) <= 1e-14


def test_tridiagonal_extremes_match_lapack():
    rng = np.random.default_rng(3)
    for trial in range(100):
        n = int(rng.integers(1, 40))
        d = rng.uniform(-1, 1, n)
        e = rng.uniform(-1, 1, max(n - 1, 0))
        ref = sla.eigvalsh_tridiagonal(d, e) if n > 1 else d
        assert abs(O.tridiag_extreme(d, e, True) - ref[-1]) < 1e-14 * (1 + abs(ref[-1])) * 10
        assert abs(O.tridiag_extreme(d, e, False) - ref[0]) < 1e-14 * (1 + abs(ref[0])) * 10


@pytest.mark.parametrize("tail", ["none", "hull", "avg2"])
def test_cf_species_none_tail_is_exact_resolvent(tail):
    # tail 'none' gives the exact finite-chain resolvent [(z - T)^-1]_11
    rng = np.random.default_rng(11)
    m = 10
    a = rng.uniform(-1, 1, m) + 1j * rng.uniform(-0.1, 0.1, m)
    b = rng.uniform(0.3, 1, m) + 0j
    z = complex(0.1, 0.2)
    g = O.cf_species(a, b, m, z, tail)[0]
    if tail == "none":
        T = np.diag(a) + np.diag(b[: m - 1], 1) + np.diag(b[: m - 1], -1)
        ref = np.linalg.solve(z * np.eye(m) - T, np.eye(m)[:, 0])[0]
        assert abs(g - ref) < 1e-13
    else:
        assert np.isfinite(g)
