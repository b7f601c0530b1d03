"""Contour moments of the simple-cubic band (test/test_contour.f90): the library's contours and ``contour_moment``
integrate the square-root-terminated continued fraction of the sc tight-binding band (hopping -1, 60 plain Lanczos
levels from one site) to the occupied fraction M0 and the band energy M1 up to E_F in {-3, -1, 0}, and the
Fermi-smeared contour (kT = 3 mRy) to M0.

The reference checks against the tetrahedron method on a 40^3 mesh (tolerances 4e-3 / 6e-3).  Here the truth is exact:
with e(k) = -2 (cos x + cos y + cos z) and x, y, z uniform, P(cos z > t) = arccos(t)/pi and
E[cos z; cos z > t] = sqrt(1 - t^2)/pi, so M0 and M1 reduce to a smooth two-dimensional average over x and y (converged
to 1e-6 at 2000^2 midpoints).  The bounds are the reference's and, below them, the measured agreement with margin."""
import numpy as np

import asr_b200
from oracle import oracle as O

NMAX = 60


def _sc_chain(nmax: int = NMAX):
    """Plain Lanczos (src/reference/asr_recursion.f90:17-58) on the sc lattice from one site; a periodic box of side
    124 > 2 nmax is exact for nmax levels (a path that wraps the box is longer than 2 nmax)."""
    n = 124
    u = np.zeros((n, n, n))
    u[0, 0, 0] = 1.0
    up = np.zeros_like(u)
    a, b = np.zeros(nmax), np.zeros(nmax)
    bn = 0.0
    for i in range(nmax):
        w = -sum(np.roll(u, s, ax) for ax in range(3) for s in (1, -1))
        a[i] = np.vdot(u, w)
        w -= a[i] * u + bn * up
        bn = float(np.sqrt(np.vdot(w, w)))
        b[i] = bn
        up, u = u, w / bn
    return a, b


def _cf_green(a, b, z):
    """``cf_green`` (src/reference/asr_greens.f90:80-90) with ``sqrt_tail`` (:12-22) at ``tail_params_avg2`` (:70-76)."""
    n = a.shape[0]
    ainf = 0.5 * (a[n - 1] + a[n - 2])
    binf = float(np.sqrt(0.5 * (b[n - 1] ** 2 + b[n - 2] ** 2)))
    out = np.zeros(len(z), np.complex128)
    for j, zz in enumerate(z):
        g = 1.0 / (zz - a[n - 1] - O.sqrt_tail(zz, ainf, binf))
        for i in range(n - 2, -1, -1):
            g = 1.0 / (zz - a[i] - b[i] * b[i] * g)
        out[j] = g
    return out


def _exact_moments(ef: float, m: int = 2000):
    th = (np.arange(m) + 0.5) * np.pi / m
    c = np.cos(th)
    t = np.clip(-0.5 * ef - c[:, None] - c[None, :], -1.0, 1.0)
    return float(np.mean(np.arccos(t)) / np.pi), float(-6.0 * np.mean(np.sqrt(1.0 - t * t)) / np.pi)


def test_sc_band_contour_moments_against_the_exact_band_integrals():
    a, b = _sc_chain()
    assert abs(a).max() < 1e-12 and abs(b[0] - np.sqrt(6.0)) < 1e-12 and abs(b[1] - 3.0) < 1e-12
    for ef in (-3.0, -1.0, 0.0):
        z, w = asr_b200.contour_nodes(-7.5, ef, 80)
        g = _cf_green(a, b, z)
        m0 = asr_b200.contour_moment(z, w, g, 0.0, 0)
        m1 = asr_b200.contour_moment(z, w, g, 0.0, 1)
        t0, t1 = _exact_moments(ef)
        assert abs(m0 - t0) < 4e-3 and abs(m1 - t1) < 6e-3                    # the reference's bounds
        assert abs(m0 - t0) < 2e-5 and abs(m1 - t1) < 5e-5, (ef, m0, t0, m1, t1)
    kt = 0.003
    npole = asr_b200.fermi_npole(kt)
    z, w = asr_b200.contour_nodes_fermi(-1.5, 0.0, kt, npole, 40, 24)
    for k2 in range(-3, 4):
        eps = 2.0 * kt * k2
        occ = asr_b200.contour_moment(z, w, 1.0 / (z - eps), 0.0, 0)
        assert abs(occ - 1.0 / (np.exp(eps / kt) + 1.0)) < 1e-6
    for mu in (-3.0, -1.0, 0.0):
        z, w = asr_b200.contour_nodes_fermi(-7.5, mu, kt, npole, 80, 24)
        m0 = asr_b200.contour_moment(z, w, _cf_green(a, b, z), 0.0, 0)
        t0 = _exact_moments(mu)[0]
        assert abs(m0 - t0) < 4e-3 and abs(m0 - t0) < 3e-5, (mu, m0, t0)
