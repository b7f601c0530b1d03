"""Complex-energy contours (src/asr_contour.f90) through the library's host entry points."""
from __future__ import annotations

import numpy as np

from ._lib import check, lib
from .augcls import _pd


def gauss_legendre(n: int):
    x, w = np.zeros(n), np.zeros(n)
    check(lib().asr_gauss_legendre(n, _pd(x), _pd(w)))
    return x, w


def contour_nodes(ebot: float, ef: float, n: int, eta_end: float | None = None):
    """``contour_nodes`` (:17-34): semicircle from E_bot to E_F through the upper half plane."""
    z, w = np.zeros(n, np.complex128), np.zeros(n, np.complex128)
    check(lib().asr_contour_nodes(ebot, ef, n, -1.0 if eta_end is None else eta_end, _pd(z.view(np.float64)), _pd(w.view(np.float64))))
    return z, w


def contour_nodes_closed(ebot: float, ef: float, eta: float, n_arc: int, n_vert: int):
    """``contour_nodes_closed`` (:39-58)."""
    z, w = np.zeros(n_arc + n_vert, np.complex128), np.zeros(n_arc + n_vert, np.complex128)
    check(lib().asr_contour_nodes_closed(ebot, ef, eta, n_arc, n_vert, _pd(z.view(np.float64)), _pd(w.view(np.float64))))
    return z, w


def fermi_npole(kt: float) -> int:
    """``fermi_npole`` (:61-64)."""
    return max(2, min(40, int(np.rint(0.1 / (2.0 * np.pi * kt)))))


def contour_nodes_fermi(ebot: float, mu: float, kt: float, npole: int, n_main: int, n_step: int):
    """``contour_nodes_fermi`` (:77-121)."""
    n = 4 + n_main + n_step + 8 + npole
    z, w = np.zeros(n, np.complex128), np.zeros(n, np.complex128)
    check(lib().asr_contour_nodes_fermi(ebot, mu, kt, npole, n_main, n_step, _pd(z.view(np.float64)), _pd(w.view(np.float64))))
    return z, w


def contour_moment(z, w, g, enu: float, k: int) -> float:
    """``contour_moment`` (:124-130): -(1/pi) Im sum_j w_j (z_j - enu)^k g_j."""
    z = np.ascontiguousarray(z, np.complex128)
    w = np.ascontiguousarray(w, np.complex128)
    g = np.ascontiguousarray(g, np.complex128)
    m = np.zeros(1)
    check(lib().asr_contour_moment(_pd(z.view(np.float64)), _pd(w.view(np.float64)), _pd(g.view(np.float64)), z.shape[0], enu, k,
                                   _pd(m)))
    return float(m[0])
