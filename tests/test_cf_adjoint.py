"""Reverse mode of cf_species (src/asr_chain.f90:67-167) in the library's host entry point asr_cf_adjoint, against
central differences of the oracle's cf_species, on the reference's golden chains cr1 and cr2
(test/test_terminators.f90:25-76), for every tail: none, hull (eigenvalue derivatives of the chain matrix), Beer-Pettifor
(implicit derivative of the fixed point) and avg2.  G is holomorphic in (a, b), so a real step gives the complex
derivative."""
import ctypes as C

import numpy as np
import pytest

from asr_b200 import _lib
from oracle import oracle as O

H = 1e-6


def _pd(x):
    return x.ctypes.data_as(C.POINTER(C.c_double))


def _adjoint(a, b, m, z, tail, w=1.0 + 0.0j):
    ab = np.zeros(m, np.complex128)
    bb = np.zeros(m, np.complex128)
    g = np.zeros(2)
    _lib.check(_lib.lib().asr_cf_adjoint(_pd(np.ascontiguousarray(a[:m])), _pd(np.ascontiguousarray(b[:m])), m, z.real, z.imag,
                                         _lib.TAILS[tail], w.real, w.imag, _pd(ab), _pd(bb), _pd(g)))
    return complex(g[0], g[1]), ab, bb


@pytest.mark.parametrize("tail", ["none", "hull", "bp", "avg2"])
@pytest.mark.parametrize("name", ["cr1", "cr2"])
def test_fraction_adjoint_matches_oracle_differences(golden, tail, name):
    c = golden[name]
    a = np.array(c["re_a"]) + 1j * np.array(c["im_a"])
    b = np.array(c["re_b"]) + 1j * np.array(c["im_b"])
    z0 = complex(*golden["zc1" if name == "cr1" else "zc2"])
    for m in (24, 12):
        for dz in (-0.03, 0.0, 0.04):
            z = z0 + dz
            g, ab, bb = _adjoint(a, b, m, z, tail)
            assert abs(g - O.cf_species(a, b, m, z, tail)[0]) <= 1e-10 * abs(g)
            scale = max(np.max(np.abs(ab)), np.max(np.abs(bb[: m - 1])))
            for k in range(m):
                for arr, gr, nmax in ((a, ab, m), (b, bb, m - 1)):
                    if k >= nmax:
                        continue
                    xp, xm = arr.copy(), arr.copy()
                    xp[k] += H
                    xm[k] -= H
                    args_p = (xp, b) if arr is a else (a, xp)
                    args_m = (xm, b) if arr is a else (a, xm)
                    fd = (O.cf_species(*args_p, m, z, tail)[0] - O.cf_species(*args_m, m, z, tail)[0]) / (2 * H)
                    assert abs(gr[k] - fd) <= 1e-6 * max(abs(fd), 1e-3 * scale), (tail, name, m, dz, k, gr[k], fd)
