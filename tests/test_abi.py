"""The C-ABI library loads and exports every entry point that include/asr_b200.h declares; host-side entry points
(contour) agree with the oracle.  No device calls."""
import ctypes
import os
import re

import numpy as np
import pytest

import asr_b200
from asr_b200 import _lib
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "asr_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*int\s+(asr_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = _declared()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
    assert sorted(_lib.EXPORTS) == names


def test_version_and_error_channel():
    assert asr_b200.lib().asr_version() == 100
    # a device-free argument error: the message comes back through asr_last_error
    rc = asr_b200.lib().asr_gauss_legendre(0, None, None)
    assert rc == _lib.ASR_EINVAL
    assert "gauss_legendre" in _lib.last_error()


def test_gauss_legendre_matches_oracle():
    for n in (1, 2, 5, 16, 48):
        x, w = asr_b200.gauss_legendre(n)
        xo, wo = O.gauss_legendre(n)
        assert np.allclose(x, xo, atol=1e-15) and np.allclose(w, wo, atol=1e-15)
        assert abs(w.sum() - 2.0) < 1e-13


def test_contours_match_oracle():
    z, w = asr_b200.contour_nodes(-0.9, 0.3, 48)
    zo, wo = O.contour_nodes(-0.9, 0.3, 48)
    assert np.max(np.abs(z - zo)) < 1e-14 and np.max(np.abs(w - wo)) < 1e-14
    z, w = asr_b200.contour_nodes(-0.9, 0.3, 32, eta_end=0.01)
    zo, wo = O.contour_nodes(-0.9, 0.3, 32, 0.01)
    assert np.max(np.abs(z - zo)) < 1e-14 and np.max(np.abs(w - wo)) < 1e-14
    z, w = asr_b200.contour_nodes_closed(-0.9, 0.3, 0.05, 24, 8)
    zo, wo = O.contour_nodes_closed(-0.9, 0.3, 0.05, 24, 8)
    assert np.max(np.abs(z - zo)) < 1e-14 and np.max(np.abs(w - wo)) < 1e-14
    kt = 0.001
    npole = asr_b200.fermi_npole(kt)
    z, w = asr_b200.contour_nodes_fermi(-0.9, 0.3, kt, npole, 32, 16)
    zo, wo = O.contour_nodes_fermi(-0.9, 0.3, kt, npole, 32, 16)
    assert np.max(np.abs(z - zo)) < 1e-13 and np.max(np.abs(w - wo)) < 1e-13


def test_contour_integrates_an_analytic_resolvent():
    # a single level at eps: int_C G dz over the closed contour occupies it fully (M0 = 1) when eps < E_F
    eps = -0.2
    z, w = asr_b200.contour_nodes_closed(-0.9, 0.3, 0.05, 48, 16)
    g = 1.0 / (z - eps)
    m0 = asr_b200.contour_moment(z, w, g, 0.0, 0)
    assert abs(m0 - 1.0) < 1e-10
    assert abs(m0 - O.contour_moment(z, w, g, 0.0, 0)) < 1e-14
    m1 = asr_b200.contour_moment(z, w, g, 0.0, 1)
    assert abs(m1 - eps) < 1e-10


def test_fermi_contour_occupation():
    # test/test_contour.f90: the Fermi contour occupies a single level by f(eps)
    kt = 0.002
    mu = 0.0
    npole = asr_b200.fermi_npole(kt)
    z, w = asr_b200.contour_nodes_fermi(-0.9, mu, kt, npole, 48, 32)
    for eps in (-0.3, -0.005, 0.0, 0.004, 0.02):
        g = 1.0 / (z - eps)
        occ = asr_b200.contour_moment(z, w, g, 0.0, 0)
        f = 1.0 / (np.exp((eps - mu) / kt) + 1.0)
        assert abs(occ - f) < 1e-6, (eps, occ, f)


def test_tuning_entry_points_check_their_arguments():
    L = asr_b200.lib()
    assert L.asr_op_set_tuning(None, _lib.FP64, 16, 4, 0) == _lib.ASR_EINVAL
    assert "asr_op_set_tuning" in _lib.last_error()
    assert L.asr_op_tuning(None, _lib.FP64, None, None, None, None) == _lib.ASR_EINVAL


def test_missing_library_fails_loudly(monkeypatch):
    monkeypatch.setattr(_lib, "_LIB", None)
    monkeypatch.setattr(_lib, "LIB_PATH", "/nonexistent/libasr_b200.so")
    with pytest.raises(ImportError):
        _lib.lib()


def test_fortran_binding_matches_the_header():
    """The iso_c_binding module include/asr_b200.f90 has one interface per entry point of the header, each with the same
    number of arguments as its C prototype."""
    src = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "asr_b200.h")).read(), flags=re.S)
    protos = {m.group(1): [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
              for m in re.finditer(r"int\s+(asr_\w+)\s*\(([^)]*)\)\s*;", src)}
    block = open(os.path.join(ROOT, "include", "asr_b200.f90")).read().replace("&\n", "")
    found = re.findall(r"function\s+(asr_\w+)\s*\(([^)]*)\)", block)
    assert {name for name, _ in found} == set(protos)      # one interface per entry point
    for name, args in found:
        assert name in protos, name
        assert len([a for a in args.split(",") if a.strip()]) == len(protos[name]), name


def test_ctypes_argtypes_match_the_header():
    """The ctypes binding declares, for every entry point, as many arguments as its C prototype."""
    src = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "asr_b200.h")).read(), flags=re.S)
    protos = {m.group(1): [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
              for m in re.finditer(r"int\s+(asr_\w+)\s*\(([^)]*)\)\s*;", src)}
    L = asr_b200.lib()
    checked = 0
    for name in _lib.EXPORTS:
        f = getattr(L, name)
        if f.argtypes is None:
            continue
        assert len(f.argtypes) == len(protos[name]), name
        checked += 1
    assert checked >= 30
