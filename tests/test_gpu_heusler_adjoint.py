"""Adjoint on the L2_1 four-sublattice bcc alloy (one sublattice Cr0.6Fe0.4-like, the others ordered): the Jacobian of
the band energy and the four sublattice charges with respect to all 45 species parameters (c_l, d_l, Delta_l for
l = s, p, d and 5 species), through torch.autograd and the device adjoint: with o = 0 against central differences
(h = 1e-5, Richardson-extrapolated) of the CUDA forward, and with edc_setup's o against the oracle's central differences
(all 45 x 5 entries, the committed fixture of tests/golden/make_c3_jacobian.py)."""
import numpy as np
import pytest
import torch

from asr_b200 import classes as CL
from asr_b200 import contour as CT
from asr_b200 import synthetic as S

pytestmark = pytest.mark.gpu

H = 1e-5
NLEV = 20


@pytest.fixture(scope="module")
def system():
    cases = [S.heusler_case(4, 3, k) for k in (1, 2, 3, 4)]
    sc = CL.SublatticeChains(cases, NLEV)
    sp = S.draw_species(5, 3)
    z, w = CT.contour_nodes(-1.2, 0.2, 32)
    return cases, sc, sp, z, w


def _params(sp):
    return [torch.tensor(x, dtype=torch.float64, requires_grad=True) for x in (sp.c, sp.d, sp.delta)]


def test_jacobian_of_band_energy_and_charges(system):
    cases, sc, sp, z, w = system
    enu = torch.zeros(5, 3, dtype=torch.float64)
    params = _params(sp)
    e_band, q = sc.energy_and_charges(*params, enu, z, w)
    outs = [e_band] + [q[k] for k in range(4)]
    jac = np.zeros((5, 45))
    for r, o in enumerate(outs):
        gr = torch.autograd.grad(o, params, retain_graph=True)
        jac[r] = np.concatenate([g.numpy().ravel() for g in gr])
    assert np.all(np.isfinite(jac)) and np.max(np.abs(jac)) > 0

    def f(vals):
        with torch.no_grad():
            e, qq = sc.energy_and_charges(*[torch.tensor(v) for v in vals], enu, z, w)
        return np.concatenate([[e.item()], qq.numpy()])

    base = [p.detach().numpy().copy() for p in params]
    worst, where = 0.0, None
    for k in range(45):
        a, idx = divmod(k, 15)

        def shifted(h):
            v = [x.copy() for x in base]
            v[a].ravel()[idx] += h
            return f(v)
        d1 = (shifted(H) - shifted(-H)) / (2 * H)
        d2 = (shifted(H / 2) - shifted(-H / 2)) / H
        fd = (4 * d2 - d1) / 3
        for r in range(5):
            # relative to the derivative itself, floored at 1e-3 of the Jacobian's largest entry: entries that vanish
            # (charges of ordered sublattices are nearly fixed by the contour) are compared on that scale
            err = abs(jac[r, k] - fd[r]) / max(abs(fd[r]), 1e-3 * np.max(np.abs(jac)))
            if err > worst:
                worst, where = err, (r, k, jac[r, k], fd[r])
    assert worst < 1e-6, (worst, where)


def test_jacobian_with_o_against_oracle_central_differences():
    """All 45 parameters x 5 outputs with edc_setup's o (o_l D_s / D_c) against the oracle's central differences
    (tests/golden/c3_oracle_jacobian.json, made by tests/golden/make_c3_jacobian.py), h = 1e-5 and h / 2.

    The plain central difference at h = 1e-5 carries a truncation error of up to 4.3e-6 of the entry (its distance from
    the Richardson combination of h and h / 2), so the 1e-6 comparison is made against the Richardson column:
    |J - R| <= 1e-6 |R| + F_r, where F_r = 8 eps |f_r| / h (1.4e-9 to 1.6e-9 per output) bounds the rounding of R; F_r is
    at most 1e-6 of every entry above 1.6e-3 in magnitude, and the entries below it (the charges of the two ordered
    sublattices whose derivatives vanish or nearly so, and small couplings) are held to F_r itself.  Against the h column
    itself: |J - D_h| <= |D_h - R| + 1e-6 |R| + F_r."""
    import json
    import os

    from tests import heusler_oracle as HO
    fx = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c3_oracle_jacobian.json")))
    fd = np.array(fx["central_h"])
    rich = np.array(fx["richardson"])
    vals = np.array(fx["values"])
    floor = (8 * np.finfo(float).eps * np.abs(vals) / fx["h"])[:, None]
    cases, sp, ol, z, w = HO.configuration()
    sc = CL.SublatticeChains(cases, HO.NLEV)
    enu = torch.zeros(5, 3, dtype=torch.float64)
    params = _params(sp)
    olt = torch.tensor(ol, dtype=torch.float64)
    e_band, q = sc.energy_and_charges(*params, enu, z, w, olt)
    assert abs(e_band.item() - vals[0]) <= 1e-9 * abs(vals[0])
    assert np.max(np.abs(q.detach().numpy() - vals[1:])) <= 1e-9 * np.max(np.abs(vals[1:]))
    outs = [e_band] + [q[k] for k in range(4)]
    jac = np.zeros((5, 45))
    for r, o in enumerate(outs):
        gr = torch.autograd.grad(o, params, retain_graph=True)
        jac[r] = np.concatenate([g.numpy().ravel() for g in gr])
    err = np.abs(jac - rich) - (1e-6 * np.abs(rich) + floor)
    r, k = np.unravel_index(np.argmax(err), err.shape)
    assert np.all(err <= 0), (r, k, jac[r, k], rich[r, k])
    err_h = np.abs(jac - fd) - (np.abs(fd - rich) + 1e-6 * np.abs(rich) + floor)
    assert np.all(err_h <= 0)
