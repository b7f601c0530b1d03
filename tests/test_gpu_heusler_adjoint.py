"""Adjoint on the L2_1 four-sublattice bcc alloy (one sublattice Cr0.6Fe0.4-like, the others ordered): the Jacobian of
the band energy and the four sublattice charges with respect to all 45 species parameters (c_l, d_l, Delta_l for
l = s, p, d and 5 species), through torch.autograd and the device adjoint, against central finite differences
(h = 1e-5, Richardson-extrapolated) of the CUDA forward and of the oracle's chain_greens."""
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


def test_charge_gradient_against_oracle_differences(system):
    """Three parameters of the disordered sublattice's species through the oracle's chain_greens (CPU restatement)."""
    from oracle.oracle import OracleOp
    cases, sc, sp, z, w = system
    enu = torch.zeros(5, 3, dtype=torch.float64)
    params = _params(sp)
    _, q = sc.energy_and_charges(*params, enu, z, w)
    gr = torch.autograd.grad(q[3], params)
    case = cases[3]
    oop = OracleOp(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, case["maxlevel"], case["maxrank"],
                   case["flippable"])
    groups, wts = sc.groups(3)
    conc = dict(sc.comps[3])
    orbs = sorted({orb for _, orb, _ in groups})
    comps = [spc for spc, _ in sc.comps[3]]

    def q4(c, d, delta):
        spp = S.SpeciesParams(c=c, d=d, delta=delta, enu=np.zeros((5, 3)))
        eds = [S.edc_params(spp, spc) for spc in comps]
        gz, _ = oop.chain_greens(eds, comps, orbs, np.full((len(comps), len(orbs)), NLEV), z, 4)
        tot = 0.0
        for (spc, orb, nlev), wt in zip(groups, wts):
            g = gz[:, orbs.index(orb), comps.index(spc)]
            tot += conc[spc] * wt * (-np.imag(np.sum(w * g)) / np.pi)
        return tot

    gmax = max(g.abs().max().item() for g in gr)
    for a, s, l in ((0, 3, 2), (1, 4, 1), (2, 3, 0)):   # c_d of species 4, d_p of species 5, Delta_s of species 4
        vals = [sp.c.copy(), sp.d.copy(), sp.delta.copy()]
        vp = [v.copy() for v in vals]
        vm = [v.copy() for v in vals]
        vp[a][s, l] += H
        vm[a][s, l] -= H
        vp2 = [v.copy() for v in vals]
        vm2 = [v.copy() for v in vals]
        vp2[a][s, l] += H / 2
        vm2[a][s, l] -= H / 2
        d1 = (q4(*vp) - q4(*vm)) / (2 * H)
        d2 = (q4(*vp2) - q4(*vm2)) / H
        fd = (4 * d2 - d1) / 3   # Richardson-extrapolated central difference
        adj = gr[a][s, l].item()
        assert abs(adj - fd) <= 1e-6 * max(abs(fd), 1e-2 * gmax), (a, s, l, adj, fd)
