"""Inputs of the effective-pair-interaction checks, after the reference's test/test_epi.f90 part (D): a 16-site bcc cell
(periodic, 4^3 half-lattice cube, NN + NNN slots), three species with seeded synthetic parameters (o != 0), the origin
on the thermodynamic path, the partner at (1, 1, 1) frozen, two sites (2, 0, 0) and (0, 2, 0) random ternary
(x = 0.5, 0.3, 0.2); the rest ordered (species 1)."""
import numpy as np

from asr_b200 import epi as EP
from asr_b200 import lattices as lat
from asr_b200 import synthetic as S

LSUP = 2
MG = 2 * LSUP
XC = (0.5, 0.3, 0.2)


def species():
    l = S.ORB_L.astype(float)
    return [EP.EpiPar(e=0.10 * l, c=0.30 - 0.15 * l, d=0.30 - 0.07 * l, o=0.10 - 0.03 * l),
            EP.EpiPar(e=0.05 * l, c=0.45 - 0.10 * l, d=0.27 - 0.06 * l, o=0.12 - 0.04 * l),
            EP.EpiPar(e=0.02 + 0.08 * l, c=0.38 - 0.18 * l, d=0.33 - 0.08 * l, o=0.08 - 0.02 * l)]


def cell(seed: int = 2):
    g, coord, bvec = lat.periodic_graph_shells("bcc", LSUP, 4)
    block, block0 = S.sk_blocks(bvec, seed)

    def site_at(c):
        hit = np.nonzero(np.all((coord - np.asarray(c)[:, None]) % MG == 0, axis=0))[0]
        return int(hit[0]) + 1
    r1, r2, jp = site_at([2, 0, 0]), site_at([0, 2, 0]), site_at([1, 1, 1])
    return dict(graph=g, coord=coord, block=block, block0=block0, r1=r1, r2=r2, jp=jp)


def chain_model(c):
    """Classes 1 (ordered, species 1), 2 (random ternary), 3 (the partner, species 1 until frozen); 4 species (the 4th is
    the path point of site 0)."""
    n = c["graph"].n
    cls = np.ones(n, np.int32)
    cls[c["r1"] - 1] = cls[c["r2"] - 1] = 2
    cls[c["jp"] - 1] = 3
    spc = np.zeros((3, 3), np.int32, order="F")
    conc = np.zeros((3, 3), order="F")
    spc[0, 0], conc[0, 0] = 1, 1.0
    spc[:, 1], conc[:, 1] = [1, 2, 3], XC
    spc[0, 2], conc[0, 2] = 1, 1.0
    mdl = S.ClassModel(nsp=4, nsc=np.array([1, 3, 1], np.int32), spc=spc, conc=conc,
                       block=np.asfortranarray(c["block"].reshape(9, 9, -1, 1)), block0=np.asfortranarray(c["block0"].reshape(9, 9, 1)))
    fl = np.zeros(n, np.int32)
    fl[c["r1"] - 1] = fl[c["r2"] - 1] = 1
    return mdl, cls, fl


def dense_h(c, par, spsite, pt, sj):
    """The dense unscaled H^(2) = E_nu + h - h o h of the cell (oracle's augcls_apply) with species spsite on every site,
    site 1 on the path point pt and the partner on species sj."""
    from oracle.oracle import OracleOp
    n = c["graph"].n
    spc = np.asfortranarray(np.array([[1, 2, 3]], np.int32))
    mdl = S.ClassModel(nsp=4, nsc=np.ones(3, np.int32), spc=spc, conc=np.asfortranarray(np.ones((1, 3))),
                       block=np.asfortranarray(c["block"].reshape(9, 9, -1, 1)), block0=np.asfortranarray(c["block0"].reshape(9, 9, 1)))
    perm1, d1 = lat.identity_group(n)
    op = OracleOp(c["graph"], mdl, np.asarray(spsite, np.int32), perm1, d1, 1, 6, 1, np.zeros(n, np.int32))
    assert op.nn == n
    cc = np.zeros((9, 4), order="F")
    dd, oo, ee = cc.copy(order="F"), cc.copy(order="F"), cc.copy(order="F")
    for s, p in enumerate(par):
        cc[:, s], dd[:, s], oo[:, s], ee[:, s] = p.c, p.d, p.o, p.e
    cc[:, 3], dd[:, 3], oo[:, 3], ee[:, 3] = pt.c, pt.d, pt.o, pt.e
    op.set_params(cc, dd, oo, ee)
    op.freeze_any(1, 4)
    op.freeze_any(c["jp"], sj)
    dim = 9 * n
    h = np.zeros((dim, dim))
    for k in range(dim):
        x = np.zeros(dim)
        x[k] = 1.0
        h[:, k] = op.apply(x)
    return h


def exact_trace(c, par, a, b, lam, sj, z):
    """Configuration average over the two random sites of Tr[(z - H)^-1 dH/dlambda] + 2 sum_L kappa_L (dH by a
    five-point difference of the dense H, step 1e-2)."""
    hs = 1.0e-2
    ref = 0.0
    for s1 in (1, 2, 3):
        for s2 in (1, 2, 3):
            spsite = np.ones(c["graph"].n, np.int32)
            spsite[c["r1"] - 1], spsite[c["r2"] - 1] = s1, s2
            spsite[c["jp"] - 1] = 1
            hh = {q: dense_h(c, par, spsite, EP.epi_path(par[a - 1], par[b - 1], lam + q * hs), sj) for q in (-2, -1, 0, 1, 2)}
            dh = (-hh[2] + 8.0 * hh[1] - 8.0 * hh[-1] + hh[-2]) / (12.0 * hs)
            km = z * np.eye(hh[0].shape[0]) - hh[0]
            ref += XC[s1 - 1] * XC[s2 - 1] * np.trace(np.linalg.solve(km, dh))
    pt = EP.epi_path(par[a - 1], par[b - 1], lam)
    return ref + 2.0 * np.sum(pt.dk)
