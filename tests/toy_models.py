"""Toy models with exact answers (restating the fixtures of asr's test_slow/test_augcls.f90:69-205): a ring of sites with
three site classes whose configuration average is enumerated exhaustively and solved densely with numpy."""
import numpy as np

from asr_b200.lattices import Graph
from asr_b200.synthetic import ClassModel

ORB_L = np.array([0, 1, 1, 1, 2, 2, 2, 2, 2])


def ring_graph(n):
    nbr_ptr = 1 + 2 * np.arange(n + 1)
    nbr = np.zeros(2 * n, dtype=np.int32)
    for i in range(1, n + 1):
        nbr[2 * i - 2] = i % n + 1
        nbr[2 * i - 1] = (i - 2 + n) % n + 1
    return Graph(n=n, nbr_ptr=nbr_ptr.astype(np.int32), nbr=nbr)


def three_classes(seed=20261111):
    """Classes: 1 = ordered {1}, 2 = binary {2,3} (0.4, 0.6), 3 = ternary {1,3,4} (0.3, 0.5, 0.2); random ring blocks."""
    rng = np.random.default_rng(seed)
    nsc = np.array([1, 2, 3], dtype=np.int32)
    spc = np.zeros((3, 3), dtype=np.int32, order="F")
    conc = np.zeros((3, 3), order="F")
    spc[:1, 0] = [1]
    conc[:1, 0] = [1.0]
    spc[:2, 1] = [2, 3]
    conc[:2, 1] = [0.4, 0.6]
    spc[:3, 2] = [1, 3, 4]
    conc[:3, 2] = [0.3, 0.5, 0.2]
    b1 = 0.5 * (rng.uniform(size=(9, 9)) - 0.5)
    block = np.zeros((9, 9, 2, 1), order="F")
    block[:, :, 0, 0] = b1
    block[:, :, 1, 0] = b1.T
    b0 = 0.6 * (rng.uniform(size=(9, 9)) - 0.5)
    b0 = np.triu(b0) + np.triu(b0, 1).T
    block0 = np.asfortranarray(b0.reshape(9, 9, 1))
    return ClassModel(nsp=4, nsc=nsc, spc=spc, conc=conc, block=block, block0=block0)


def species_lmto(nsp=4, seed=5):
    """Per species and orbital: cm = C - E_nu, dl = Delta, om = o, en = E_nu  (each (9, nsp))."""
    rng = np.random.default_rng(seed)
    per_l = lambda lo, hi: np.asfortranarray(rng.uniform(lo, hi, size=(nsp, 3))[:, ORB_L].T)
    return dict(cm=per_l(-0.3, 0.3), dl=per_l(0.02, 0.09), om=per_l(-0.4, 0.4), en=per_l(-0.1, 0.1))


def edc_setup(sp, central):
    """src/asr_edc.f90:41-71 on already-alpha parameters: operator (c, d, o, e) and (dc, del, enu) for a central species."""
    dc = sp["dl"][:, central - 1].copy()
    c = np.asfortranarray(dc[:, None] / sp["dl"] * sp["cm"])
    d = np.asfortranarray(np.repeat(np.sqrt(dc)[:, None], sp["dl"].shape[1], axis=1))
    o = np.asfortranarray(sp["om"] * sp["dl"] / dc[:, None])
    e = np.zeros_like(c, order="F")
    return dict(c=c, d=d, o=o, e=e, dc=dc, dl=np.asfortranarray(sp["dl"]), enu=np.asfortranarray(sp["en"]))


def dense_g(model, graph, cfg, central, sp, z, l0):
    """[E - H(E)]^-1_{l0,l0} at site 1 for one configuration (test_slow/test_augcls.f90:149-192)."""
    n = graph.n
    nd = 9 * n
    s = np.zeros((nd, nd))
    for ii in range(n):
        s[9 * ii:9 * ii + 9, 9 * ii:9 * ii + 9] = model.block0[:, :, 0]
        for kk in range(graph.nbr_ptr[ii + 1] - graph.nbr_ptr[ii]):
            jj = graph.nbr[graph.nbr_ptr[ii] - 1 + kk] - 1
            s[9 * ii:9 * ii + 9, 9 * jj:9 * jj + 9] += model.block[:, :, kk, 0]
    sidx = np.repeat(np.asarray(cfg) - 1, 9)
    orb = np.tile(np.arange(9), n)
    dl = sp["dl"][orb, sidx]
    cm = sp["cm"][orb, sidx]
    en = sp["en"][orb, sidx]
    om = sp["om"][orb, sidx]
    dc = sp["dl"][orb, central - 1]
    hm = np.sqrt(dl)[:, None] * s * np.sqrt(dl)[None, :] + np.diag(cm)
    hoh = hm @ (om[:, None] * hm)
    tt = np.sqrt(dc / dl)
    ae = tt[:, None] * tt[None, :] * (np.diag(z - en) - hm + hoh)
    rhs = np.zeros(nd, complex)
    rhs[l0 - 1] = 1.0
    return np.linalg.solve(ae, rhs)[l0 - 1]


def exact_average(model, graph, rcls, central, sp, z, l0):
    """Configuration average of dense_g over every species pattern of sites 2..n (site 1 frozen to ``central``)."""
    n = graph.n
    sizes = [int(model.nsc[rcls[i] - 1]) for i in range(1, n)]
    tot = 0.0 + 0.0j
    psum = 0.0
    for idx in np.ndindex(*sizes):
        cfg = [central]
        pc = 1.0
        for i, k in enumerate(idx, start=1):
            kc = rcls[i] - 1
            cfg.append(int(model.spc[k, kc]))
            pc *= model.conc[k, kc]
        tot += pc * dense_g(model, graph, cfg, central, sp, z, l0)
        psum += pc
    return tot, psum
