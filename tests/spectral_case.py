"""Inputs of the spectral readout checks: a random bcc binary A0.6B0.4 on the periodic 8^3 half-lattice cell (lsup 4),
one class, levels 2, rank 1, the start site frozen to species 1; the operator reduced by D4h (16), D2h (8) and the
identity; targets: the origin and the first two bcc shells (15 sites)."""
import numpy as np

from asr_b200 import lattices as lat
from asr_b200 import spectral as SP
from asr_b200 import synthetic as S

LSUP = 4
CONC = (0.6, 0.4)


def readout_inputs(seed: int = 0):
    case = S.cubic_case("bcc", LSUP, 2, list(CONC), seed=seed, group="d4h")
    coord, g = case["coord"], case["graph"]
    cls = case["cls"]
    p4, m4 = lat.class_ops(coord, 2 * LSUP, cls)
    p2, m2 = lat.d2h_ops(coord, 2 * LSUP, cls)
    p1, d1 = lat.identity_group(g.n)
    groups = {"d4h": (np.asfortranarray(p4, dtype=np.int32), np.asfortranarray(lat.orbital_rep(m4))),
              "d2h": (np.asfortranarray(p2, dtype=np.int32), np.asfortranarray(lat.orbital_rep(m2))),
              "identity": (np.asfortranarray(p1, dtype=np.int32), np.asfortranarray(d1))}
    h = (coord + LSUP) % (2 * LSUP) - LSUP
    sel = np.nonzero(np.sum(h * h, axis=0) <= 4)[0]
    tsite = (sel + 1).astype(np.int32)
    tdisp = 0.5 * h[:, sel].astype(float)
    t0 = int(np.nonzero(tsite == 1)[0][0])
    fl = np.ones(g.n, np.int32)
    fl[0] = 0
    ed = S.edc_params(S.draw_species(2, 11 + seed), 1)
    tw = np.zeros((9, 2, len(tsite)))
    for t in range(len(tsite)):
        tw[:, :, t] = SP.spectral_dressing(ed["dc"], ed["dl"], [1, 2], CONC, tsite[t] == 1)
    return dict(graph=g, model=case["model"], cls=cls, groups=groups, tsite=tsite, tdisp=tdisp, t0=t0, flippable=fl, ed=ed,
                tw=tw)
