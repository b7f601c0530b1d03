"""The L2_1 four-sublattice adjoint configuration evaluated by the oracle: band energy and sublattice charges from the
oracle's chain_greens (src/asr_class_scf.f90:966-1160) and the contour moments of ed_moments (:797-877), the same
quantities as asr_b200.classes.SublatticeChains.energy_and_charges.  Test infrastructure."""
import numpy as np

from asr_b200 import autograd as AG
from asr_b200 import contour as CT
from asr_b200 import synthetic as S

NLEV = 20
SEED = 3


def configuration():
    """(cases, species parameters, o_l, contour z, w) of the configuration: heusler_case(4, 3, k) for the four
    sublattices, 5 species from seed 3, o_l from seed 3, a 32-point contour on [-1.2, 0.2]."""
    cases = [S.heusler_case(4, SEED, k) for k in (1, 2, 3, 4)]
    sp = S.draw_species(5, SEED)
    ol = S.draw_o(5, SEED)
    z, w = CT.contour_nodes(-1.2, 0.2, 32)
    return cases, sp, ol, z, w


class OracleHeusler:
    def __init__(self, cases, nthreads=0):
        from oracle.oracle import OracleOp
        self.ops, self.comps, self.orbits = [], [], []
        for c in cases:
            self.ops.append(OracleOp(c["graph"], c["model"], c["cls"], c["perm"], c["dmat"], 1, c["maxlevel"], c["maxrank"],
                                     c["flippable"]))
            mdl, k = c["model"], int(c["cls"][0]) - 1
            self.comps.append([(int(mdl.spc[j, k]), float(mdl.conc[j, k])) for j in range(int(mdl.nsc[k]))])
            self.orbits.append(AG.orbital_orbits(c["dmat"]))
        self.nthreads = nthreads

    def energy_and_charges(self, c, d, delta, ol, z, w, enu=None):
        """(band energy, charges (4,)) at the species parameters c, d, delta, o_l (5, 3 each)."""
        enu = np.zeros((5, 3)) if enu is None else enu
        spp = S.SpeciesParams(c=c, d=d, delta=delta, enu=enu)
        e_band, q = 0.0, []
        for kap, oop in enumerate(self.ops):
            comps = [s for s, _ in self.comps[kap]]
            conc = dict(self.comps[kap])
            orbs = [o[0] + 1 for o in self.orbits[kap]]
            wts = [len(o) for o in self.orbits[kap]]
            eds = [S.edc_params_o(spp, ol, s) for s in comps]
            groups = [dict(c=ed["c"], d=ed["d"], o=ed["o"], e=ed["e"], dc=ed["dc"], dl=ed["dl"], enu=ed["enu"]) for ed in eds]
            gz, _ = oop.chain_greens(groups, comps, orbs, np.full((len(comps), len(orbs)), NLEV, np.int32), z, 4,
                                     nthreads=self.nthreads)
            qk = 0.0
            for ci, s in enumerate(comps):
                for oi, orb in enumerate(orbs):
                    g = gz[:, oi, ci]
                    en = enu[s - 1, S.ORB_L[orb - 1]]
                    m0 = -np.imag(np.sum(w * g)) / np.pi
                    m1 = -np.imag(np.sum(w * (z - en) * g)) / np.pi
                    qk += conc[s] * wts[oi] * m0
                    e_band += conc[s] * wts[oi] * (m1 + en * m0)
            q.append(qk)
        return e_band, np.array(q)
