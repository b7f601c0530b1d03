"""A bcc binary class with a third species outside it (the shape of a path species in an EPI set-up): freeze cases."""
import numpy as np

from asr_b200 import synthetic as S
from tests import cases as K


def three_species_case():
    """bcc 3^3 periodic cluster, D4h, one class of species {1, 2} at 0.5 / 0.5 and nsp = 3; the start site is not
    flippable."""
    case = K.cubic("bcc", 3, 2, (0.5, 0.5), group="d4h", maxlevel=2, maxrank=1)
    m = case["model"]
    case["model"] = S.ClassModel(nsp=3, nsc=m.nsc, spc=m.spc, conc=m.conc, block=m.block, block0=m.block0)
    return case


def params3(seed=5):
    rng = np.random.default_rng(seed)
    per = lambda lo, hi: np.asfortranarray(rng.uniform(lo, hi, size=(3, 3))[:, S.ORB_L].T)
    return per(-0.6, 0.2), per(0.05, 0.4), per(-0.2, 0.2), per(-0.1, 0.1)
