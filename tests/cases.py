"""Shared small operator cases for the parity tests (seeded synthetic inputs)."""
import numpy as np

from asr_b200 import synthetic as S
from tests import toy_models as T


def cubic(kind="bcc", l=3, nsp=2, conc=(0.5, 0.5), seed=0, group="d2h", maxlevel=2, maxrank=0, start_flippable=False):
    case = S.cubic_case(kind, l, nsp, list(conc), seed=seed, group=group)
    fl = np.ones(case["graph"].n, np.int32)
    if not start_flippable:
        fl[0] = 0
    case.update(maxlevel=maxlevel, maxrank=maxrank, flippable=fl)
    return case


def ring():
    g = T.ring_graph(4)
    mdl = T.three_classes()
    return dict(graph=g, model=mdl, cls=np.array([1, 2, 3, 2], np.int32),
                perm=np.asfortranarray(np.arange(1, 5, dtype=np.int32).reshape(4, 1)),
                dmat=np.asfortranarray(np.eye(9).reshape(9, 9, 1)), maxlevel=80, maxrank=0,
                flippable=np.array([0, 1, 1, 1], np.int32))


def build_both(case, build_gpu, build_oracle):
    args = (case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, case["maxlevel"])
    gop = build_gpu(*args, maxrank=case["maxrank"], flippable=case["flippable"])
    oop = build_oracle(*args, case["maxrank"], case["flippable"])
    return gop, oop


def general_params(nsp, seed=3, o_scale=0.3, e_scale=0.1):
    """A general operator: species-dependent c, d, o, e (exercises every term of H = E_nu + h - h o h)."""
    rng = np.random.default_rng(seed)
    per = lambda lo, hi: np.asfortranarray(rng.uniform(lo, hi, size=(nsp, 3))[:, S.ORB_L].T)
    return per(-0.6, 0.2), per(0.05, 0.4), per(-o_scale, o_scale), per(-e_scale, e_scale)
