"""The committed oracle Jacobian of the L2_1 adjoint configuration (tests/golden/c3_oracle_jacobian.json) is the oracle's:
its output values and one central difference, recomputed now."""
import json
import os

import numpy as np

from tests import heusler_oracle as HO


def test_fixture_matches_the_oracle():
    fx = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c3_oracle_jacobian.json")))
    cases, sp, ol, z, w = HO.configuration()
    orc = HO.OracleHeusler(cases)
    base = [sp.c.copy(), sp.d.copy(), sp.delta.copy()]
    e, q = orc.energy_and_charges(*base, ol, z, w)
    assert np.allclose(np.concatenate([[e], q]), fx["values"], rtol=1e-12, atol=0)
    k = 40                                   # Delta_p of species 4 (the disordered sublattice)
    a, idx = divmod(k, 15)
    out = []
    for h in (fx["h"], -fx["h"]):
        v = [x.copy() for x in base]
        v[a].ravel()[idx] += h
        ev, qv = orc.energy_and_charges(*v, ol, z, w)
        out.append(np.concatenate([[ev], qv]))
    col = (out[0] - out[1]) / (2 * fx["h"])
    assert np.allclose(col, np.array(fx["central_h"])[:, k], rtol=1e-9, atol=1e-12)
