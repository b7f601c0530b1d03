"""Writes tests/golden/c3_oracle_jacobian.json: the Jacobian of the band energy and the four sublattice charges of the
L2_1 adjoint configuration (tests/heusler_oracle.py) with respect to the 45 species parameters (c_l, d_l, Delta_l for
l = s, p, d and 5 species, row-major (parameter kind, species, l)), by central differences of the oracle with h = 1e-5
and with h / 2, with edc_setup's o = o_l D_s / D_c.  Test infrastructure; about an hour on 8 host cores:
    python tests/golden/make_c3_jacobian.py
"""
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from tests import heusler_oracle as HO  # noqa: E402

H = 1e-5


def main():
    cases, sp, ol, z, w = HO.configuration()
    orc = HO.OracleHeusler(cases)
    base = [sp.c.copy(), sp.d.copy(), sp.delta.copy()]

    def f(vals):
        e, q = orc.energy_and_charges(*vals, ol, z, w)
        return np.concatenate([[e], q])
    t0 = time.time()
    f0 = f(base)
    jac_h = np.zeros((5, 45))
    jac_h2 = np.zeros((5, 45))
    for k in range(45):
        a, idx = divmod(k, 15)
        out = {}
        for h in (H, -H, H / 2, -H / 2):
            v = [x.copy() for x in base]
            v[a].ravel()[idx] += h
            out[h] = f(v)
        jac_h[:, k] = (out[H] - out[-H]) / (2 * H)
        jac_h2[:, k] = (out[H / 2] - out[-H / 2]) / H
        print(f"parameter {k + 1}/45 {time.time() - t0:.0f} s", flush=True)
    rich = (4 * jac_h2 - jac_h) / 3
    doc = {"configuration": "L2_1 bcc 4^3 cell, heusler_case(4, 3, k), 5 species and o_l from seed 3, depth 20, 32-point "
                            "contour on [-1.2, 0.2], hull tail, edc_setup's o",
           "outputs": ["band energy", "charge 1", "charge 2", "charge 3", "charge 4"],
           "parameters": "45 = (c, d, Delta) x 5 species x (s, p, d), row-major",
           "h": H, "values": f0.tolist(), "central_h": jac_h.tolist(), "central_h_over_2": jac_h2.tolist(),
           "richardson": rich.tolist()}
    with open(os.path.join(ROOT, "tests", "golden", "c3_oracle_jacobian.json"), "w") as fh:
        json.dump(doc, fh)


if __name__ == "__main__":
    main()
