"""EPI block chains on the device (asr_epi_blocks, epi_blocks of src/asr_epi.f90:639-663) against the oracle's
restatement and against the exact configuration average of Tr[G dH/dlambda] on the 16-site cell of the reference's
test/test_epi.f90 part (D); the thermodynamic integration of the pair table against the same integral of the exact
traces."""
import numpy as np
import pytest

from asr_b200 import augcls as A
from asr_b200 import contour as CT
from asr_b200 import epi as EP
from asr_b200 import lattices as lat
from oracle.oracle import OracleOp
from tests import epi_case as E

pytestmark = pytest.mark.gpu

LAM = 0.35
ZS = np.array([0.12 + 0.3j, -0.3 + 0.05j, 0.5 + 0.02j])


def _ops(group):
    c = E.cell()
    mdl, cls, fl = E.chain_model(c)
    if group == "pair":
        perm, mats = EP.epi_pair_ops(c["coord"], E.MG, cls)
        d = lat.orbital_rep(mats)
    else:
        perm, d = lat.identity_group(c["graph"].n)
    args = (c["graph"], mdl, cls, perm, d, 1, 8)
    return c, A.build_augcls_operator(*args, maxrank=2, flippable=fl), OracleOp(*args, 2, fl), d


@pytest.mark.parametrize("group,tail,nlev", [("pair", "none", 100), ("pair", "hull", 12), ("identity", "avg2", 16)])
def test_device_blocks_match_the_oracle(group, tail, nlev):
    c, dop, oop, d = _ops(group)
    par = E.species()
    pt = EP.epi_path(par[0], par[2], LAM)
    params, ed = EP.epi_setup(par, pt)
    vec, chi, lo = EP.epi_adapted(d)
    for op in (dop, oop):
        op.set_params(*params)
        op.freeze_any(1, 4)
        op.freeze_any(c["jp"], 2)
    x, m = EP.epi_blocks(dop, params, ed, vec, chi, lo, ZS, nlev, tail)
    worst = 0.0
    for ia in range(9):
        oop.set_chi(chi[: oop.nop, ia])
        for j, z in enumerate(ZS):
            xo, mo = oop.epi_blocks(ed, vec[:, ia], z, nlev, tail=tail)
            assert tuple(m[:, j, ia]) == mo
            worst = max(worst, np.max(np.abs(x[:, j, ia] - xo)) / np.max(np.abs(xo[:3])))
    assert worst < 1e-10, worst


@pytest.mark.parametrize("group", ["pair", "identity"])
def test_device_trace_equals_the_exact_configuration_average(group):
    c, dop, _, d = _ops(group)
    par = E.species()
    for sj in (2, 3):
        dop.unfreeze()
        dop.freeze_any(1, 4)
        dop.freeze_any(c["jp"], sj)
        tr, mism = EP.trace_at(dop, par, 1, 2, LAM, d, ZS[:1], 100, tail="none")
        ref = E.exact_trace(c, par, 1, 2, LAM, sj, ZS[0])
        assert abs(tr[0] - ref) / abs(ref) < 1e-8, (sj, tr[0], ref)
        assert mism < 1e-8


def test_fp32_blocks_close_to_fp64():
    c, dop, _, d = _ops("pair")
    par = E.species()
    pt = EP.epi_path(par[0], par[1], LAM)
    params, ed = EP.epi_setup(par, pt)
    vec, chi, lo = EP.epi_adapted(d)
    dop.set_params(*params)
    dop.freeze_any(1, 4)
    dop.freeze_any(c["jp"], 3)
    x64, _ = EP.epi_blocks(dop, params, ed, vec, chi, lo, ZS, 16, "hull", "fp64")
    x32, _ = EP.epi_blocks(dop, params, ed, vec, chi, lo, ZS, 16, "hull", "fp32")
    assert np.max(np.abs(x32[:3] - x64[:3])) < 1e-4 * np.max(np.abs(x64[:3]))


def test_pair_table_against_the_exact_integral():
    """U(c, s) for c in {1, 2, 3} on the path from species 1 and s in {1, 2, 3} on the partner: 2 Gauss-Legendre nodes in
    lambda and a 12-point contour, from the device chains and from the exact traces at the same nodes."""
    c, dop, _, d = _ops("pair")
    par = E.species()
    z, w = CT.contour_nodes(-1.6, 0.2, 12)

    def op_for(s):
        dop.unfreeze()
        dop.freeze_any(1, 4)
        dop.freeze_any(c["jp"], s)
        return dop
    u = EP.pair_table(op_for, par, [1, 2, 3], [1, 2, 3], d, z, w, 2, 100, tail="none")
    xg, wg = np.polynomial.legendre.leggauss(2)
    lam, wl = 0.5 * (xg + 1.0), 0.5 * wg
    dom = np.zeros((3, 3))
    for js, s in enumerate((1, 2, 3)):
        for ic, cc in enumerate((2, 3), start=1):
            for lq, wq in zip(lam, wl):
                tr = np.array([E.exact_trace(c, par, 1, cc, float(lq), s, zz) for zz in z])
                dom[ic, js] += wq * (-np.imag(np.sum(w * tr)) / np.pi)
    uex = dom - dom[:, :1]
    assert np.max(np.abs(uex)) > 1e-5
    # the exact side differentiates the dense H by a five-point difference of step 1e-2 (error ~1e-8 of U), so the
    # comparison is at 1e-7 of the largest entry
    assert np.max(np.abs(u - uex)) < 1e-7 * np.max(np.abs(uex)), (u, uex)
    assert np.all(u[0] == 0.0) and np.all(u[:, 0] == 0.0)
