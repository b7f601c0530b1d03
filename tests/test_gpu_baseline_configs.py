"""Parity at the sizes of the benchmark configurations, through the C-ABI against the oracle.

* Batched uneven-depth configuration (fcc ternary, 5^3-cell cluster, levels 3, rank 1, D2h: 20,969 nodes; 54 chain
  groups at depths 16-28): all 54 groups over 192 energies (the 48 contour nodes and 144 real energies spread over the
  whole 4096-point real axis) run in depth-sorted batches of 16 tiles x 4 nodes per warp with the step kernel's
  fixed-offset link gathers (the shape and kernel the autotuner keeps for this operator on a B200).  The oracle
  (``chain_greens`` / ``edc_green_blk``, src/asr_class_scf.f90:966-1160, src/asr_edc.f90:237-316) evaluates a sample of
  8 energies per group that touches every 32-lane tile of the run: 2 contour nodes and 6 real energies from the band
  bottom to the top.  FP64: a and b within 1e-9 relative, G within 1e-8, equal depths.  FP32 vectors and matvec with
  FP64 coefficients and fractions: DOS within 1e-6 of the oracle's on the sample and of the FP64 device DOS at all 4096
  real energies for every group, both relative to the largest DOS on the real axis.
* Plain configuration (bcc A0.5B0.5, levels 4, D2h, 9 real chains of depth 12, Beer-Pettifor tail, 2000 energies): the
  DOS of every start orbital against the oracle's lanczos + terminated fraction (src/reference/asr_recursion.f90:17-58,
  src/reference/asr_terminator.f90) within 1e-8.
"""
import numpy as np
import pytest

import asr_b200 as A
from asr_b200 import synthetic as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

NZ = 192
CONTOUR_SAMPLE = (5, 37)                      # tiles 0 and 1 of a group
REAL_SAMPLE = (4, 29, 62, 93, 122, 141)       # of the 144 real energies: tiles 1, 2, 3, 4, 5, 5


@pytest.fixture(scope="module")
def batched():
    case, fl, groups, z_all = S.batched_ternary_workload()
    zr = z_all[48:]
    ridx = np.round(np.arange(144) * (zr.shape[0] - 1) / 143).astype(int)
    z = np.concatenate([z_all[:48], zr[ridx]])
    sel = list(CONTOUR_SAMPLE) + [48 + r for r in REAL_SAMPLE]
    op = A.build_augcls_operator(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, 3, maxrank=1,
                                 flippable=fl)
    specs = [A.ChainSpec(c=g["ed"]["c"], d=g["ed"]["d"], o=g["ed"]["o"], e=g["ed"]["e"], pa=g["ed"]["pa"], pb=g["ed"]["pb"],
                         frozen_sp=g["cen"], start_orb=g["l0"], nlev=g["nlev"]) for g in groups]
    # the oracle on the sample: one block chain per (spin, central species, start orbital) over the 8 sampled energies
    oop = O.OracleOp(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, 3, 1, fl)
    gps, gcomp, nlevq = [], [], []
    for spin in range(2):
        for cen in (1, 2, 3):
            gq = [g for g in groups if g["spin"] == spin and g["cen"] == cen]
            ed = gq[0]["ed"]
            gps.append(dict(c=ed["c"], d=ed["d"], o=ed["o"], e=ed["e"], dc=ed["dc"], dl=ed["dl"], enu=ed["enu"]))
            gcomp.append(cen)
            nlevq.append([g["nlev"] for g in gq])
    gz, _, cf = oop.chain_greens(gps, gcomp, list(range(1, 10)), np.array(nlevq, np.int32), z[sel], len(sel), coefs=True)
    # oracle arrays (nz, norb, ngroup) -> (nz, 54) in the device's group order (spin, central species, start orbital)
    go = gz.reshape(len(sel), 54, order="F")
    ao = cf["a"].reshape(cf["a"].shape[0], len(sel), 54, order="F")
    bo = cf["b"].reshape(cf["b"].shape[0], len(sel), 54, order="F")
    mo = cf["m"].reshape(len(sel), 54, order="F")
    return dict(op=op, specs=specs, groups=groups, z=z, sel=sel, go=go, ao=ao, bo=bo, mo=mo, real=slice(48, NZ))


def test_batched_workload_fp64_matches_oracle(batched):
    op, specs = batched["op"], batched["specs"]
    assert op.nn == 20969 and len(specs) == 54
    A.set_tuning(op, "fp64", 16, 4, "fixed-offset")
    try:
        r = A.chains_run(op, specs, batched["z"], "edc", 0.0, "hull", "fp64", coefs=True)
    finally:
        A.set_tuning(op, "fp64", 0, 0, "general")
    sel = batched["sel"]
    g, m, a, b = r["g"][sel], r["m"][sel], r["a"][:, sel], r["b"][:, sel]
    assert np.array_equal(m, batched["mo"])
    ao, bo = batched["ao"], batched["bo"]
    for q in range(54):
        for j in range(len(sel)):
            mj = int(m[j, q])
            assert mj == specs[q].nlev
            ea = np.max(np.abs(a[:mj, j, q] - ao[:mj, j, q]) / np.abs(ao[:mj, j, q]))
            eb = np.max(np.abs(b[:mj - 1, j, q] - bo[:mj - 1, j, q]) / np.abs(bo[:mj - 1, j, q]))
            assert ea < 1e-9 and eb < 1e-9, (q, j, ea, eb)
    err = np.max(np.abs(g - batched["go"]) / np.abs(batched["go"]))
    assert err < 1e-8, err


def test_batched_workload_fp32_dos_within_1e6(batched):
    """DOS errors relative to the largest DOS on the real axis (all 54 groups, all 4096 real energies of the FP64 device
    run, which the FP64 test pins to the oracle): the FP32 form against the oracle on the sampled energies, and against
    the FP64 device run at every real energy."""
    op, specs, sel = batched["op"], batched["specs"], batched["sel"]
    _, _, _, z_all = S.batched_ternary_workload()
    zr = z_all[48:]
    g64 = A.chains_run(op, specs, zr, "edc", 0.0, "hull", "fp64")["g"]
    g32 = A.chains_run(op, specs, zr, "edc", 0.0, "hull", "fp32")["g"]
    d64, d32 = -g64.imag / np.pi, -g32.imag / np.pi
    dmax = np.max(np.abs(d64))
    err_band = np.max(np.abs(d32 - d64)) / dmax
    assert err_band <= 1e-6, err_band
    g32s = A.chains_run(op, specs, batched["z"], "edc", 0.0, "hull", "fp32")["g"]
    nr = len(CONTOUR_SAMPLE)
    dos32, doso = -g32s[sel[nr:]].imag / np.pi, -batched["go"][nr:].imag / np.pi
    err_oracle = np.max(np.abs(dos32 - doso)) / dmax
    assert err_oracle <= 1e-6, err_oracle


def test_plain_configuration_dos_matches_oracle():
    case = S.cubic_case("bcc", 4, 2, [0.5, 0.5], seed=0, group="d2h")
    fl = np.ones(case["graph"].n, np.int32)
    op = A.build_augcls_operator(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, 4, maxrank=1,
                                 flippable=fl)
    c, d, o, e = S.plain_params(S.draw_species(2, 0))
    specs = [A.ChainSpec(c=c, d=d, o=o, e=e, start_orb=l0, nlev=12) for l0 in range(1, 10)]
    z = np.linspace(-1.5, 1.0, 2000) + 0.005j
    g = A.chains_run(op, specs, z, mode="plain", tail="bp")["g"]
    oop = O.OracleOp(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, 4, 1, fl)
    oop.set_params(c, d, o, e)
    assert op.nn == oop.nn
    for l0 in range(1, 10):
        oop.set_start(l0)
        v0 = np.zeros(oop.dim)
        v0[l0 - 1] = 1.0
        ao, bo, no = oop.lanczos(v0, 12)
        go, _ = O.terminated_green(ao, bo, no, z, "beer-pettifor")
        err = np.max(np.abs(g[:, l0 - 1].imag - go.imag)) / np.pi
        assert err < 1e-8, (l0, err)
