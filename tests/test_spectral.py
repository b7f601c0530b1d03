"""Bloch spectral function helpers and the projected chains (edc_green_proj) of the oracle, after the reference's
test/test_spectral.f90: (A) the k path, the unfolded Bloch sum (exact for a lattice Green function), the Fourier window,
the dressing weights; (B) readout on a random bcc binary: the projections are the same with the operator reduced by
D4h, D2h and the identity (the same Krylov process in three bases), the projection on the origin is g_11, and the cubic
rotation (x, y, z) -> (y, z, x) maps G_{px,px}(d) onto G_{pz,pz}(P d)."""
import numpy as np
import pytest

from asr_b200 import spectral as SP
from oracle.oracle import OracleOp
from tests.spectral_case import readout_inputs

Z = 0.35 + 0.08j


def test_kpath():
    kv, dist, ic = SP.spectral_kpath(np.array([[0, 1, 1], [0, 0, 0.5], [0, 0, 0]], float), 4)
    assert kv.shape[1] == 9 and list(ic) == [0, 4, 8]
    assert abs(dist[-1] - 1.5) < 1e-12 and np.max(np.abs(kv[:, -1] - [1, 0.5, 0])) < 1e-14


def test_unfolded_bloch_sum_is_exact_for_a_lattice_green_function():
    nper, z = 6, 0.13 + 0.07j
    ks = np.array([[jx, jy, jz] for jx in range(nper) for jy in range(nper) for jz in range(nper)], float).T / nper
    ek = -0.5 * np.sum(np.cos(2 * np.pi * ks), axis=0)
    r = np.array([[ix, iy, iz] for ix in range(nper) for iy in range(nper) for iz in range(nper)], float).T
    disp = r - nper * np.rint(r / nper)
    gR = np.exp(2j * np.pi * (ks.T @ disp)).T @ (1.0 / (z - ek)) / nper ** 3
    v = -np.imag(gR) / np.pi
    err = max(abs(SP.spectral_unfold(disp, v, ks[:, q]) + np.imag(1.0 / (z - ek[q])) / np.pi) for q in range(ks.shape[1]))
    assert err < 1e-12


def test_window():
    assert SP.spectral_window("ball", 0.0, 2.0) == 1.0 and SP.spectral_window("ball", 2.0, 2.0) == 0.0
    assert SP.spectral_window("ball", 2.5, 2.0) == 0.0 and abs(SP.spectral_window("ball", 1.0, 2.0) - 0.3125) < 1e-15
    assert SP.spectral_window("sharp", 2.0, 2.0) == 1.0 and SP.spectral_window("sharp", 2.01, 2.0) == 0.0
    rng = np.random.default_rng(3)
    for lat in ("fcc", "bcc"):
        wmin = {"ball": np.inf, "sharp": np.inf}
        i = np.arange(-8, 9)
        h = 0.5 * np.array(np.meshgrid(i, i, i, indexing="ij")).reshape(3, -1)
        hi = np.rint(2 * h).astype(int)
        on = (np.sum(hi, axis=0) % 2 == 0) if lat == "fcc" else ((hi[0] - hi[1]) % 2 == 0) & ((hi[1] - hi[2]) % 2 == 0)
        h = h[:, on]
        for rm in (1.0, 1.5, 2.0, 3.0):
            keep = np.linalg.norm(h, axis=0) <= rm + 1e-9
            rr = h[:, keep]
            for kind in wmin:
                ww = np.array([SP.spectral_window(kind, np.linalg.norm(rr[:, q]), rm) for q in range(rr.shape[1])])
                for _ in range(400):
                    k = 2 * rng.random(3) - 1
                    wmin[kind] = min(wmin[kind], SP.spectral_unfold(rr, ww, k) / ww.sum())
        assert wmin["ball"] > -1e-12 and wmin["sharp"] < -0.01


def test_dressing():
    dc = np.full(9, 0.04)
    dl = np.zeros((9, 2))
    dl[:, 0], dl[:, 1] = 0.04, 0.09
    tau = SP.spectral_dressing(dc, dl, [1, 2], [0.6, 0.4], True)
    assert np.all(tau[:, 0] == 1.0) and np.all(tau[:, 1] == 0.0)
    tau = SP.spectral_dressing(dc, dl, [2], [1.0], False)
    assert np.max(np.abs(tau[:, 0] - np.sqrt(0.04 / 0.09))) < 1e-14
    dl[:, 1] = 0.04
    tau = SP.spectral_dressing(dc, dl, [1, 2], [0.6, 0.4], False)
    assert np.max(np.abs(tau[:, 0] - 1.0)) + np.max(np.abs(tau[:, 1])) < 1e-14


@pytest.fixture(scope="module")
def readout():
    r = readout_inputs()
    ops = {}
    for key, (perm, dmat) in r["groups"].items():
        op = OracleOp(r["graph"], r["model"], r["cls"], perm, dmat, 1, 2, 1, r["flippable"], tsite=r["tsite"])
        ed = r["ed"]
        op.set_params(ed["c"], ed["d"], ed["o"], ed["e"])
        op.freeze_site(1, 1)
        ops[key] = op
    return r, ops


def test_target_links(readout):
    r, ops = readout
    assert len(r["tsite"]) == 15 and ops["d4h"].nop == 16 and ops["d2h"].nop == 8
    t0 = r["t0"]
    other = np.arange(15) != t0
    tn1 = ops["identity"].tnode
    assert np.all(tn1[:, other] > 0) and tn1[0, t0] > 0 and tn1[1, t0] == 0
    for key in ("d2h", "d4h"):
        assert np.all(ops[key].tnode[:, other] > 0) and ops[key].tnode[1, t0] == 0


@pytest.mark.parametrize("nlev,tol_abs,tol_origin", [(8, 1e-11, 1e-13), (24, None, 1e-9)])
def test_projections_in_three_bases(readout, nlev, tol_abs, tol_origin):
    r, ops = readout
    ed, tw, t0 = r["ed"], r["tw"], r["t0"]
    d4 = r["groups"]["d4h"][1]
    gp = {}
    e21 = e41 = e0 = 0.0
    for l0 in range(1, 10):
        out = {}
        for key in ("identity", "d2h", "d4h"):
            if key == "d4h" and not np.all(np.abs(np.abs(d4[l0 - 1, l0 - 1, :]) - 1.0) < 1e-9):
                continue
            op = ops[key]
            op.set_start(l0)
            g, p, p4, m = op.edc_green_proj(ed, Z, l0, nlev, op.tnode, op.tgop, tw, tail="none")
            assert m == nlev
            out[key] = (g, p)
        gp[l0] = out["d2h"][1]
        e21 = max(e21, np.max(np.abs(out["d2h"][1] - out["identity"][1])), abs(out["d2h"][0] - out["identity"][0]))
        e0 = max(e0, abs(out["d2h"][1][l0 - 1, t0] - out["d2h"][0]))
        if "d4h" in out:
            e41 = max(e41, np.max(np.abs(out["d4h"][1] - out["identity"][1])))
    gmax = max(np.max(np.abs(np.delete(gp[l0], t0, axis=1))) for l0 in gp)
    assert gmax > 1e-3
    if tol_abs is not None:
        assert e21 < tol_abs and e41 < tol_abs
    else:
        assert e21 / gmax < 1e-8 and e41 / gmax < 1e-8
    assert e0 < tol_origin
    if nlev == 8:   # cubic rotation P: (d1, d2, d3) -> (d2, d3, d1) maps p_x onto p_z
        td = r["tdisp"]
        erot = 0.0
        for t in range(td.shape[1]):
            pd = np.array([td[1, t], td[2, t], td[0, t]])
            tr = int(np.nonzero(np.all(np.abs(td - pd[:, None]) < 1e-9, axis=0))[0][0])
            erot = max(erot, abs(gp[4][3, t] - gp[3][2, tr]))
        assert erot < 1e-11


def test_structure_and_origin_classes():
    """The reference's checks of spectral_structure_ok and spectral_origin_classes: fcc one origin of weight 1; B2 and
    hcp accepted, hcp's two sites one origin (inversion, signs +1, -1); NiAs: the cations in two origins, the anions in
    one, weights 1/4, 1/4, 1/2; L1_2: four origins (corner and three faces) of weight 1/4; a sublattice that merges
    inequivalent sites is refused."""
    from asr_b200 import crystal as X
    s = X.prototype_structure("fcc")
    assert SP.spectral_structure_ok(s)
    bcl, ob, osg, ow = SP.spectral_origin_classes(s)
    assert list(ob) == [1] and abs(ow[0] - 1.0) < 1e-14
    assert SP.spectral_structure_ok(X.prototype_structure("b2"))
    s = X.prototype_structure("hcp")
    assert SP.spectral_structure_ok(s)
    bcl, ob, osg, ow = SP.spectral_origin_classes(s)
    assert len(ob) == 1 and list(osg) == [1, -1] and abs(ow[0] - 1.0) < 1e-14
    s = X.prototype_structure("nias", 1.62)
    assert SP.spectral_structure_ok(s)
    bcl, ob, osg, ow = SP.spectral_origin_classes(s)
    assert list(ob) == [1, 2, 3] and list(osg) == [1, 1, 1, -1] and np.max(np.abs(ow - [0.25, 0.25, 0.5])) < 1e-14
    l12 = X.Structure(np.eye(3), np.array([[0, 0.5, 0.5, 0], [0, 0.5, 0, 0.5], [0, 0, 0.5, 0.5]]), [1, 2, 2, 2])
    assert SP.spectral_structure_ok(l12)
    bcl, ob, osg, ow = SP.spectral_origin_classes(l12)
    assert len(ob) == 4 and np.max(np.abs(ow - 0.25)) < 1e-14
    bad = X.Structure(np.diag([1.0, 1.0, 2.0]), np.array([[0, 0, 0], [0, 0, 0], [0, 0.2, 0.5]]), [1, 1, 1])
    assert not SP.spectral_structure_ok(bad)


def test_unfolded_projections_give_the_band_structure():
    """An ordered bcc crystal on the 16-site periodic cell (one species, unreduced): the projected chains of the oracle
    (edc_green_proj, tail none, closed) give every off-site element <G_{0L,RL}>, and their Bloch sum at the commensurate
    wavevectors equals -Im tr_l (z - H(k))^-1 / pi of the dense H(k) (1e-9)."""
    from asr_b200 import lattices as lat
    from asr_b200 import synthetic as S
    case = S.cubic_case("bcc", 2, 1, [1.0], seed=5, group="identity")
    g, coord = case["graph"], case["coord"]
    n = g.n
    tsite = np.arange(1, n + 1, dtype=np.int32)
    fl = np.zeros(n, np.int32)
    op = OracleOp(g, case["model"], case["cls"], case["perm"], case["dmat"], 1, 6, 0, fl, tsite=tsite)
    assert op.nn == n
    ed = S.edc_params(S.draw_species(1, 5), 1)
    op.set_params(ed["c"], ed["d"], ed["o"], ed["e"])
    dim = 9 * n
    h = np.zeros((dim, dim))
    for k in range(dim):
        x = np.zeros(dim)
        x[k] = 1.0
        h[:, k] = op.apply(x)
    disp = 0.5 * ((coord + 2) % 4 - 2).astype(float)     # minimum-image displacements (alat)
    tw = np.zeros((9, 1, n))
    tw[:, 0, :] = 1.0
    z = 0.15 + 0.1j
    gdg = np.zeros((9, n), np.complex128)
    for l0 in range(1, 10):
        op.set_start(l0)
        _, gp, _, m = op.edc_green_proj(ed, z, l0, 200, op.tnode, op.tgop, tw, tail="none")
        gdg[l0 - 1] = gp[l0 - 1]
    ks = [np.array(v) / 2.0 for v in ((0, 0, 0), (1, 0, 0), (1, 1, 0), (1, 1, 1), (0, 0, 1))]
    orb_l = S.ORB_L
    site = op.tables()["site"]                          # the dense H is in node order; node j sits on site site[j]
    for k in ks:
        ph = np.exp(2j * np.pi * (k @ disp))
        hk = sum(ph[site[j] - 1] * h[0:9, 9 * j:9 * j + 9] for j in range(n))
        gk = np.linalg.inv(z * np.eye(9) - hk)
        for l in range(3):
            exact = -np.imag(np.trace(gk[np.ix_(orb_l == l, orb_l == l)])) / np.pi
            v = -np.imag(np.sum(gdg[orb_l == l], axis=0)) / np.pi
            unf = SP.spectral_unfold(disp, v, k)
            assert abs(unf - exact) < 1e-9 * max(1.0, abs(exact)), (k, l, unf, exact)


def test_multi_origin_sum_on_an_ordered_b2_crystal():
    """Two origin classes (the two sublattices of an ordered B2 crystal on the 16-site periodic cell, species with equal
    Delta and d and different c): the projected elements of each origin's operator, the partner average and the
    weighted Bloch sum equal (1/N) sum_ij cos(2 pi k.(r_j - r_i)) (-Im G_ij / pi) of the dense G at commensurate k."""
    from asr_b200 import lattices as lat
    from asr_b200 import synthetic as S
    sp = S.draw_species(2, 12)
    sp.d[1] = sp.d[0]
    sp.delta[1] = sp.delta[0]
    z = 0.1 + 0.12j
    gdg, tdisp, tbase, tsign, dense = [], [], [], [], None
    for u in (1, 2):
        case = S.example_case("cuzn_b2", u, l=2)
        g, coord, cls = case["graph"], case["coord"], case["cls"]
        n = g.n
        perm, dmat = lat.identity_group(n)
        op = OracleOp(g, case["model"], cls, perm, dmat, 1, 6, 0, np.zeros(n, np.int32), tsite=np.arange(1, n + 1, dtype=np.int32))
        ed = S.edc_params(sp, u)
        op.set_params(ed["c"], ed["d"], ed["o"], ed["e"])
        op.freeze_site(1, u)
        tw = np.zeros((9, 1, n))
        tw[:, 0, :] = 1.0
        gu = np.zeros((9, n, 1), np.complex128)
        for l0 in range(1, 10):
            op.set_start(l0)
            _, gp, _, _ = op.edc_green_proj(ed, z, l0, 200, op.tnode, op.tgop, tw, tail="none")
            gu[l0 - 1, :, 0] = gp[l0 - 1]
        gdg.append(gu)
        tdisp.append(0.5 * ((coord + 2) % 4 - 2).astype(float))
        tbase.append(np.asarray(cls) - 1)
        tsign.append(np.ones(n))
        if u == 1:                                        # the dense G of the whole cell, in site order
            dim = 9 * n
            h = np.zeros((dim, dim))
            for k in range(dim):
                x = np.zeros(dim)
                x[k] = 1.0
                h[:, k] = op.apply(x)
            site = op.tables()["site"] - 1
            pidx = np.concatenate([9 * np.argsort(site)[s_] + np.arange(9) for s_ in range(n)])
            gd = np.linalg.inv(z * np.eye(dim) - h)[np.ix_(pidx, pidx)]
            dense = (gd, 0.5 * coord.astype(float), n)
    ks = np.array([[0, 0, 0], [0.5, 0, 0], [0.5, 0.5, 0], [0.5, 0.5, 0.5]]).T
    A, parts, _ = SP.spectral_sum_origins(gdg, tdisp, tbase, tsign, [0.5, 0.5], ks, 2.0, "sharp")
    assert np.allclose(parts.sum(axis=0), A.sum(axis=2), rtol=0, atol=1e-13)
    gd, r, n = dense
    orb_l = S.ORB_L
    for q in range(ks.shape[1]):
        k = ks[:, q]
        c = np.cos(2 * np.pi * (k @ (r[:, None, :] - r[:, :, None]).reshape(3, -1))).reshape(n, n)
        for l in range(3):
            v = sum(-np.imag(gd[o::9, o::9]) / np.pi for o in np.nonzero(orb_l == l)[0])
            exact = float(np.sum(c * v)) / n
            assert abs(A[0, q, l] - exact) < 1e-9 * max(1.0, abs(exact)), (k, l, A[0, q, l], exact)


def test_targets_per_origin_class_and_their_partners():
    """Targets of every origin class (spectral_final, src/asr_class_scf.f90:1562-1601) for the ordered B2 cell (two
    classes, translations only) and hcp (one class, the second site by inversion): the origin comes first, every target
    lies within rmax, tbase / tsign follow the basis site, and every target of B2 finds its partner at -R in its own
    origin class's list (so the partner average of spectral_sum_origins never falls back)."""
    from asr_b200 import crystal as CR
    for name, ca, rmax, nor in (("b2", None, 1.01, 2), ("hcp", None, 1.5, 1)):
        s = CR.prototype_structure(name, ca)
        ops = CR.space_group(s)
        bclass, orig_b, orig_sign, orig_w = SP.spectral_origin_classes(s, ops)
        assert len(orig_b) == nor and abs(np.sum(orig_w) - 1.0) < 1e-12
        tg = []
        for u in range(nor):
            cg = CR.crystal_graph(s, ops, 1.0, 2, start=int(orig_b[u]) - 1, rmin=rmax)
            t = SP.spectral_targets(cg, bclass, orig_sign, rmax)
            assert t["t0"] == 0 and np.all(t["tdisp"][:, 0] == 0.0)
            assert np.all(np.linalg.norm(t["tdisp"], axis=0) <= rmax + 1e-9)
            assert np.array_equal(t["tbase"], bclass[cg.basis[t["tsite"] - 1]] - 1)
            assert t["tbase"][0] == u
            tg.append(t)
        if name == "b2":
            assert all(np.all(t["tsign"] == 1.0) for t in tg)
            for u in range(nor):
                for j in range(tg[u]["tsite"].shape[0]):
                    u2 = tg[u]["tbase"][j]
                    d = tg[u2]["tdisp"] + tg[u]["tsign"][j] * tg[u]["tdisp"][:, j:j + 1]
                    hit = (tg[u2]["tbase"] == u) & (np.max(np.abs(d), axis=0) < 1e-9)
                    assert hit.sum() == 1
            # NN shell of the other sublattice, NNN shell of the own one
            r = np.linalg.norm(tg[0]["tdisp"], axis=0)
            assert set(tg[0]["tbase"][np.abs(r - np.sqrt(0.75)) < 1e-9]) == {1}
            assert set(tg[0]["tbase"][np.abs(r - 1.0) < 1e-9]) == {0}
        else:
            assert sorted(set(tg[0]["tsign"])) == [-1.0, 1.0]
