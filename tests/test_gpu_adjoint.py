"""Device adjoint of the edc chains against central finite differences (h = 1e-5), of the CUDA forward and of the
oracle's forward, and the torch.autograd binding."""
import numpy as np
import pytest

from asr_b200 import augcls as A
from asr_b200 import chains as CH
from asr_b200 import synthetic as S
from asr_b200 import autograd as AG
from tests import cases as K

pytestmark = pytest.mark.gpu

H = 1e-5
KINDS = {"c": 0, "e": 0, "pb": 0, "d": 1, "pa": 2}


def _setup(seed=0, nsp=2, group="d4h"):
    case = K.cubic("bcc", 3, nsp, (0.5, 0.5) if nsp == 2 else (0.66, 0.14, 0.2), group=group, maxlevel=3, maxrank=1)
    args = (case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, case["maxlevel"])
    op = A.build_augcls_operator(*args, maxrank=case["maxrank"], flippable=case["flippable"])
    sp = S.draw_species(nsp, seed)
    specs = []
    for q, (central, orb, nlev) in enumerate([(1, 1, 12), (2, 5, 9), (1, 3, 14)]):
        ed = S.edc_params(sp, central)
        e = np.asfortranarray(0.05 * np.cos(np.arange(nsp)[None, :] + 0.3 * q) * np.ones((9, 1)))
        d = ed["d"].copy(order="F")
        if q == 2:   # species-dependent d: the general (unfolded) S path
            d = np.asfortranarray(d * (1.0 + 0.2 * np.arange(nsp))[None, :])
        specs.append(CH.ChainSpec(c=ed["c"], d=d, o=ed["o"], e=e, pa=ed["pa"], pb=ed["pb"], frozen_sp=central if q < 2 else 0,
                                  start_orb=orb, nlev=nlev))
    return op, specs, AG.orbital_orbits(case["dmat"])


def _central(f, h=H):
    """Central difference with step h, Richardson-extrapolated with step h/2 (truncation error O(h^4))."""
    d1 = (f(h) - f(-h)) / (2 * h)
    d2 = (f(h / 2) - f(-h / 2)) / h
    return (4 * d2 - d1) / 3


def _loss(op, specs, z, w, tail, project):
    g = CH.chains_run(op, specs, z, "edc", 0.0, tail, "fp64", project)["g"]
    return np.sum(w * g)


def _perturbed(specs, q, kind, orbit, s, h):
    out = []
    for p, sp in enumerate(specs):
        vals = {k: getattr(sp, k).copy(order="F") for k in ("c", "d", "o", "e", "pa", "pb")}
        if p == q:
            vals[kind][orbit, s] += h
        out.append(CH.ChainSpec(**vals, frozen_sp=sp.frozen_sp, start_orb=sp.start_orb, nlev=sp.nlev))
    return out


@pytest.mark.parametrize("tail,project", [("hull", True), ("avg2", False), ("none", True)])
def test_adjoint_matches_central_differences(tail, project):
    """Every (kind, orbit, species) direction of every group: the derivative along a group-invariant direction is the
    sum of the per-orbital entries over the orbit."""
    op, specs, orbits = _setup()
    z = np.linspace(-0.5, 0.3, 6) + 0.1j
    rng = np.random.default_rng(5)
    w = rng.standard_normal((6, 3)) + 1j * rng.standard_normal((6, 3))
    g, grad = CH.chains_adjoint(op, specs, z, w, tail, "fp64", project)
    g_fwd = CH.chains_run(op, specs, z, "edc", 0.0, tail, "fp64", project)["g"]
    assert np.max(np.abs(g - g_fwd) / np.abs(g_fwd)) < 1e-12
    worst, where = 0.0, None
    for q in range(3):
        scale = np.max(np.abs(grad[q]))
        for kind in ("c", "d", "pa", "e", "pb"):
            for orbit in orbits:
                s = int(rng.integers(2))
                fd = _central(lambda h: _loss(op, _perturbed(specs, q, kind, orbit, s, h), z, w, tail, project))
                adj = np.sum(grad[q, KINDS[kind], s, orbit])
                err = abs(adj - fd) / max(abs(fd), 1e-2 * scale)
                if err > worst:
                    worst, where = err, (q, kind, orbit, s, adj, fd)
    assert worst < 1e-6, (worst, where)


def test_adjoint_is_independent_of_the_checkpoint_stride():
    op, specs, _ = _setup(seed=2)
    z = np.linspace(-0.4, 0.2, 5) + 0.06j
    w = np.ones((5, 3), complex)
    ref = CH.chains_adjoint(op, specs, z, w, "hull", "fp64", True, stride=1)[1]
    for stride in (2, 5, 0, 40):
        gr = CH.chains_adjoint(op, specs, z, w, "hull", "fp64", True, stride=stride)[1]
        assert np.array_equal(gr, ref), stride


def test_adjoint_fp32_matvec_close_to_fp64():
    op, specs, _ = _setup(seed=1)
    z = np.linspace(-0.4, 0.2, 4) + 0.1j
    w = np.ones((4, 3), complex)
    g64 = CH.chains_adjoint(op, specs, z, w, "hull", "fp64", True)[1]
    g32 = CH.chains_adjoint(op, specs, z, w, "hull", "fp32", True)[1]
    assert np.max(np.abs(g32 - g64)) < 1e-3 * np.max(np.abs(g64))


def test_adjoint_against_oracle_differences():
    """The same gradient from central differences of the oracle's edc_green_blk (the CPU restatement)."""
    from oracle.oracle import OracleOp
    case = K.cubic("bcc", 3, 2, (0.5, 0.5), group="d4h", maxlevel=3, maxrank=1)
    args = (case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, case["maxlevel"])
    op = A.build_augcls_operator(*args, maxrank=case["maxrank"], flippable=case["flippable"])
    oop = OracleOp(*args, case["maxrank"], case["flippable"])
    ed = S.edc_params(S.draw_species(2, 3), 2)
    z = np.linspace(-0.45, 0.25, 5) + 0.1j
    nlev, iv = 10, 3
    spec = CH.ChainSpec(c=ed["c"], d=ed["d"], o=ed["o"], e=ed["e"], pa=ed["pa"], pb=ed["pb"], frozen_sp=2, start_orb=iv, nlev=nlev)
    w = np.linspace(1.0, 2.0, 5).astype(complex).reshape(5, 1)
    _, grad = CH.chains_adjoint(op, [spec], z, w, "hull", "fp64", True)

    oop.set_start(iv)
    orbits = AG.orbital_orbits(case["dmat"])

    def oracle_loss(c, d):
        oop.set_params(c, d, ed["o"], ed["e"])
        oop.unfreeze()
        oop.freeze_site(1, 2)
        g = oop.edc_green_blk(ed, z, iv, nlev, depth_tol=0.0, tail="hull")[0]
        return np.sum(w[:, 0] * g)

    for kind, l, s in [("c", 0, 0), ("c", 4, 1), ("c", 2, 1), ("d", 4, 0), ("d", 7, 1), ("d", 1, 1)]:
        orbit = next(o for o in orbits if l in o)
        vals = {"c": ed["c"].copy(order="F"), "d": ed["d"].copy(order="F")}
        vp = {k: v.copy(order="F") for k, v in vals.items()}
        vm = {k: v.copy(order="F") for k, v in vals.items()}
        vp[kind][orbit, s] += H
        vm[kind][orbit, s] -= H
        fd = (oracle_loss(vp["c"], vp["d"]) - oracle_loss(vm["c"], vm["d"])) / (2 * H)
        adj = np.sum(grad[0, KINDS[kind], s, orbit])
        assert abs(adj - fd) <= 1e-6 * max(abs(fd), 1e-2 * np.max(np.abs(grad))), (kind, l, s, adj, fd)


def test_torch_autograd_band_energy_and_charge():
    """d(band energy, charge)/d(c_l, d_l, Delta_l) through ChainGreens against central differences."""
    import torch
    from asr_b200 import contour as CT
    op, _, _ = _setup(seed=4)
    nsp = 2
    rng = np.random.default_rng(11)
    cl = torch.tensor(rng.uniform(-0.6, 0.2, (nsp, 3)), dtype=torch.float64, requires_grad=True)
    dl = torch.tensor(rng.uniform(0.05, 0.4, (nsp, 3)), dtype=torch.float64, requires_grad=True)
    Dl = torch.tensor(rng.uniform(0.5, 1.5, (nsp, 3)), dtype=torch.float64, requires_grad=True)
    enu = torch.zeros(nsp, 3, dtype=torch.float64)
    z, wq = CT.contour_nodes(-1.0, 0.1, 12)
    conc = [0.5, 0.5]

    def energy_charge(cl, dl, Dl):
        e_band = 0.0
        q = 0.0
        for central in (1, 2):
            arrs = AG.edc_group_arrays(cl, dl, Dl, enu, central)
            groups = [(central, o, 10) for o in (1, 3, 7)]   # s, p_z, d_3z2-r2: one-dimensional under D4h
            stk = [a[None].expand(len(groups), -1, -1).contiguous() for a in arrs]
            g = AG.chain_greens(*stk, op, groups, z, "hull")
            mo = AG.contour_moments(g, z, wq, 0.0, kmax=1)
            mult = torch.tensor([1.0, 3.0, 5.0], dtype=torch.float64)   # orbitals per l represented by each start
            q = q + conc[central - 1] * torch.sum(mult * mo[:, 0])
            e_band = e_band + conc[central - 1] * torch.sum(mult * mo[:, 1])
        return e_band, q

    e_band, q = energy_charge(cl, dl, Dl)
    (ge_c, ge_d, ge_D) = torch.autograd.grad(e_band, (cl, dl, Dl), retain_graph=True)
    (gq_c, gq_d, gq_D) = torch.autograd.grad(q, (cl, dl, Dl))
    with torch.no_grad():
        for name, x, ge, gq in (("c", cl, ge_c, gq_c), ("d", dl, ge_d, gq_d), ("D", Dl, ge_D, gq_D)):
            for s in range(nsp):
                for l in range(3):
                    x[s, l] += H
                    ep, qp = energy_charge(cl, dl, Dl)
                    x[s, l] -= 2 * H
                    em, qm = energy_charge(cl, dl, Dl)
                    x[s, l] += H
                    fe, fq = (ep - em).item() / (2 * H), (qp - qm).item() / (2 * H)
                    assert abs(ge[s, l].item() - fe) <= 1e-6 * max(abs(fe), 1e-2 * ge.abs().max().item()), (name, s, l)
                    assert abs(gq[s, l].item() - fq) <= 1e-6 * max(abs(fq), 1e-2 * gq.abs().max().item()), (name, s, l)
