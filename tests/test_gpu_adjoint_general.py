"""The device adjoint on the reference's whole operator form (asr_chains_adjoint_ext): H = E_nu + h - h o h + X(z) with
edc_setup's o = o_l D_s / D_c (src/asr_edc.f90:66), the Beer-Pettifor tail (src/asr_chain.f90:126-156) and chains
stopped by the depth test (src/asr_edc.f90:121-127), against central differences (h = 1e-5, Richardson-extrapolated) of
the CUDA forward; the o = 0 form equals asr_chains_adjoint; the DOS gradient through torch.autograd."""
import numpy as np
import pytest

from asr_b200 import augcls as A
from asr_b200 import autograd as AG
from asr_b200 import chains as CH
from asr_b200 import synthetic as S
from tests import cases as K

pytestmark = pytest.mark.gpu

H = 1e-5
KIND = {"c": 0, "d": 1, "pa": 2, "o": 3, "e": 4, "pb": 4}


def _setup(seed=0, depths=(12, 9, 14)):
    case = K.cubic("bcc", 3, 2, (0.5, 0.5), group="d4h", maxlevel=3, maxrank=1)
    args = (case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, case["maxlevel"])
    op = A.build_augcls_operator(*args, maxrank=case["maxrank"], flippable=case["flippable"])
    sp = S.draw_species(2, seed)
    ol = S.draw_o(2, seed)
    specs = []
    for q, (central, orb) in enumerate([(1, 1), (2, 5), (1, 3)]):
        ed = S.edc_params_o(sp, ol, central)
        e = np.asfortranarray(0.05 * np.cos(np.arange(2)[None, :] + 0.3 * q) * np.ones((9, 1)))
        specs.append(CH.ChainSpec(c=ed["c"], d=ed["d"], o=ed["o"], e=e, pa=ed["pa"], pb=ed["pb"], frozen_sp=central,
                                  start_orb=orb, nlev=depths[q]))
    return op, specs, AG.orbital_orbits(case["dmat"])


def _central(f, h=H):
    d1 = (f(h) - f(-h)) / (2 * h)
    d2 = (f(h / 2) - f(-h / 2)) / h
    return (4 * d2 - d1) / 3


def _perturbed(specs, q, kind, orbit, s, h):
    out = []
    for p, sp in enumerate(specs):
        vals = {k: getattr(sp, k).copy(order="F") for k in ("c", "d", "o", "e", "pa", "pb")}
        if p == q:
            vals[kind][orbit, s] += h
        out.append(CH.ChainSpec(**vals, frozen_sp=sp.frozen_sp, start_orb=sp.start_orb, nlev=sp.nlev))
    return out


@pytest.mark.parametrize("tail", ["hull", "bp"])
def test_general_operator_adjoint_matches_differences(tail):
    """Every kind (c, d, pa, o, e, pb) along every orbit direction of a random species of every group, o != 0."""
    op, specs, orbits = _setup()
    z = np.linspace(-0.5, 0.3, 6) + 0.1j
    rng = np.random.default_rng(5)
    w = rng.standard_normal((6, 3)) + 1j * rng.standard_normal((6, 3))
    g, m, grad = CH.chains_adjoint_ext(op, specs, z, w, 0.0, tail)
    g_fwd = CH.chains_run(op, specs, z, "edc", 0.0, tail, "fp64")["g"]
    assert np.max(np.abs(g - g_fwd) / np.abs(g_fwd)) < 1e-12
    assert np.max(np.abs(grad[:, 3])) > 0          # the o kind is live

    def loss(sp):
        return np.sum(w * CH.chains_run(op, sp, z, "edc", 0.0, tail, "fp64")["g"])
    worst, where = 0.0, None
    for q in range(3):
        scale = np.max(np.abs(grad[q]))
        for kind in ("c", "d", "pa", "o", "e", "pb"):
            for orbit in orbits:
                s = int(rng.integers(2))
                fd = _central(lambda h: loss(_perturbed(specs, q, kind, orbit, s, h)))
                adj = np.sum(grad[q, KIND[kind], s, orbit])
                err = abs(adj - fd) / max(abs(fd), 1e-2 * scale)
                if err > worst:
                    worst, where = err, (q, kind, orbit, s, adj, fd)
    assert worst < 1e-6, (worst, where)


def test_adjoint_at_the_depth_the_depth_test_stopped():
    """With the depth test the chains stop at different depths; the adjoint differentiates each chain at its depth (the
    perturbed forwards stop at the same depths)."""
    op, specs, orbits = _setup(seed=3, depths=(40, 40, 40))
    z = np.linspace(-0.8, 0.4, 9) + 0.02j
    w = np.linspace(1.0, 2.0, 27).reshape(9, 3) + 0.5j
    tol = 1e-4
    g, m, grad = CH.chains_adjoint_ext(op, specs, z, w, tol, "hull")
    r = CH.chains_run(op, specs, z, "edc", tol, "hull", "fp64")
    assert np.array_equal(m, r["m"]) and len(set(m.ravel().tolist())) > 1 and np.min(m) < 40
    assert np.max(np.abs(g - r["g"]) / np.abs(r["g"])) < 1e-12

    def loss(sp):
        rr = CH.chains_run(op, sp, z, "edc", tol, "hull", "fp64")
        assert np.array_equal(rr["m"], m)
        return np.sum(w * rr["g"])
    worst = 0.0
    for q in range(3):
        scale = np.max(np.abs(grad[q]))
        for kind, s in (("c", 0), ("d", 1), ("o", 1), ("pa", 0)):
            for orbit in orbits[:3]:
                fd = _central(lambda h: loss(_perturbed(specs, q, kind, orbit, s, h)))
                adj = np.sum(grad[q, KIND[kind], s, orbit])
                worst = max(worst, abs(adj - fd) / max(abs(fd), 1e-2 * scale))
    assert worst < 1e-6, worst


def test_o_zero_form_equals_the_three_kind_entry_point():
    op, specs, _ = _setup(seed=1)
    zero = np.zeros((9, 2), order="F")
    specs = [CH.ChainSpec(c=s.c, d=s.d, o=zero, e=s.e, pa=s.pa, pb=s.pb, frozen_sp=s.frozen_sp, start_orb=s.start_orb,
                          nlev=s.nlev) for s in specs]
    z = np.linspace(-0.4, 0.2, 4) + 0.08j
    w = np.ones((4, 3), complex)
    _, g3 = CH.chains_adjoint(op, specs, z, w, "hull", "fp64", True)
    _, _, g5 = CH.chains_adjoint_ext(op, specs, z, w, 0.0, "hull", "fp64", True)
    assert np.array_equal(g5[:, :3], g3)
    assert np.array_equal(g5[:, 4], g5[:, 0]) and not np.any(g5[:, 3])


def test_the_three_kind_entry_point_refuses_o():
    op, specs, _ = _setup()
    with pytest.raises(Exception, match="o != 0"):
        CH.chains_adjoint(op, specs, np.array([0.1j]), np.ones((1, 3)), "hull", "fp64", True)


def test_dos_gradient_through_autograd():
    """d DOS(E) / d(c_l, d_l, Delta_l) of a sublattice with o != 0 against central differences of the forward."""
    import torch
    from asr_b200 import classes as CL
    cases = [S.heusler_case(4, 3, k) for k in (4,)]
    sc = CL.SublatticeChains(cases, 16)
    sp = S.draw_species(5, 3)
    ol = torch.tensor(S.draw_o(5, 3), dtype=torch.float64)
    enu = torch.zeros(5, 3, dtype=torch.float64)
    e = np.linspace(-0.9, 0.3, 7)
    params = [torch.tensor(x, dtype=torch.float64, requires_grad=True) for x in (sp.c, sp.d, sp.delta)]
    dos = sc.dos(*params, enu, e, 0.02, ol)[0]
    seed = torch.linspace(0.5, 1.5, 7, dtype=torch.float64)
    grads = torch.autograd.grad(torch.sum(seed * dos), params)
    gmax = max(g.abs().max().item() for g in grads)
    base = [p.detach().numpy().copy() for p in params]

    def f(vals):
        with torch.no_grad():
            return torch.sum(seed * sc.dos(*[torch.tensor(v) for v in vals], enu, e, 0.02, ol)[0]).item()
    for a, s, l in ((0, 3, 2), (1, 4, 1), (2, 3, 0), (2, 4, 2), (0, 0, 1)):
        def shifted(h):
            v = [x.copy() for x in base]
            v[a][s, l] += h
            return f(v)
        fd = _central(shifted)
        assert abs(grads[a][s, l].item() - fd) <= 1e-6 * max(abs(fd), 1e-2 * gmax), (a, s, l, grads[a][s, l].item(), fd)


def test_kept_vectors_and_checkpoints_give_the_same_bits():
    """stride 0 keeps every level's vectors when the device has room (no recomputation); explicit strides checkpoint and
    recompute: the general operator's gradient is the same bit for bit."""
    op, specs, _ = _setup(seed=2)
    z = np.linspace(-0.4, 0.2, 5) + 0.06j
    w = np.ones((5, 3), complex)
    ref = CH.chains_adjoint_ext(op, specs, z, w, 0.0, "hull", "fp64", True, stride=0)[2]
    for stride in (1, 3, 40):
        gr = CH.chains_adjoint_ext(op, specs, z, w, 0.0, "hull", "fp64", True, stride=stride)[2]
        assert np.array_equal(gr, ref), stride


def test_held_workspace_gives_the_same_bits():
    """asr_ctx_hold_workspace: the vector memory kept in the context and reused by the next calls (also by a smaller
    call) gives the gradient of the allocating call bit for bit; turning it off frees it."""
    op, specs, _ = _setup(seed=4)
    z = np.linspace(-0.4, 0.2, 5) + 0.06j
    w = np.ones((5, 3), complex)
    ref = CH.chains_adjoint_ext(op, specs, z, w, 0.0, "hull", "fp64", True)[2]
    op.ctx.hold_workspace(True)
    try:
        for zz, ww in ((z, w), (z, w), (z[:2], w[:2])):
            gr = CH.chains_adjoint_ext(op, specs, zz, ww, 0.0, "hull", "fp64", True)[2]
            if zz is z:
                assert np.array_equal(gr, ref)
    finally:
        op.ctx.hold_workspace(False)
    assert np.array_equal(CH.chains_adjoint_ext(op, specs, z, w, 0.0, "hull", "fp64", True)[2], ref)
