"""SCF coupling on the GPU: the adjoint Jacobian of the charges against central differences at fixed E_F, and the
fixed point reached by Anderson mixing (the reference's) and by the adjoint-fed Broyden mixer."""
import numpy as np
import pytest

from asr_b200 import augcls as A
from asr_b200 import scf as SC
from asr_b200 import synthetic as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def model():
    case = S.cubic_case("bcc", 3, 2, [0.5, 0.5], seed=3, group="d2h")
    fl = np.ones(case["graph"].n, np.int32)
    fl[0] = 0
    op = A.build_augcls_operator(case["graph"], case["model"], case["cls"], case["perm"], case["dmat"], 1, 2, maxrank=1,
                                 flippable=fl)
    sp = S.draw_species(2, 3)
    return SC.ScfModel(op=op, x=np.array([0.5, 0.5]), c0=sp.c, d=sp.d, delta=sp.delta, z=np.array([7.0, 9.0]),
                       u=np.array([0.10, 0.08]), stoner=np.array([0.06, 0.04]), depths=np.full((2, 2, 9), 12),
                       ebot=-2.0, ncont=16)


def test_adjoint_jacobian_of_the_charges(model):
    q0 = np.array([[4.0, 5.0], [3.2, 4.1]])
    c = model.band_centres(q0)
    ef = 0.0
    q, eb, dos, data = model.moments(c, ef)
    jac = model.jacobian(c, data)
    h = 1e-5
    fd = np.zeros_like(jac)
    for k in range(4):
        for sgn in (1.0, -1.0):
            x = q0.ravel().copy()
            x[k] += sgn * h
            qk = model.moments(model.band_centres(x.reshape(2, 2)), ef)[0].ravel()
            fd[:, k] += sgn * qk / (2 * h)
    assert np.max(np.abs(jac - fd)) < 1e-6 * np.max(np.abs(fd))


def test_anderson_and_adjoint_broyden_reach_the_same_fixed_point(model):
    """Without exchange splitting the fixed point is unique: both mixers reach it, the adjoint-fed one in fewer
    iterations.  With it (Stoner term) each mixer reaches a self-consistent solution with neutral charge (the magnetic
    and the non-magnetic solutions are both fixed points of the model)."""
    from dataclasses import replace
    m0 = replace(model, stoner=np.zeros(2))
    q0 = np.array([[4.0, 5.0], [3.0, 4.0]])
    ra = SC.scf_run(m0, q0, 0.0, mixer="anderson", tol=1e-7, maxit=80, beta=0.2)
    rb = SC.scf_run(m0, q0, 0.0, mixer="broyden", tol=1e-7, maxit=80, beta=0.2)
    assert ra["converged"] and rb["converged"]
    assert np.max(np.abs(ra["q"] - rb["q"])) < 1e-6
    assert rb["iterations"] <= ra["iterations"]
    for mixer in ("anderson", "broyden"):
        r = SC.scf_run(model, q0, 0.0, mixer=mixer, tol=1e-7, maxit=80, beta=0.2)
        assert r["converged"], mixer
        assert abs(np.sum(model.x * (r["q"][0] + r["q"][1])) - model.nelec) < 1e-6
