"""The mixing step of the SCF loop on host: Anderson mixing with the safeguards of src/asr_mixing.f90, and the
quasi-Newton (Broyden) mixer that the adjoint Jacobian feeds."""
import numpy as np

from asr_b200.scf import Anderson, Broyden


def _linear_map(n=12, rho=0.95, seed=0):
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    a = q @ np.diag(rng.uniform(-rho, rho, n)) @ q.T
    b = rng.standard_normal(n)
    return (lambda x: a @ x + b), np.linalg.solve(np.eye(n) - a, b), a


def _iterate(step, f, x, tol=1e-10, maxit=500):
    for it in range(1, maxit + 1):
        fx = f(x)
        if np.max(np.abs(fx - x)) < tol:
            return x, it
        x = step(x, fx)
    return x, maxit


def test_anderson_beats_linear_mixing_on_a_stiff_linear_map():
    f, xs, _ = _linear_map()
    x0 = np.zeros(12)
    xl, nl = _iterate(lambda x, fx: x + 0.2 * (fx - x), f, x0)
    mx = Anderson(12, m=8, beta=0.2)
    xa, na = _iterate(mx.step, f, x0)
    assert np.max(np.abs(xa - xs)) < 1e-8
    assert na < nl / 5


def test_anderson_restarts_when_the_residual_blows_up():
    mx = Anderson(3, m=4, beta=0.5)
    x = np.zeros(3)
    x = mx.step(x, np.ones(3))                  # r = 1
    x = mx.step(x, x + 10.0 * np.ones(3))       # |r| grew tenfold: the history is dropped
    assert mx.nrestart >= 1
    assert mx.nh <= 1


def test_anderson_step_never_points_against_the_residual():
    rng = np.random.default_rng(3)
    f, xs, _ = _linear_map(8, 0.99, seed=3)
    mx = Anderson(8, m=5, beta=0.3)
    x = rng.standard_normal(8)
    for _ in range(30):
        fx = f(x)
        xn = mx.step(x, fx)
        assert np.dot(xn - x, fx - x) > 0.0 or np.allclose(fx, x)
        x = xn


def test_broyden_with_the_exact_jacobian_is_newton():
    f, xs, a = _linear_map(10, 0.9, seed=1)
    mx = Broyden(10)
    mx.set_jacobian(a)
    x = mx.step(np.zeros(10), f(np.zeros(10)))
    assert np.max(np.abs(x - xs)) < 1e-10


def test_broyden_converges_on_a_nonlinear_map_from_linear_mixing():
    rng = np.random.default_rng(2)
    _, _, a = _linear_map(6, 0.8, seed=2)
    b = rng.standard_normal(6)
    f = lambda x: a @ np.tanh(x) + b
    mx = Broyden(6, beta=0.3)
    x, n = _iterate(mx.step, f, np.zeros(6), tol=1e-10)
    assert np.max(np.abs(f(x) - x)) < 1e-9
    assert n < 60
