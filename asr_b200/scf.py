"""Self-consistency around the chains: contour moments, Fermi-level search and the mixing step.

This is the caller side of the hot path in the reference's ``class_scf`` (src/asr_class_scf.f90): ``ed_moments``
(:797-877) integrates the chain Green's functions over the contour into the moments M_k(component, spin, l) and the DOS
at E_F; the E_F search (:470-560) brackets N(E_F) = N_elec with secant steps and a first-order step from the DOS at E_F;
the mixing step is Anderson mixing with safeguards (``anderson_step``, src/asr_mixing.f90:1-102).  The reference's
potential update (radial densities, Poisson, exchange-correlation, Madelung) is TB-LMTO-ASA physics outside this
project; here a model potential update closes the loop: the band centres of species s, spin sigma respond to the
charges as C_{s,l,sigma} = C0_{s,l} + U_s (Q_s - Z_s) - sigma I_s m_s / 2 (screened on-site response and a Stoner term).
The fixed point x = (Q_{s,sigma}) is reached with

* ``Anderson`` -- the reference's mixer, restated: x_{k+1} = x_k + beta r_k - sum_j gamma_j (dX_j + beta dR_j), gamma
  from a ridge-regularised least-squares fit of r_k by the residual differences, history reset when |r| doubles and
  when the step points against the residual (newest pair first, then a linear step);
* ``Broyden`` -- quasi-Newton on r(x) = F(x) - x whose first inverse Jacobian (and, with ``refresh``, every one) comes
  from the adjoint: dF/dx = dQ/dC . dC/dx with dQ/dC from one reverse sweep of all chain groups (each group feeds one
  charge, so one sweep gives every row); Broyden's rank-one update corrects it between refreshes.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import contour as CT
from .chains import ChainSpec, chains_adjoint, chains_run

ORB_L = np.array([0, 1, 1, 1, 2, 2, 2, 2, 2])


# ---------------------------------------------------------------------------------------------------------- mixers
class Anderson:
    """Anderson mixing with the safeguards of src/asr_mixing.f90:18-102 (history m, step beta, metric w)."""

    def __init__(self, n: int, m: int = 6, beta: float = 0.2, beta_restart: float | None = None, w=None):
        self.n, self.m, self.beta = n, m, beta
        self.beta_restart = beta if beta_restart is None else beta_restart
        self.w = np.ones(n) if w is None else np.asarray(w, float)
        self.dx = np.zeros((n, m))
        self.dr = np.zeros((n, m))
        self.xold = None
        self.rold = None
        self.nfill = 0
        self.nh = 0
        self.nrestart = 0

    def _norm(self, v):
        return float(np.sqrt(np.sum(self.w * v * v)))

    def _restart(self):
        self.nh = 0
        self.nfill = 0
        self.nrestart += 1

    def _fit(self, xin, r, br):
        nh = self.nh
        if nh == 0:
            return xin + br * r
        xn = xin + self.beta * r
        dr = self.dr[:, :nh]
        a = (dr * self.w[:, None]).T @ dr
        rhs = (dr * self.w[:, None]).T @ r
        a[np.diag_indices(nh)] = a[np.diag_indices(nh)] * (1.0 + 1.0e-8) + 1.0e-30
        try:
            g = np.linalg.solve(a, rhs)
        except np.linalg.LinAlgError:
            return xn
        return xn - (self.dx[:, :nh] + self.beta * dr) @ g

    def step(self, xin, xout, safeguard: bool = True):
        """x_next from the input xin and its image xout = F(xin)."""
        xin = np.asarray(xin, float)
        r = np.asarray(xout, float) - xin
        if safeguard and self.rold is not None and self._norm(r) > 2.0 * self._norm(self.rold):
            self._restart()                                          # the residual blew up
        if self.rold is not None:
            slot = self.nfill % self.m
            self.dx[:, slot] = xin - self.xold
            self.dr[:, slot] = r - self.rold
            self.nfill += 1
            self.nh = min(self.nfill, self.m)
        self.xold, self.rold = xin.copy(), r.copy()
        xn = self._fit(xin, r, self.beta_restart)
        if not safeguard or self.nh == 0 or np.sum(self.w * (xn - xin) * r) > 0.0:
            return xn
        if self.nh > 1:                                               # against the residual: the newest pair alone
            slot = (self.nfill - 1) % self.m
            self.dx[:, 0], self.dr[:, 0] = self.dx[:, slot].copy(), self.dr[:, slot].copy()
            self._restart()
            self.nfill, self.nh = 1, 1
            xn = self._fit(xin, r, self.beta_restart)
            if np.sum(self.w * (xn - xin) * r) > 0.0:
                return xn
        self._restart()
        return xin + self.beta_restart * r


class Broyden:
    """Quasi-Newton on r(x) = F(x) - x: x_next = x - H r with H ~ (dF/dx - I)^-1, Broyden's rank-one update
    H += (dx - H dr) dx^T H / (dx^T H dr) between Jacobians supplied by ``set_jacobian``."""

    def __init__(self, n: int, beta: float = 0.2, damping: float = 1.0):
        self.n, self.beta, self.damping = n, beta, damping
        self.H = -beta * np.eye(n)          # no Jacobian yet: linear mixing
        self.xold = None
        self.rold = None

    def set_jacobian(self, dfdx):
        j = np.asarray(dfdx, float) - np.eye(self.n)
        self.H = np.linalg.inv(j)

    def step(self, xin, xout):
        xin = np.asarray(xin, float)
        r = np.asarray(xout, float) - xin
        if self.xold is not None:
            dx, dr = xin - self.xold, r - self.rold
            hdr = self.H @ dr
            den = dx @ hdr
            if abs(den) > 1e-14 * (np.linalg.norm(dx) * np.linalg.norm(hdr) + 1e-300):
                self.H += np.outer(dx - hdr, dx @ self.H) / den
        self.xold, self.rold = xin.copy(), r.copy()
        return xin - self.damping * (self.H @ r)


# ---------------------------------------------------------------------------------------------------------- the model
@dataclass
class ScfModel:
    """One site class with nsp components (concentrations x), spin-polarised, the edc route.

    c0, d, delta (nsp, 3): species parameters per l of the start potential; z (nsp): valence of each species;
    u (nsp): screened on-site response (Ry per electron); stoner (nsp): exchange splitting per unit moment."""
    op: object
    x: np.ndarray
    c0: np.ndarray
    d: np.ndarray
    delta: np.ndarray
    z: np.ndarray
    u: np.ndarray
    stoner: np.ndarray
    depths: np.ndarray          # (2, nsp, 9) chain depth of every group
    ebot: float = -1.2
    ncont: int = 64
    eta: float = 0.005
    tail: str = "hull"
    precision: str = "fp64"
    orbitals: tuple = tuple(range(1, 10))
    weights: tuple = (1,) * 9
    stats: dict = field(default_factory=lambda: {"forward": 0, "adjoint": 0, "chain_steps": 0})

    @property
    def nsp(self):
        return len(self.x)

    @property
    def nelec(self):
        return float(np.sum(self.x * self.z))

    def band_centres(self, q):
        """C (2, nsp, 3) from the charges q (2, nsp): the model potential update."""
        qt = q[0] + q[1]
        m = q[0] - q[1]
        shift = self.u * (qt - self.z)
        c = np.empty((2, self.nsp, 3))
        for sg, sign in enumerate((1.0, -1.0)):
            c[sg] = self.c0 + (shift - 0.5 * sign * self.stoner * m)[:, None]
        return c

    def specs(self, c):
        """Chain groups (spin, central species, orbital) in the edc form of ``edc_setup`` (src/asr_edc.f90:41-71)."""
        out = []
        for sg in range(2):
            for cen in range(self.nsp):
                dc = self.delta[cen][ORB_L]
                r = dc[:, None] / self.delta[:, ORB_L].T                         # (9, nsp): D_c / D_s
                cc = np.asfortranarray(r * c[sg][:, ORB_L].T)
                dd = np.asfortranarray(np.repeat(self.d[cen][ORB_L][:, None], self.nsp, axis=1))
                z9 = np.zeros((9, self.nsp), order="F")
                for o in self.orbitals:
                    out.append(ChainSpec(c=cc, d=dd, o=z9, e=z9, pa=np.asfortranarray(1.0 - r), pb=z9.copy(order="F"),
                                         frozen_sp=cen + 1, start_orb=o, nlev=int(self.depths[sg, cen, o - 1])))
        return out

    def contour(self, ef):
        z, w = CT.contour_nodes(self.ebot, ef, self.ncont)
        return np.concatenate([z, [complex(ef, self.eta)]]), np.concatenate([w, [0.0]])

    def moments(self, c, ef):
        """``ed_moments``: charges q (2, nsp) (sum over l and the orbital weights), band energy, DOS at E_F (2, nsp), and
        the chain data for the adjoint."""
        zs, ws = self.contour(ef)
        specs = self.specs(c)
        g = chains_run(self.op, specs, zs, "edc", 0.0, self.tail, self.precision)["g"]     # (nz, ngroup)
        self.stats["forward"] += 1
        self.stats["chain_steps"] += int(sum(s.nlev for s in specs)) * len(zs)
        no = len(self.orbitals)
        wt = np.asarray(self.weights, float)
        gq = g.reshape(len(zs), 2, self.nsp, no)
        m0 = -np.imag(np.einsum("j,jsco->sco", ws, gq)) / np.pi
        m1 = -np.imag(np.einsum("j,jsco->sco", ws * zs, gq)) / np.pi
        dos = -np.imag(gq[-1]) / np.pi
        q = np.einsum("sco,o->sc", m0, wt)
        eb = float(np.einsum("sco,o,c->", m1, wt, self.x))
        return q, eb, np.einsum("sco,o->sc", dos, wt), (zs, ws, specs)

    def fermi_level(self, c, ef, maxit: int = 12, tol: float = 1e-8):
        """E_F with sum_s x_s Q_s = N_elec: secant steps on a bracket, else a first-order step from the DOS at E_F clamped
        to 0.15 Ry (the scheme of src/asr_class_scf.f90:470-526).  Returns (ef, q, eb, data, passes)."""
        lo = hi = None
        for it in range(maxit):
            q, eb, dos, data = self.moments(c, ef)
            n = float(np.sum(self.x * (q[0] + q[1])))
            res = n - self.nelec
            if abs(res) < tol:
                return ef, q, eb, data, it + 1
            if res < 0:
                lo = (ef, res)
            else:
                hi = (ef, res)
            if lo is not None and hi is not None:
                e = (lo[0] * hi[1] - hi[0] * lo[1]) / (hi[1] - lo[1])
                w_ = abs(hi[0] - lo[0])
                if not (min(lo[0], hi[0]) + 1e-3 * w_ < e < max(lo[0], hi[0]) - 1e-3 * w_):
                    e = 0.5 * (lo[0] + hi[0])
                ef = e
            else:
                dn = float(np.sum(self.x * (dos[0] + dos[1])))
                ef = ef + max(-0.15, min(0.15, -res / max(dn, 1.0)))
        return ef, q, eb, data, maxit

    def jacobian(self, c, data):
        """dQ_out/dx (2 nsp, 2 nsp) at fixed E_F: one adjoint sweep of every group (seeds = the contour weights), the
        per-group parameter gradients summed into dQ_{s,sigma}/dC_{s',l,sigma}, times dC/dx of the model."""
        zs, ws, specs = data
        ng = len(specs)
        no = len(self.orbitals)
        wt = np.asarray(self.weights, float)
        # Q = -(1/pi) Im sum_j w_j G_j = Re(sum_j (i/pi) w_j G_j): seeds (i/pi) w_j, the real part of the gradient
        seeds = np.repeat(((1j / np.pi) * ws)[:, None], ng, axis=1)
        _, grad = chains_adjoint(self.op, specs, zs, seeds, self.tail, self.precision)
        self.stats["adjoint"] += 1
        gr = grad.real.reshape(2, self.nsp, no, 3, self.nsp, 9)          # (spin, central, orbital, kind, species, l)
        # dQ_{sg,cen}/dC_{sg,s,l}: kind 0 is d/dc of the group arrays, c_s = (D_c / D_s) C_s
        dq_dc = np.zeros((2, self.nsp, self.nsp, 3))
        for sg in range(2):
            for cen in range(self.nsp):
                r = self.delta[cen][ORB_L][:, None] / self.delta[:, ORB_L].T             # (9, nsp)
                g0 = np.einsum("o,osl->ls", wt, gr[sg, cen, :, 0])                      # (9 l, nsp)
                for l in range(3):
                    sel = ORB_L == l
                    dq_dc[sg, cen, :, l] = np.sum((g0 * r)[sel], axis=0)
        # model: C_{sg,s,l} = C0 + U_s (Q_s - Z_s) - sign_sg I_s m_s / 2
        n = 2 * self.nsp
        dcdx = np.zeros((2, self.nsp, n))          # dC_{sg,s}/dx (same for every l)
        for sg, sign in enumerate((1.0, -1.0)):
            for s in range(self.nsp):
                for sg2, sign2 in enumerate((1.0, -1.0)):
                    dcdx[sg, s, sg2 * self.nsp + s] = self.u[s] - 0.5 * sign * self.stoner[s] * sign2
        jac = np.zeros((n, n))
        for sg in range(2):
            for cen in range(self.nsp):
                jac[sg * self.nsp + cen] = np.einsum("sl,sx->x", dq_dc[sg, cen], dcdx[sg])
        return jac


def scf_run(model: ScfModel, q0, ef0: float, mixer: str = "anderson", tol: float = 1e-6, maxit: int = 40, beta: float = 0.2,
            refresh: int = 1, refine_below: float = 1e-2, verbose: bool = False):
    """Iterate x = (Q_{s,sigma}) to |F(x) - x|_inf < tol.  mixer 'anderson' (the reference's) or 'broyden' (adjoint
    Jacobian every ``refresh`` iterations).  A model running in FP32 (matvec and vectors) switches to FP64 once the
    residual is below ``refine_below``: on a 5-component alloy the quasi-Newton steps from FP32 charges and Jacobians
    stalled between 1e-4 and 1e-3, so the last iterations refine in FP64.
    Returns dict(q, ef, iterations, history, seconds, stats)."""
    x = np.asarray(q0, float).ravel()
    start_precision = model.precision
    n = x.size
    mx = Anderson(n, beta=beta) if mixer == "anderson" else Broyden(n, beta=beta)
    ef = ef0
    hist = []
    t0 = time.perf_counter()
    for it in range(1, maxit + 1):
        c = model.band_centres(x.reshape(2, -1))
        ef, q, eb, data, npass = model.fermi_level(c, ef)
        r = q.ravel() - x
        hist.append(dict(iteration=it, residual=float(np.max(np.abs(r))), ef=ef, band_energy=eb, ef_passes=npass))
        if verbose:
            print(hist[-1])
        if np.max(np.abs(r)) < tol and model.precision == "fp64":
            x = q.ravel()
            break
        if model.precision == "fp32" and np.max(np.abs(r)) < refine_below:
            model.precision = "fp64"
        if mixer == "broyden" and (it - 1) % max(refresh, 1) == 0:
            mx.set_jacobian(model.jacobian(c, data))
        x = mx.step(x, q.ravel())
    conv = hist[-1]["residual"] < tol and model.precision == "fp64"
    model.precision = start_precision
    return dict(q=x.reshape(2, -1), ef=ef, iterations=len(hist), converged=conv, history=hist, seconds=time.perf_counter() - t0,
                stats=dict(model.stats))
