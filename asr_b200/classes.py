"""Multi-sublattice chain sets and their moments: the differentiable form of ``chain_greens`` + ``ed_moments``.

The reference runs, per (sublattice, component, start orbital, spin), one energy-dependent chain on the operator whose
start site lies on that sublattice (``chain_greens``, src/asr_class_scf.f90:966-1054, ``chain_worker`` :1071-1160), and
integrates the Green's functions over the contour into the moments M_k(component, spin, k, l) (``ed_moments``
:797-877): M_k = -(1/pi) sum_o w_o Im sum_j w_j (z_j - E_nu)^k G_o(z_j).  Here the start orbitals are one per orbit of
the point group (weight = orbit size, the ``worbk`` of the reference), the species parameters are per l (c_l, d_l,
Delta_l, E_nu,l), and every quantity is a torch function of them, so that band energy, sublattice charges and the DOS
can be differentiated through the device adjoint (``asr_b200.autograd.ChainGreens``).
"""
from __future__ import annotations

import torch

from . import autograd as AG
from .augcls import Context, build_augcls_operator


class SublatticeChains:
    """Operators of the sublattices of one alloy and the chain groups on each.

    cases: one dict per sublattice (graph, model, cls, perm, dmat, maxlevel, maxrank, flippable) whose site 1 lies on
    that sublattice (the same alloy with shifted site classes); nlev: chain depth."""

    def __init__(self, cases, nlev: int, ctx: Context | None = None, tail: str = "hull", precision: str = "fp64",
                 project: bool = True, depth_tol: float = 0.0):
        self.cases = cases
        self.nlev = nlev
        self.tail, self.precision, self.project, self.depth_tol = tail, precision, project, depth_tol
        self.ops = [build_augcls_operator(c["graph"], c["model"], c["cls"], c["perm"], c["dmat"], 1, c["maxlevel"],
                                          maxrank=c["maxrank"], flippable=c["flippable"], ctx=ctx) for c in cases]
        self.nsp = cases[0]["model"].nsp
        # components of each sublattice: (species, concentration) of the class of site 1
        self.comps = []
        for c in cases:
            mdl, k = c["model"], int(c["cls"][0]) - 1
            self.comps.append([(int(mdl.spc[j, k]), float(mdl.conc[j, k])) for j in range(int(mdl.nsc[k]))])
        self.orbits = [AG.orbital_orbits(c["dmat"]) for c in cases]

    def groups(self, kap: int):
        """(frozen species, start orbital, depth) of every group of sublattice kap (0-based), and the orbit weights."""
        out, wts = [], []
        for sp, _ in self.comps[kap]:
            for orb in self.orbits[kap]:
                out.append((sp, orb[0] + 1, self.nlev))
                wts.append(len(orb))
        return out, wts

    def greens(self, cl, dl, Dl, enu, z, ol=None):
        """G per sublattice: list of (ngroup, nz) complex tensors (component-major, then orbit).  ol (nsp, 3): o_l of every
        species (edc_setup's o = o_l D_s / D_c, src/asr_edc.f90:66); None: o = 0."""
        out = []
        for kap, op in enumerate(self.ops):
            groups, _ = self.groups(kap)
            arrs = [[], [], [], [], []]
            oarr = []
            for sp, _, _ in groups:
                for a, v in zip(arrs, AG.edc_group_arrays(cl, dl, Dl, enu, sp)):
                    a.append(v)
                if ol is not None:
                    oarr.append(AG.edc_group_o(ol, Dl, sp))
            stk = [torch.stack(a) for a in arrs]
            out.append(AG.chain_greens(*stk, op, groups, z, self.tail, self.precision, self.project,
                                       o=torch.stack(oarr) if ol is not None else None, depth_tol=self.depth_tol))
        return out

    def energy_and_charges(self, cl, dl, Dl, enu, z, w, ol=None):
        """Band energy sum_kap sum_s x_s sum_l (M_1 + E_nu M_0) and sublattice charges Q_kap = sum_s x_s sum_l M_0 from the
        contour (z, w); the moments are taken about E_nu of each (species, orbital)."""
        gs = self.greens(cl, dl, Dl, enu, z, ol)
        e_band = torch.zeros((), dtype=torch.float64)
        q = []
        for kap, g in enumerate(gs):
            groups, wts = self.groups(kap)
            en = torch.stack([AG.per_orbital(enu)[sp - 1, orb - 1] for sp, orb, _ in groups])
            mo = AG.contour_moments(g, z, w, en.detach().numpy(), kmax=1)
            x = torch.tensor([dict(self.comps[kap])[sp] for sp, _, _ in groups], dtype=torch.float64)
            wt = torch.tensor(wts, dtype=torch.float64)
            q.append(torch.sum(x * wt * mo[:, 0]))
            e_band = e_band + torch.sum(x * wt * (mo[:, 1] + en * mo[:, 0]))
        return e_band, torch.stack(q)

    def dos(self, cl, dl, Dl, enu, e, eta: float, ol=None):
        """DOS per sublattice on the real axis, -(1/pi) Im sum_s x_s sum_o w_o G_o(e + i eta) (the l-summed form of
        ``dos_final``, src/asr_class_scf.f90:1912-1931), differentiable in the species parameters: a list of (ne,) tensors."""
        import numpy as np
        z = np.asarray(e, dtype=np.float64) + 1j * eta
        gs = self.greens(cl, dl, Dl, enu, z, ol)
        out = []
        for kap, g in enumerate(gs):
            groups, wts = self.groups(kap)
            x = torch.tensor([dict(self.comps[kap])[sp] for sp, _, _ in groups], dtype=torch.float64)
            wt = torch.tensor(wts, dtype=torch.float64)
            out.append(-torch.sum((x * wt)[:, None] * torch.imag(g), dim=0) / np.pi)
        return out
