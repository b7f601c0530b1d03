"""Gradients of the energy-dependent chains behind ``torch.autograd.Function``.

The reference has no derivatives; these are the reverse mode of its edc route (``edc_setup`` / ``edc_green_blk``,
src/asr_edc.f90:41-71 and :237-316) and of the contour moments of ``ed_moments`` (src/asr_class_scf.f90:797-877,
``contour_moment`` src/asr_contour.f90:124-130), so that the band energy, the sublattice charges and the DOS can be
differentiated with respect to the species parameters (c_l, d_l, Delta_l).

* ``ChainGreens`` -- G(group, energy) of a batch of chain groups as a function of the groups' parameter arrays
  (c, d, o, e, pa, pb per orbital and species).  Forward: ``asr_chains_run``; backward: ``asr_chains_adjoint_ext``, the
  device adjoint (the Lanczos vectors of every level kept where they fit, else every sqrt(depth) levels and
  recomputed; reverse sweep through the recurrence; reverse mode of the continued fraction).
* ``edc_group_arrays``, ``edc_group_o`` -- the map of ``edc_setup`` from species parameters to a group's arrays, in
  torch.
* ``contour_moments`` -- M_k = -(1/pi) Im sum_j w_j (z_j - E_nu)^k G_j.
"""
from __future__ import annotations

import numpy as np
import torch

from .augcls import AugclsOp
from .chains import ChainSpec, chains_adjoint_ext, chains_run

ORB_L = (0, 1, 1, 1, 2, 2, 2, 2, 2)   # l of the nine orbitals s | y z x | xy yz 3z2-r2 xz x2-y2


def _arr(t: torch.Tensor) -> np.ndarray:
    # (nsp, 9) row-major is the (9, nsp) Fortran array of the ABI
    return np.asfortranarray(t.detach().cpu().numpy().astype(np.float64).T)


def _specs(c, d, e, pa, pb, groups, o=None):
    out = []
    for q, (frozen_sp, start_orb, nlev) in enumerate(groups):
        oq = _arr(o[q]) if o is not None else np.zeros((9, c.shape[1]), order="F")
        out.append(ChainSpec(c=_arr(c[q]), d=_arr(d[q]), o=oq, e=_arr(e[q]), pa=_arr(pa[q]), pb=_arr(pb[q]),
                             frozen_sp=int(frozen_sp), start_orb=int(start_orb), nlev=int(nlev)))
    return out


class ChainGreens(torch.autograd.Function):
    """G (ngroup, nz) complex128 of the edc chain groups.

    Inputs: c, d, e, pa, pb -- (ngroup, nsp, 9) float64 tensors (each group's (9, nsp) arrays); o -- the same shape or
    None (o = 0); op -- the operator; groups -- [(frozen_sp, start_orb, nlev)] per group; z (nz) complex energies; tail
    ('none' | 'hull' | 'bp' | 'avg2'); precision ('fp64' | 'fp32'); project; stride (checkpoint spacing; 0: every level
    where it fits, else sqrt(depth)); depth_tol (> 0: the depth test of src/asr_edc.f90:121-127, the derivative taken at the depth each chain stopped at).

    The backward pass gives d(real loss)/dpar = Re(sum conj(dL/dG) dG/dpar): the seeds of the adjoint are the conjugated
    output gradients.  e and pb enter the operator the same way and share one derivative (and c with them when o = 0)."""

    @staticmethod
    def forward(ctx, c, d, e, pa, pb, o, op: AugclsOp, groups, z, tail="hull", precision="fp64", project=True, stride=0,
                depth_tol=0.0):
        specs = _specs(c, d, e, pa, pb, groups, o)
        z = np.ascontiguousarray(np.atleast_1d(z), dtype=np.complex128)
        g = chains_run(op, specs, z, "edc", depth_tol, tail, precision, project)["g"]
        ctx.save_for_backward(c, d, e, pa, pb)
        ctx.o = o.detach() if o is not None else None
        ctx.meta = (op, list(groups), z, tail, precision, project, stride, depth_tol)
        return torch.from_numpy(np.ascontiguousarray(g.T)).to(c.device)

    @staticmethod
    def backward(ctx, gout):
        c, d, e, pa, pb = ctx.saved_tensors
        op, groups, z, tail, precision, project, stride, depth_tol = ctx.meta
        w = np.conj(gout.detach().cpu().numpy()).T
        _, _, gr = chains_adjoint_ext(op, _specs(c, d, e, pa, pb, groups, ctx.o), z, w, depth_tol, tail, precision, project,
                                      stride)
        gr = torch.from_numpy(np.ascontiguousarray(gr.real)).to(device=c.device, dtype=c.dtype)
        ge = gr[:, 4]
        go = gr[:, 3] if ctx.o is not None else None
        return gr[:, 0], gr[:, 1], ge, gr[:, 2], ge.clone(), go, None, None, None, None, None, None, None, None


def chain_greens(c, d, e, pa, pb, op, groups, z, tail="hull", precision="fp64", project=True, stride=0, o=None,
                 depth_tol=0.0):
    """G (ngroup, nz) of the edc chain groups, differentiable in c, d, e, pa, pb and (when given) o."""
    return ChainGreens.apply(c, d, e, pa, pb, o, op, groups, z, tail, precision, project, stride, depth_tol)


def orbital_orbits(dmat) -> list[list[int]]:
    """Orbits (0-based orbital lists) of the nine orbitals under the signed-permutation matrices dmat (9, 9, nop): the
    parameter directions the group-reduced operator can represent are constant on each orbit, and the adjoint's
    per-orbital entries are symmetrised over them."""
    dmat = np.asarray(dmat)
    root = list(range(9))

    def find(l):
        while root[l] != l:
            l = root[l]
        return l
    for g in range(dmat.shape[2]):
        for l in range(9):
            m = int(np.argmax(np.abs(dmat[:, l, g])))
            a, b = find(l), find(m)
            if a != b:
                root[max(a, b)] = min(a, b)
    out = {}
    for l in range(9):
        out.setdefault(find(l), []).append(l)
    return list(out.values())


def per_orbital(x: torch.Tensor) -> torch.Tensor:
    """(nsp, 3) per-l parameters -> (nsp, 9) per-orbital."""
    return x[:, list(ORB_L)]


def edc_group_arrays(cl, dl, Dl, enu, central: int):
    """``edc_setup`` (src/asr_edc.f90:41-71) in torch for central species ``central`` (1-based): from the per-l species
    parameters cl, dl, Dl, enu (nsp, 3) the group arrays (c, d, e, pa, pb), each (nsp, 9): c_s = (D_c / D_s) c_s,
    d = d_c for every species, e = 0, X(z) = z pa + pb with pa = 1 - D_c / D_s and pb = D_c E_nu,s / D_s."""
    c, d, D, en = per_orbital(cl), per_orbital(dl), per_orbital(Dl), per_orbital(enu)
    dc = D[central - 1]
    r = dc[None, :] / D
    return r * c, d[central - 1][None, :].expand_as(d), torch.zeros_like(c), 1.0 - r, r * en


def edc_group_o(ol, Dl, central: int):
    """o of ``edc_setup`` (src/asr_edc.f90:66) in torch: o_s = o_l,s D_s / D_c per (species, orbital), from the per-l
    o_l (nsp, 3) of every species (o of the alpha representation, ``o_alpha`` src/asr_lmto_ham.f90:131-139) and the
    Delta_l (nsp, 3); central 1-based.  Returns (nsp, 9)."""
    o, D = per_orbital(ol), per_orbital(Dl)
    return o * D / D[central - 1][None, :]


def contour_moments(g: torch.Tensor, z, w, enu, kmax: int = 1) -> torch.Tensor:
    """M_k = -(1/pi) Im sum_j w_j (z_j - E_nu)^k G_j (``contour_moment``, src/asr_contour.f90:124-130) for k = 0..kmax
    along the last axis of g; enu broadcasts against g's leading axes.  Returns (..., kmax + 1)."""
    z = torch.as_tensor(np.asarray(z), dtype=torch.complex128, device=g.device)
    w = torch.as_tensor(np.asarray(w), dtype=torch.complex128, device=g.device)
    en = torch.as_tensor(enu, dtype=torch.float64, device=g.device)[..., None]
    out = []
    for k in range(kmax + 1):
        out.append(-torch.imag(torch.sum(w * (z - en) ** k * g, dim=-1)) / np.pi)
    return torch.stack(out, dim=-1)
