"""Operator inputs: periodic cubic graphs and cubic point-group operations.

Host-side restatement of the graph and symmetry inputs that asr's operator builder consumes:

* ``periodic_graph_shells`` -- ``src/asr_lattices.f90:201-250`` (site order, slot order by (|v|^2, components));
* ``periodic_graph`` -- ``src/asr_lattices.f90:166-197`` (nearest-neighbour shell only);
* ``cubic_site_perms`` -- ``src/asr_symmetry.f90:13-42`` (48 signed axis permutations, operation 1 = identity);
* ``class_ops`` -- ``src/asr_symmetry.f90:67-92`` (class-preserving D4h subset);
* ``d2h_ops`` -- the diagonal operations of the class-preserving group (``src/asr_class_scf.f90:1613-1619``), under which
  all nine real orbitals are one dimensional;
* ``ylm_real`` / ``orbital_rep`` -- ``src/asr_harmonics.f90`` and ``src/asr_symmetry.f90:100-129``.

Arrays follow the reference layout: ``perm`` is (nsite, nop) in Fortran order with 1-based site values, ``dmat`` is
(9, 9, nop) in Fortran order, graphs are CSR with 1-based ``nbr_ptr`` / ``nbr``.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

__all__ = ["Graph", "periodic_graph_shells", "periodic_graph", "cubic_site_perms", "class_ops", "d2h_ops", "ylm_real",
           "orbital_rep", "identity_group"]


@dataclass
class Graph:
    """CSR neighbour lists (``graph_t``, src/asr_augspace.f90:22-25): 1-based ``nbr_ptr`` (n+1) and ``nbr``."""
    n: int
    nbr_ptr: np.ndarray
    nbr: np.ndarray

    @property
    def nslot(self) -> int:
        return int(np.max(np.diff(self.nbr_ptr))) if self.n else 0


def _on_lat(kind: str, i, j, k):
    i, j, k = np.asarray(i), np.asarray(j), np.asarray(k)
    if kind == "sc":
        return (i % 2 == 0) & (j % 2 == 0) & (k % 2 == 0)
    if kind == "bcc":
        return (i % 2 == j % 2) & (j % 2 == k % 2)
    if kind == "fcc":
        return (i + j + k) % 2 == 0
    raise ValueError(f"unknown lattice {kind!r}")


def _sites(kind: str, m: int):
    # loop order of the reference: k outer, j, i inner (i fastest)
    k, j, i = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    on = _on_lat(kind, i, j, k)
    coord = np.stack([i[on], j[on], k[on]]).astype(np.int64)
    idx = -np.ones((m, m, m), dtype=np.int64)
    idx[coord[0], coord[1], coord[2]] = np.arange(coord.shape[1])
    return coord, idx


def periodic_graph_shells(kind: str, l: int, r2max: int):
    """Periodic graph with every neighbour within ``r2max`` (half-lattice units squared).

    Returns ``(graph, coord, bvec)``; slot k of every site is the bond vector ``bvec[:, k]``.
    """
    m = 2 * l
    coord, idx = _sites(kind, m)
    rmax = int(np.sqrt(float(r2max))) + 1
    vecs = []
    for k in range(-rmax, rmax + 1):
        for j in range(-rmax, rmax + 1):
            for i in range(-rmax, rmax + 1):
                if i == 0 and j == 0 and k == 0:
                    continue
                if kind != "sc" and not _on_lat(kind, i % 2, j % 2, k % 2):
                    continue
                if kind == "sc" and (i % 2 or j % 2 or k % 2):
                    continue
                if i * i + j * j + k * k > r2max:
                    continue
                vecs.append((i, j, k))
    key = [(v[0] ** 2 + v[1] ** 2 + v[2] ** 2) * 100000 + (v[0] + 50) * 10000 + (v[1] + 50) * 100 + (v[2] + 50) for v in vecs]
    order = np.argsort(np.asarray(key), kind="stable")
    bvec = np.asarray(vecs, dtype=np.int64)[order].T.copy()
    nv = bvec.shape[1]
    n = coord.shape[1]
    q = (coord[:, :, None] + bvec[:, None, :]) % m               # (3, n, nv)
    nbr = idx[q[0], q[1], q[2]] + 1                                # 1-based
    nbr_ptr = 1 + nv * np.arange(n + 1)
    g = Graph(n=n, nbr_ptr=nbr_ptr.astype(np.int32), nbr=nbr.reshape(-1).astype(np.int32))
    return g, coord, bvec


def periodic_graph(kind: str, l: int):
    """Nearest-neighbour periodic graph (src/asr_lattices.f90:166-197)."""
    vec = {"sc": [(2 * j if a == i else 0 for a in range(3)) for i in range(3) for j in (-1, 1)],
           "bcc": [(i, j, k) for i in (-1, 1) for j in (-1, 1) for k in (-1, 1)],
           "fcc": sum([[(i, j, 0), (i, 0, j), (0, i, j)] for i in (-1, 1) for j in (-1, 1)], [])}[kind]
    bvec = np.asarray([tuple(v) for v in vec], dtype=np.int64).T
    m = 2 * l
    coord, idx = _sites(kind, m)
    n = coord.shape[1]
    q = (coord[:, :, None] + bvec[:, None, :]) % m
    nbr = idx[q[0], q[1], q[2]] + 1
    nv = bvec.shape[1]
    return Graph(n=n, nbr_ptr=(1 + nv * np.arange(n + 1)).astype(np.int32), nbr=nbr.reshape(-1).astype(np.int32)), coord


_AX = np.array([[1, 2, 3], [1, 3, 2], [2, 1, 3], [2, 3, 1], [3, 1, 2], [3, 2, 1]], dtype=np.int64)


def cubic_site_perms(coord: np.ndarray, m: int):
    """perm (n, 48) Fortran order, 1-based; mats (3, 3, 48): the signed axis permutations about the origin site."""
    n = coord.shape[1]
    idx = -np.ones((m, m, m), dtype=np.int64)
    idx[coord[0], coord[1], coord[2]] = np.arange(n)
    perm = np.zeros((n, 48), dtype=np.int32, order="F")
    mats = np.zeros((3, 3, 48), dtype=np.int64, order="F")
    iop = 0
    for ip in range(6):
        pp = _AX[ip] - 1
        for is_ in range(8):
            sg = np.array([1 - 2 * (is_ & 1), 1 - 2 * ((is_ >> 1) & 1), 1 - 2 * ((is_ >> 2) & 1)], dtype=np.int64)
            for i in range(3):
                mats[i, pp[i], iop] = sg[i]
            q = np.stack([(sg[a] * coord[pp[a]]) % m for a in range(3)])
            img = idx[q[0], q[1], q[2]]
            if np.any(img < 0):
                raise ValueError("cubic_site_perms: image is not a lattice site")
            perm[:, iop] = img + 1
            iop += 1
    return perm, mats


def class_ops(coord: np.ndarray, m: int, cls: np.ndarray):
    """Class-preserving D4h operations (identity first), src/asr_symmetry.f90:67-92."""
    p48, m48 = cubic_site_perms(coord, m)
    cls = np.asarray(cls)
    keep = [bool(np.all(cls[p48[:, k] - 1] == cls)) and abs(m48[2, 2, k]) == 1 for k in range(48)]
    if not keep[0]:
        raise ValueError("class_ops: the identity does not preserve the classes")
    sel = [k for k in range(48) if keep[k]]
    return np.asfortranarray(p48[:, sel]), np.asfortranarray(m48[:, :, sel])


def d2h_ops(coord: np.ndarray, m: int, cls: np.ndarray):
    """The diagonal (D2h) operations of the class-preserving cubic group, identity first (src/asr_class_scf.f90:1613-1619)."""
    p48, m48 = cubic_site_perms(coord, m)
    cls = np.asarray(cls)
    sel = [k for k in range(48) if bool(np.all(cls[p48[:, k] - 1] == cls))
           and all(abs(m48[i, i, k]) == 1 for i in range(3))]
    return np.asfortranarray(p48[:, sel]), np.asfortranarray(m48[:, :, sel])


def identity_group(n: int):
    """The group of the identity alone: the unreduced operator."""
    perm = np.asfortranarray(np.arange(1, n + 1, dtype=np.int32).reshape(n, 1))
    d = np.asfortranarray(np.eye(9).reshape(9, 9, 1))
    return perm, d


def ylm_real(x: float, y: float, z: float) -> np.ndarray:
    """Real orthonormal harmonics l <= 2 in the order s | y z x | xy yz 3z2-r2 xz x2-y2 (src/asr_harmonics.f90:18-60)."""
    lmax = 2
    r = np.sqrt(x * x + y * y + z * z)
    ct = z / r
    st = np.sqrt(max(0.0, 1.0 - ct * ct))
    phi = np.arctan2(y, x)
    p = np.zeros((lmax + 1, lmax + 1))
    p[0, 0] = 1.0
    for mm in range(1, lmax + 1):
        p[mm, mm] = p[mm - 1, mm - 1] * (2 * mm - 1) * st
    for mm in range(0, lmax):
        p[mm + 1, mm] = ct * (2 * mm + 1) * p[mm, mm]
    for mm in range(0, lmax + 1):
        for ll in range(mm + 2, lmax + 1):
            p[ll, mm] = (ct * (2 * ll - 1) * p[ll - 1, mm] - (ll + mm - 1) * p[ll - 2, mm]) / (ll - mm)
    yl = np.zeros((lmax + 1) ** 2)
    for ll in range(lmax + 1):
        for mm in range(ll + 1):
            fr = 1.0
            for k in range(ll - mm + 1, ll + mm + 1):
                fr /= k
            nrm = np.sqrt((2 * ll + 1) / (4.0 * np.pi) * fr)
            if mm == 0:
                yl[ll * ll + ll] = nrm * p[ll, 0]
            else:
                yl[ll * ll + ll + mm] = np.sqrt(2.0) * nrm * p[ll, mm] * np.cos(mm * phi)
                yl[ll * ll + ll - mm] = np.sqrt(2.0) * nrm * p[ll, mm] * np.sin(mm * phi)
    return yl


def orbital_rep(mats: np.ndarray) -> np.ndarray:
    """d(9, 9, nop), Y_k(M p) = sum_j d(k, j) Y_j(p), fitted on a fixed Weyl sequence and rounded near integers
    (src/asr_symmetry.f90:100-129)."""
    npt = 24
    wq = np.array([0.414213562373095, 0.732050807568877, 0.236067977499790])
    pts = np.zeros((3, npt))
    a = np.zeros((npt, 9))
    for ip in range(npt):
        v = (ip + 1) * wq
        v = v - np.trunc(v) - 0.5
        pts[:, ip] = v
        a[ip, :] = ylm_real(*v)
    ata = a.T @ a
    nop = mats.shape[2]
    d = np.zeros((9, 9, nop), order="F")
    for iop in range(nop):
        b = np.zeros((npt, 9))
        for ip in range(npt):
            mp = mats[:, :, iop].astype(float) @ pts[:, ip]
            b[ip, :] = ylm_real(*mp)
        x = np.linalg.solve(ata, a.T @ b)
        dd = x.T.copy()
        near = np.abs(dd - np.rint(dd)) < 1.0e-9
        dd[near] = np.rint(dd[near])
        d[:, :, iop] = dd
    return d
