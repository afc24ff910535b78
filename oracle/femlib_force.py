"""CPU restatement of femlib's force-driven coarsening (test infrastructure only).

Only tests/ import this module.  It restates, in numpy / scipy on small cells,
the path behind NumericalCoarsening::computeCoarsenedElasticityTensorAndParameters3D
(SamplesGenerator/NumericalCoarsening.cpp:266-340):

* the vertex mesh of ElementRegGrid: (nx+1)(ny+1)(nz+1) vertices, spacing
  1 / max(nx, ny, nz) (femlib/src/ElementRegGrid.cpp:107-160), one material
  index per element;
* the assembled stiffness with every diagonal entry scaled by 1 + 1e-5
  (NumericalCoarsening.cpp:1238-1296; optional here, ``regularize``);
* multiplier rows fixing the summed displacement and the summed moment about
  the centre (femlib/src/EMeshStiffness.cpp:53-140) and making the jump between
  every pair of opposite face vertices equal to the corner jump (:142-274);
* the six unit face-force loads -- three normal, three shear pairs
  (NumericalCoarsening.cpp:756-794 and 941-988: each face element spreads a
  quarter of f / (face elements) onto its four face vertices, -f on the low
  face, +f on the high face);
* the coarse strain at the centre of the cell-sized hex of the eight corner
  vertices, and the tensor C = G^-T (sum_e sum_q w_q Gv^T E Gv / nelem) G^-1
  whose strain columns hold tensor shear strains and E is StrainLin::EMatrix
  (femlib/src/MeshUtilities.cpp:960-1060 and computeStrains; femlib/src/StrainLin.cpp:39-58);
* the parameters (rho, Y, nu, G) (NumericalCoarsening.cpp:300-339,
  Utilities/src/cfgMaterialUtilities.cpp:595-640, 660-671).

The reference's own solver for this path (PARDISO) is absent, so these values
were never compared with outputs of the reference itself: the restatement
follows its formulation step by step, and ``tensor_from_fields`` is the
independent second route (the same tensor from strain-driven fields) that the
engine uses.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import oracle as _oracle

_G = 1.0 / np.sqrt(3.0)
_SIGNS = np.array([[(a >> 2) & 1, (a >> 1) & 1, a & 1] for a in range(8)], dtype=float) * 2.0 - 1.0
_TENSOR_SHEAR = np.array([1.0, 1.0, 1.0, 0.5, 0.5, 0.5])
# load cases of computeHarmonicDisplacements (NumericalCoarsening.cpp:1152)
FORCES = ((1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0), (0.5, 0.5, 0.0), (0.0, 0.5, 0.5), (0.5, 0.0, 0.5))


def iso_matrix(E: float, nu: float) -> np.ndarray:
    """Engineering-Voigt isotropic matrix (xx, yy, zz, yz, xz, xy)."""
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[np.arange(3), np.arange(3)] += 2 * mu
    D[3, 3] = D[4, 4] = D[5, 5] = mu
    return D


def b_matrices(h: float) -> np.ndarray:
    """B[q, 6, 24]: engineering strains at the 2x2x2 Gauss points of a cube of
    edge h; local vertex a = 4ax + 2ay + az, DOFs interleaved xyz."""
    B = np.zeros((8, 6, 24))
    for q in range(8):
        xi = _SIGNS[q] * _G
        for a in range(8):
            s = _SIGNS[a]
            dN = np.empty(3)
            for d in range(3):
                v = s[d] / 8.0
                for e in range(3):
                    if e != d:
                        v *= 1.0 + s[e] * xi[e]
                dN[d] = 2.0 * v / h
            B[q, 0, 3 * a] = dN[0]
            B[q, 1, 3 * a + 1] = dN[1]
            B[q, 2, 3 * a + 2] = dN[2]
            B[q, 3, 3 * a + 1], B[q, 3, 3 * a + 2] = dN[2], dN[1]
            B[q, 4, 3 * a], B[q, 4, 3 * a + 2] = dN[2], dN[0]
            B[q, 5, 3 * a], B[q, 5, 3 * a + 1] = dN[1], dN[0]
    return B


def _elements(n):
    nx, ny, nz = n
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    return i.ravel(), j.ravel(), k.ravel()   # element (i*ny + j)*nz + k


def harmonic_displacements(mats, n, E, nu: float, regularize: bool = True, force: float = 1.0):
    """Solve femlib's multiplier system for the six face-force loads.

    mats: material index per element, voxel-major (i*ny + j)*nz + k; E[m]:
    Young's modulus of material m.  Returns (u[6, nv, 3], X[nv, 3], n)."""
    nx, ny, nz = n
    dx = 1.0 / max(n)
    Vx, Vy, Vz = nx + 1, ny + 1, nz + 1
    nv = Vx * Vy * Vz

    def vid(i, j, k):
        return (i * Vy + j) * Vz + k

    vi, vj, vk = np.meshgrid(np.arange(Vx), np.arange(Vy), np.arange(Vz), indexing="ij")
    X = np.stack([vi.ravel(), vj.ravel(), vk.ravel()], axis=1) * dx
    B = b_matrices(dx)
    K0 = sum(dx ** 3 / 8.0 * B[q].T @ iso_matrix(1.0, nu) @ B[q] for q in range(8))
    ei, ej, ek = _elements(n)
    E = np.asarray(E, dtype=float)
    kc = E[np.asarray(mats).ravel()]
    dofs = np.empty((ei.size, 24), dtype=np.int64)
    for a in range(8):
        ax, ay, az = (a >> 2) & 1, (a >> 1) & 1, a & 1
        v = vid(ei + ax, ej + ay, ek + az)
        for c in range(3):
            dofs[:, 3 * a + c] = 3 * v + c
    rows = np.repeat(dofs, 24, axis=1).ravel()
    cols = np.tile(dofs, (1, 24)).ravel()
    vals = (kc[:, None, None] * K0[None]).ravel()
    K = sp.csr_matrix((vals, (rows, cols)), shape=(3 * nv, 3 * nv))
    if regularize:
        K = K + sp.diags(1e-5 * K.diagonal())
    # multiplier rows
    crow, ccol, cval = [], [], []
    nr = 0

    def add(entries):
        nonlocal nr
        for col, val in entries:
            crow.append(nr)
            ccol.append(col)
            cval.append(val)
        nr += 1

    for c in range(3):   # summed displacement
        add([(3 * v + c, 1.0) for v in range(nv)])
    rel = X - X.mean(axis=0)
    for c in range(3):   # summed moment (rel x u)_c
        c1, c2 = (c + 1) % 3, (c + 2) % 3
        add([(3 * v + c2, rel[v, c1]) for v in range(nv)] + [(3 * v + c1, -rel[v, c2]) for v in range(nv)])
    o = vid(0, 0, 0)
    for axis in range(3):
        corner = vid(*[(Vx - 1, Vy - 1, Vz - 1)[d] if d == axis else 0 for d in range(3)])
        ranges = {0: [range(Vy), range(Vz)], 1: [range(Vx - 1), range(Vz)], 2: [range(Vx - 1), range(Vy - 1)]}[axis]
        for p in ranges[0]:
            for q in ranges[1]:
                if p == 0 and q == 0:
                    continue
                lo = [p, q]
                lo.insert(axis, 0)
                hi = list(lo)
                hi[axis] = (Vx - 1, Vy - 1, Vz - 1)[axis]
                for c in range(3):
                    add([(3 * vid(*hi) + c, 1.0), (3 * vid(*lo) + c, -1.0), (3 * corner + c, -1.0), (3 * o + c, 1.0)])
    Bc = sp.csr_matrix((cval, (crow, ccol)), shape=(nr, 3 * nv))
    KKT = sp.bmat([[K, Bc.T], [Bc, None]], format="csc")
    lu = spla.splu(KKT)
    us = []
    for fx, fy, fz in FORCES:
        f = np.zeros(3 * nv + nr)
        parts = []
        if fy == 0 and fz == 0:
            parts = [(0, (fx, 0, 0))]
        elif fx == 0 and fz == 0:
            parts = [(1, (0, fy, 0))]
        elif fx == 0 and fy == 0:
            parts = [(2, (0, 0, fz))]
        elif fz == 0:
            parts = [(1, (fx, 0, 0)), (0, (0, fy, 0))]
        elif fy == 0:
            parts = [(2, (fx, 0, 0)), (0, (0, 0, fz))]
        else:
            parts = [(2, (0, fy, 0)), (1, (0, 0, fz))]
        for axis, fv in parts:
            nb = [nx, ny, nz]
            nb.pop(axis)
            coeff = force / (nb[0] * nb[1]) / 4.0
            for side, sign in ((0, -1.0), (1, 1.0)):
                # every element on the face spreads coeff * fv onto its 4 face vertices
                for p in range(nb[0]):
                    for q in range(nb[1]):
                        for dp in (0, 1):
                            for dq in (0, 1):
                                ijk = [p + dp, q + dq]
                                ijk.insert(axis, side * (nx, ny, nz)[axis])
                                v = vid(*ijk)
                                for c in range(3):
                                    f[3 * v + c] += sign * coeff * fv[c]
        us.append(lu.solve(f)[:3 * nv].reshape(nv, 3))
    return np.array(us), X, (nx, ny, nz)


def coarse_strain(u, X, n) -> np.ndarray:
    """Tensor strain (3x3) at the centre of the hex of the cell's 8 corners."""
    nx, ny, nz = n
    Vy, Vz = ny + 1, nz + 1
    L = np.array([nx, ny, nz]) / max(n)
    grad = np.zeros((3, 3))
    for a in range(8):
        s = _SIGNS[a]
        v = (((a >> 2) & 1) * nx * Vy + ((a >> 1) & 1) * ny) * Vz + (a & 1) * nz
        grad += np.outer(u[v], s / (4.0 * L))
    return 0.5 * (grad + grad.T)


def _voigt_t(eps):
    return np.array([eps[0, 0], eps[1, 1], eps[2, 2], eps[1, 2], eps[0, 2], eps[0, 1]])


def femlib_tensor(us, X, n, mats, E, nu: float) -> np.ndarray:
    """C = G^-T (sum_e sum_q w_q Gv^T E_e Gv / nelem) G^-1, tensor-shear columns."""
    nx, ny, nz = n
    dx = 1.0 / max(n)
    Vy, Vz = ny + 1, nz + 1
    G = np.stack([_voigt_t(coarse_strain(u, X, n)) for u in us], axis=1)
    B = b_matrices(dx) * _TENSOR_SHEAR[None, :, None]   # tensor-shear local strains
    ei, ej, ek = _elements(n)
    E = np.asarray(E, dtype=float)
    kc = E[np.asarray(mats).ravel()]
    idx = np.empty((ei.size, 8), dtype=np.int64)
    for a in range(8):
        idx[:, a] = ((ei + ((a >> 2) & 1)) * Vy + ej + ((a >> 1) & 1)) * Vz + ek + (a & 1)
    ue = np.stack([u[idx].reshape(ei.size, 24) for u in us], axis=2)   # [e, 24, 6]
    D = iso_matrix(1.0, nu)
    acc = np.zeros((6, 6))
    for q in range(8):
        Gv = np.einsum("sk,ekd->esd", B[q], ue)
        acc += 0.125 * np.einsum("e,esd,st,etf->df", kc, Gv, D, Gv)
    Gi = np.linalg.inv(G)
    return Gi.T @ (acc / ei.size) @ Gi


def parameters(us, X, n, C, mats_in, dens, cubic: bool = True):
    """(rho, Y.., nu_xy[, nu_xz, nu_yz], G..) from the harmonic displacements."""
    strains = [_voigt_t(coarse_strain(u, X, n)) for u in us]
    r = float(np.mean([dens[m] for m in np.ravel(mats_in)]))
    naxis = 1 if cubic else 3
    out = [r] + [1.0 / strains[a][a] for a in range(naxis)]   # force magnitude 1
    out.append(-strains[0][1] / strains[0][0])
    if not cubic:
        out += [-strains[0][2] / strains[0][0], -strains[1][2] / strains[1][1]]
    out += [C[3 + i, 3 + i] for i in range(naxis)]
    return np.array(out)


def coarsen(mats, n, E, nu, mats_in=None, dens=(0.0, 1.0), cubic=True, regularize=True):
    """femlib's outputs for one structure: (C[6,6], 21 lower-triangle values, parameters)."""
    us, X, n = harmonic_displacements(mats, n, E, nu, regularize=regularize)
    C = femlib_tensor(us, X, n, mats, E, nu)
    tv = np.array([C[i, j] for i in range(6) for j in range(i + 1)])
    pv = parameters(us, X, n, C, mats if mats_in is None else mats_in, dens, cubic)
    return C, tv, pv


def tensor_from_fields(mats, n, E, nu: float, chi=None) -> np.ndarray:
    """The same tensor from the six strain-driven fields u^I = eps^I x + chi^I
    (unit engineering strains, periodic chi from the oracle's solve when not
    given): S W' S with W'_IJ the cell average of eps(u^I).(S_t E S_t) eps(u^J),
    S_t = diag(1,1,1,1/2,1/2,1/2), S = diag(1,1,1,2,2,2).  Equal to
    ``femlib_tensor`` of the multiplier solve on cubic cells; on other cells
    femlib's shear face loads are out of moment balance and the two differ."""
    nx, ny, nz = n
    dx = 1.0 / max(n)
    E = np.asarray(E, dtype=float)
    mats = np.asarray(mats).reshape(n)
    if chi is None:
        rho = (mats == 1).astype(float)
        mat = _oracle.material(interp=_oracle.INTERP_BINARY, nu=nu, bin_hi=E[1], bin_lo=E[0])
        _, chi, _, rel, _ = _oracle.homogenize(rho, h=dx, mat=mat, tol=1e-13, max_iter=200000)
    B = b_matrices(dx)
    ei, ej, ek = _elements(n)
    kc = E[mats.ravel()]
    ue = np.zeros((ei.size, 24, 6))
    for I in range(6):
        eps = np.zeros((3, 3))
        if I < 3:
            eps[I, I] = 1.0
        else:
            a, b = {3: (1, 2), 4: (0, 2), 5: (0, 1)}[I]
            eps[a, b] = eps[b, a] = 0.5
        for a8 in range(8):
            ax, ay, az = (a8 >> 2) & 1, (a8 >> 1) & 1, a8 & 1
            x = np.stack([(ei + ax) * dx, (ej + ay) * dx, (ek + az) * dx], axis=1)
            per = chi[I][(ei + ax) % nx, (ej + ay) % ny, (ek + az) % nz]
            ue[:, 3 * a8:3 * a8 + 3, I] = x @ eps.T + per
    Dp = iso_matrix(1.0, nu) * np.outer(_TENSOR_SHEAR, _TENSOR_SHEAR)
    W = np.zeros((6, 6))
    for q in range(8):
        ge = np.einsum("sk,ekd->esd", B[q], ue)
        W += 0.125 * np.einsum("e,esd,st,etf->df", kc, ge, Dp, ge)
    W /= ei.size
    S = np.diag(1.0 / _TENSOR_SHEAR)
    return S @ W @ S
