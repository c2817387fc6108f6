"""FP64 CPU oracle for tetmag's effective-field + LLG right-hand-side path.

TEST INFRASTRUCTURE ONLY.  This module is the checker: tests/, the smoke test
and the CPU-baseline leg of bench.py may import it; the product (the
``tetmag_b200`` package and its CUDA library) never does.

It restates, in numpy/scipy, the algorithms of the reference (R-Hertel/tetmag
v1.7.7) that produce the field and the LLG right-hand side:

* P1 FEM preprocessing        preproc/FEMprocessing.cpp:104-286, 329-369
* boundary extraction         preproc/Boundary.cpp:47-224
* solid angles, dense BEM     preproc/BEMprocessing.cpp:358-411,
                              preproc/Lindholm.cpp:41-128
* local fields                main/EffFieldCalc.cpp:59-170, 280-298
* total field and LLG         main/TheLLG.cpp:150-199, 238-254, 426-449
* demag (Fredkin-Koehler)     main/DemagField.cpp:92-240
* units                       specs/SimulationData.cpp:45-57,
                              utils/PhysicalConstants.h:39-43

The reference cannot be built in this environment (Eigen, Boost, VTK,
SUNDIALS, AMGCL and H2Lib are absent), so no golden output of the reference
binary exists.  The oracle is pinned against the reference's own built-in
known-answer checks: the dense BEM row-sum test B.(-1) summed equals Nb
within 5e-3 (preproc/BEMprocessing.cpp:55-72, 440-445) and the exactness of
the nodal gradient operators on linear functions to 1e-10
(preproc/FEMprocessing.cpp:288-326); plus analytic identities (demag factors
of a uniformly magnetised prism).  Field-level parity with the reference
binary, and the AMGCL / H2Lib / CVODE iteration-level behaviour, are
unpinned.

Linear solves are direct (SuperLU on the reference's own row-pinned
matrices), the analogue of the reference's default ``solver type = LU``
(main/SolverFactory.cpp:78-93).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

# utils/PhysicalConstants.h:37-43
PI = np.pi
MU0 = 1.256637061435917295376e-6
GAMMA0 = 221276.14886372426114160400
EPS = np.finfo(np.float64).eps


# --------------------------------------------------------------------------------------
# FEM preprocessing  (preproc/FEMprocessing.cpp)
# --------------------------------------------------------------------------------------
@dataclass
class FEM:
    nx: int
    elem_vol: np.ndarray          # (E,)
    node_vol: np.ndarray          # (N,)
    sgrad: np.ndarray             # (E, 4, 3) shape-function gradients
    stiff: sp.csr_matrix          # K
    grad: list                    # [gradX, gradY, gradZ]  (volume-averaged nodal gradient)
    tgrad: list                   # [tGradX, tGradY, tGradZ] (weak divergence)


def _det3(m):
    """3x3 determinants by cofactor expansion (Eigen's fixed-size path)."""
    return (m[..., 0, 0] * (m[..., 1, 1] * m[..., 2, 2] - m[..., 1, 2] * m[..., 2, 1])
            - m[..., 0, 1] * (m[..., 1, 0] * m[..., 2, 2] - m[..., 1, 2] * m[..., 2, 0])
            + m[..., 0, 2] * (m[..., 1, 0] * m[..., 2, 1] - m[..., 1, 1] * m[..., 2, 0]))


def signed_volume6(p):
    """det([[1,p1],[1,p2],[1,p3],[1,p4]]) -- FEMprocessing.cpp:115-123, 141-150."""
    a = p[:, 1] - p[:, 0]
    b = p[:, 2] - p[:, 0]
    c = p[:, 3] - p[:, 0]
    return np.einsum("ij,ij->i", a, np.cross(b, c))


def fem_prepare(xyz: np.ndarray, tets: np.ndarray) -> FEM:
    """Volumes, shape gradients, grad/tGrad operators and stiffness matrix.

    Restates PreprocessMesh::calculateVolumes (:104-113), calcShapeFuncGrads
    (:153-195), calculateGradientOperators (:228-253) and
    assembleStiffnessMatrix (:266-286).  All seven matrices are assembled over
    every (local_i, local_j) node pair of every element, so they share one
    sparsity pattern (explicit zeros kept, as Eigen's coeffRef inserts them).
    """
    xyz = np.asarray(xyz, dtype=np.float64)
    tets = np.asarray(tets, dtype=np.int64)
    n = xyz.shape[0]
    p = xyz[tets]                                   # (E,4,3)
    V6 = signed_volume6(p)
    vol = np.abs(V6) / 6.0
    node_vol = np.bincount(tets.ravel(), weights=np.repeat(vol / 4.0, 4), minlength=n)

    sgrad = np.empty((tets.shape[0], 4, 3))
    for nn in range(4):
        node_mat = p[:, [(nn + 1) % 4, (nn + 2) % 4, (nn + 3) % 4], :].copy()  # rows: other nodes
        sign = (-1.0) ** (nn + 1)
        for d in range(3):
            gm = node_mat.copy()
            gm[:, :, d] = 1.0
            sgrad[:, nn, d] = sign * _det3(gm) / V6

    li, lj = np.meshgrid(np.arange(4), np.arange(4), indexing="ij")
    li, lj = li.ravel(), lj.ravel()
    gi = tets[:, li].ravel()
    gj = tets[:, lj].ravel()
    w = np.repeat(vol / 4.0, 16)
    shape = (n, n)

    def assemble(vals):
        m = sp.coo_matrix((vals, (gi, gj)), shape=shape).tocsr()
        m.sum_duplicates()
        m.sort_indices()
        return m

    grad, tgrad = [], []
    for d in range(3):
        bj = sgrad[:, lj, d].ravel()
        bi = sgrad[:, li, d].ravel()
        grad.append(assemble(bj * w / node_vol[gi]))
        tgrad.append(assemble(bi * w))
    kval = (np.einsum("eid,ejd->eij", sgrad, sgrad) * vol[:, None, None]).reshape(-1)
    stiff = assemble(kval)
    return FEM(nx=n, elem_vol=vol, node_vol=node_vol, sgrad=sgrad, stiff=stiff,
               grad=grad, tgrad=tgrad)


# --------------------------------------------------------------------------------------
# Boundary  (preproc/Boundary.cpp)
# --------------------------------------------------------------------------------------
@dataclass
class Boundary:
    tri: np.ndarray            # (T,3) global node ids, ascending within a triangle
    tri_tet: np.ndarray        # (T,) owning tetrahedron
    tri_area: np.ndarray       # (T,)
    tri_normal: np.ndarray     # (T,3) outward unit normal
    bnodes: np.ndarray         # (Nb,) ascending global ids
    bindex: np.ndarray         # (N,) boundary index or -1
    node_area: np.ndarray      # (N,) 1/3 of adjacent boundary-triangle areas
    node_normal: np.ndarray    # (N,3) area-weighted, normalised, 0 off the boundary


def triangle_area(p0, p1, p2):
    """auxiliaries.cpp:63-68."""
    return 0.5 * np.linalg.norm(np.cross(p0 - p1, p0 - p2), axis=-1)


def triangle_unit_normal(p0, p1, p2):
    """auxiliaries.cpp:71-76."""
    c = np.cross(p0 - p1, p0 - p2)
    return c / np.linalg.norm(c, axis=-1, keepdims=True)


def extract_boundary(xyz: np.ndarray, tets: np.ndarray) -> Boundary:
    """MeshBoundary::extractFeatures (Boundary.cpp:47-55).

    Faces are the sorted node triples of each tet (findBoundaryElements,
    :159-197); a face that occurs once is a boundary triangle.  The outward
    normal points away from the owning tet's centre (:109-125); node areas
    (:214-224) and node normals (:78-89) are accumulated from the triangles.
    """
    tets = np.asarray(tets, dtype=np.int64)
    n = xyz.shape[0]
    faces = []
    for j in range(4):
        others = [k for k in range(4) if k != j]
        faces.append(np.sort(tets[:, others], axis=1))
    faces = np.stack(faces, axis=1).reshape(-1, 3)
    owner = np.repeat(np.arange(tets.shape[0]), 4)
    key = (faces[:, 0] * n + faces[:, 1]) * n + faces[:, 2] if n < 2 ** 21 else None
    if key is not None:
        _, inv, cnt = np.unique(key, return_inverse=True, return_counts=True)
    else:
        _, inv, cnt = np.unique(faces, axis=0, return_inverse=True, return_counts=True)
    once = cnt[inv.ravel()] == 1
    tri = faces[once]
    tri_tet = owner[once]
    p0, p1, p2 = xyz[tri[:, 0]], xyz[tri[:, 1]], xyz[tri[:, 2]]
    area = triangle_area(p0, p1, p2)
    nrm = triangle_unit_normal(p0, p1, p2)
    centre = xyz[tets[tri_tet]].mean(axis=1)
    s = np.sign(np.einsum("ij,ij->i", nrm, centre - p0))
    nrm = -nrm * s[:, None]

    bnodes = np.unique(tri.ravel())
    bindex = -np.ones(n, dtype=np.int64)
    bindex[bnodes] = np.arange(bnodes.size)
    node_area = np.bincount(tri.ravel(), weights=np.repeat(area / 3.0, 3), minlength=n)
    nv = np.zeros((n, 3))
    for d in range(3):
        nv[:, d] = np.bincount(tri.ravel(), weights=np.repeat(nrm[:, d] * area / 3.0, 3), minlength=n)
    with np.errstate(invalid="ignore", divide="ignore"):
        nv = nv / np.linalg.norm(nv, axis=1, keepdims=True)
    nv[~np.isfinite(nv)] = 0.0
    return Boundary(tri=tri, tri_tet=tri_tet, tri_area=area, tri_normal=nrm, bnodes=bnodes,
                    bindex=bindex, node_area=node_area, node_normal=nv)


# --------------------------------------------------------------------------------------
# Solid angles and Lindholm double-layer BEM  (preproc/Lindholm.cpp, BEMprocessing.cpp)
# --------------------------------------------------------------------------------------
def _are_equal(x, y, ulp=100):
    """auxiliaries.cpp:42-47."""
    close = np.abs(x - y) < EPS * np.abs(x + y) * ulp
    zero = (np.abs(x) < EPS * ulp) & (np.abs(y) < EPS * ulp)
    return close | zero


def solid_angle(x, t1, t2, t3):
    """Lindholm::solidAngle (Lindholm.cpp:41-61), vectorised over leading axes."""
    r1, r2, r3 = t1 - x, t2 - x, t3 - x
    r1n = np.linalg.norm(r1, axis=-1)
    r2n = np.linalg.norm(r2, axis=-1)
    r3n = np.linalg.norm(r3, axis=-1)
    r123 = r1n * r2n * r3n
    r23 = np.sum(r2 * r3, axis=-1)
    r12 = np.sum(r1 * r2, axis=-1)
    r31 = np.sum(r3 * r1, axis=-1)
    numer = r123 + r1n * r23 + r2n * r31 + r3n * r12
    denom = np.sqrt(2.0 * (r2n * r3n + r23) * (r3n * r1n + r31) * (r1n * r2n + r12))
    arg = numer / denom
    arg = np.where(_are_equal(arg, 1.0), 1.0, arg)
    return 2.0 * np.arccos(arg)


def solid_angles(xyz, tets, bnd: Boundary) -> np.ndarray:
    """BEMprocessing::calculateSolidAngles (:358-372): interior solid angle per boundary node."""
    tets = np.asarray(tets, dtype=np.int64)
    sub = np.zeros(bnd.bnodes.size)
    for j in range(4):
        node = tets[:, j]
        isb = bnd.bindex[node] >= 0
        P = xyz[node[isb]]
        T1 = xyz[tets[isb, (j + 1) % 4]]
        T2 = xyz[tets[isb, (j + 2) % 4]]
        T3 = xyz[tets[isb, (j + 3) % 4]]
        np.add.at(sub, bnd.bindex[node[isb]], solid_angle(P, T1, T2, T3))
    return sub


def lindholm_weights(x0, p0, p1, p2, area, nv):
    """Lindholm::weights with isOrdered = false (Lindholm.cpp:64-128).

    x0: (M,3) observation points; p*: (M,3) triangle vertices; area (M,);
    nv (M,3) outward normal.  Returns (M,3) weights for the three vertices.
    Implements D.A. Lindholm, IEEE Trans. Magn. 20, 2025 (1984).
    """
    p = np.stack([p0, p1, p2], axis=1)                  # (M,3vert,3)
    chi = triangle_unit_normal(p0, p1, p2)               # (M,3)
    rho_vec = p - x0[:, None, :]
    xi = np.roll(rho_vec, -1, axis=1) - rho_vec          # xi_i = rho_{i+1} - rho_i
    s = np.linalg.norm(xi, axis=-1)                      # (M,3)
    xi = xi / s[..., None]
    eta = np.cross(chi[:, None, :], xi)
    eta0 = np.sum(eta * rho_vec, axis=-1)
    rho = np.linalg.norm(rho_vec, axis=-1)
    chi0 = np.sum(chi * rho_vec[:, 0, :], axis=-1)
    # gamma(i,j) = xi_{(i+1)%3} . xi_j
    gamma = np.einsum("mid,mjd->mij", np.roll(xi, -1, axis=1), xi)
    rs = rho + np.roll(rho, -1, axis=1)
    P = np.log((rs + s) / (rs - s))
    omega = solid_angle(x0, p0, p1, p2)
    omega = np.where(chi0 < 0.0, -omega, omega)
    gP = np.einsum("mij,mj->mi", gamma, P)
    s1 = np.roll(s, -1, axis=1)
    eta01 = np.roll(eta0, -1, axis=1)
    L = s1 / (8.0 * PI * area[:, None]) * (eta01 * omega[:, None] - chi0[:, None] * gP)
    flip = np.sum(nv * chi, axis=-1) < 0.0
    L[flip] = -L[flip]
    return L


def lindholm_weights_accurate(x0, p0, p1, p2, area, nv):
    """The weights of ``lindholm_weights`` in a far-field-accurate arithmetic (the form the
    device uses for the low-rank blocks of its hierarchical matrix; not a reference function).

    The solid angle is 2 atan2(N, D) with N = |e01 x e02| chi0 (Van Oosterom & Strackee,
    IEEE Trans. Biomed. Eng. 30, 125 (1983)) instead of 2 acos(arg), edges are vertex
    differences and the edge logarithms use log1p, so that the cancellation of the two terms of
    a weight (about r / h) works on full-precision inputs.
    """
    p = np.stack([p0, p1, p2], axis=1)
    e = np.roll(p, -1, axis=1) - p                       # edges p_{i+1} - p_i
    c = np.cross(p1 - p0, p2 - p0)
    cn = np.linalg.norm(c, axis=-1)
    chi = c / cn[:, None]
    s = np.linalg.norm(e, axis=-1)
    xi = e / s[..., None]
    rv = p - x0[:, None, :]
    rho = np.linalg.norm(rv, axis=-1)
    chi0 = np.sum(chi * rv[:, 0, :], axis=-1)
    d01 = np.sum(rv[:, 0] * rv[:, 1], -1)
    d02 = np.sum(rv[:, 0] * rv[:, 2], -1)
    d12 = np.sum(rv[:, 1] * rv[:, 2], -1)
    D = rho[:, 0] * rho[:, 1] * rho[:, 2] + d01 * rho[:, 2] + d02 * rho[:, 1] + d12 * rho[:, 0]
    omega = 2.0 * np.arctan2(cn * chi0, D)
    P = np.log1p(2.0 * s / (rho + np.roll(rho, -1, axis=1) - s))
    eta0 = np.sum(np.cross(chi[:, None, :], xi) * rv, axis=-1)
    gamma = np.einsum("mid,mjd->mij", np.roll(xi, -1, axis=1), xi)
    gP = np.einsum("mij,mj->mi", gamma, P)
    L = np.roll(s, -1, axis=1) / (8.0 * PI * area[:, None]) * (np.roll(eta0, -1, axis=1) * omega[:, None]
                                                             - chi0[:, None] * gP)
    flip = np.sum(nv * chi, axis=-1) < 0.0
    L[flip] = -L[flip]
    return L


def dense_bem(xyz, tets, bnd: Boundary, sub: Optional[np.ndarray] = None,
              rows: Optional[np.ndarray] = None, chunk_pairs: int = 2_000_000) -> np.ndarray:
    """BEMprocessing::assembleLaplaceBEMmatrix (:375-411) -> (Nb, Nb) FP64.

    Diagonal: Omega/(4 pi) - 1; off-diagonal: Lindholm weights, zero for the
    triangles that contain the observation node.  ``rows`` selects a subset of
    rows (used to bound the CPU cost on large meshes).
    """
    if sub is None:
        sub = solid_angles(xyz, tets, bnd)
    nb = bnd.bnodes.size
    rows = np.arange(nb) if rows is None else np.asarray(rows)
    B = np.zeros((rows.size, nb))
    T = bnd.tri.shape[0]
    tri_b = bnd.bindex[bnd.tri]                                  # (T,3) boundary indices
    p0, p1, p2 = xyz[bnd.tri[:, 0]], xyz[bnd.tri[:, 1]], xyz[bnd.tri[:, 2]]
    rows_per = max(1, chunk_pairs // max(T, 1))
    for r0 in range(0, rows.size, rows_per):
        rr = rows[r0:r0 + rows_per]
        R = rr.size
        x0 = np.repeat(xyz[bnd.bnodes[rr]], T, axis=0)
        L = lindholm_weights(x0, np.tile(p0, (R, 1)), np.tile(p1, (R, 1)), np.tile(p2, (R, 1)),
                             np.tile(bnd.tri_area, R), np.tile(bnd.tri_normal, (R, 1)))
        L = L.reshape(R, T, 3)
        own = (tri_b[None, :, :] == rr[:, None, None]).any(axis=2)   # triangle contains node
        L[own] = 0.0
        rloc = np.repeat(np.arange(R), T * 3)
        cols = np.tile(tri_b.ravel(), R)
        blk = np.zeros((R, nb))
        np.add.at(blk, (rloc, cols), L.ravel())
        B[r0:r0 + R] = blk
    diag = sub / (4.0 * PI) - 1.0
    B[np.arange(rows.size), rows] = diag[rows]
    return B


def bem_rowsum_error(B: np.ndarray) -> float:
    """getH2err(sum(B.(-1)), Nb) -- preproc/BEMprocessing.cpp:55-58, 440-445."""
    nb = B.shape[1]
    s = (B @ (-np.ones(nb))).sum()
    return abs((s - nb) / nb)


# --------------------------------------------------------------------------------------
# Problem: mesh + operators + material, everything the field path consumes
# --------------------------------------------------------------------------------------
@dataclass
class Problem:
    xyz: np.ndarray
    tets: np.ndarray
    scale: float
    fem: FEM
    bnd: Boundary
    B: Optional[np.ndarray]         # dense BEM (Nb, Nb) or None
    Js: np.ndarray                  # (N,) Tesla
    A: np.ndarray                   # (N,) J/m, already divided by scale^2
    Ku: np.ndarray                  # (N,) J/m^3
    ku_axis: np.ndarray             # (N,3)
    D: np.ndarray                   # (N,) J/m^2, already divided by scale
    alpha: float
    hext: np.ndarray                # (N,3) A/m
    gamma: float = GAMMA0
    dmi_kind: str = "bulk"          # "bulk" (reference) or "interfacial"
    extra: dict = field(default_factory=dict)

    @property
    def nx(self):
        return self.xyz.shape[0]

    def time_scale(self) -> float:
        """Reduced time units per ps: gamma/(1+alpha^2)*1e-12 (SimulationData.cpp:52-57)."""
        return self.gamma / (1.0 + self.alpha * self.alpha) * 1e-12


def make_problem(xyz, tets, scale, Ms, A, alpha, Ku=0.0, ku_axis=(0, 0, 1), D=0.0,
                 hext=None, with_bem=True, dmi_kind="bulk") -> Problem:
    """Per-node material vectors (SimulationData.cpp:125-163) with the length
    scaling of scaleToRealSize (:45-49): A /= s^2, D /= s."""
    fem = fem_prepare(xyz, tets)
    bnd = extract_boundary(xyz, tets)
    n = xyz.shape[0]
    B = dense_bem(xyz, tets, bnd) if with_bem else None
    axis = np.asarray(ku_axis, dtype=np.float64)
    axis = np.broadcast_to(axis / np.linalg.norm(axis, axis=-1, keepdims=True), (n, 3)).copy()
    h = np.zeros((n, 3)) if hext is None else np.asarray(hext, dtype=np.float64).reshape(3, n).T.copy()
    return Problem(xyz=np.asarray(xyz, np.float64), tets=np.asarray(tets), scale=scale, fem=fem,
                   bnd=bnd, B=B, Js=np.full(n, MU0 * Ms) if np.isscalar(Ms) else MU0 * np.asarray(Ms),
                   A=np.broadcast_to(np.asarray(A, np.float64) / scale ** 2, (n,)).copy(),
                   Ku=np.broadcast_to(np.asarray(Ku, np.float64), (n,)).copy(), ku_axis=axis,
                   D=np.broadcast_to(np.asarray(D, np.float64) / scale, (n,)).copy(),
                   alpha=float(alpha), hext=h, dmi_kind=dmi_kind)


def soa_to_rows(v):
    v = np.asarray(v, dtype=np.float64)
    n = v.size // 3
    return v.reshape(3, n).T


def rows_to_soa(m):
    return np.ascontiguousarray(np.asarray(m).T.ravel())


def cross(a, b):
    return np.cross(a, b)


# --------------------------------------------------------------------------------------
# Local fields  (main/EffFieldCalc.cpp)
# --------------------------------------------------------------------------------------
def exchange_field(pb: Problem, m):
    """EffFieldCalc::setExchangeFieldOperator/exchangeField (:59-63, 97-100): -2 diag(A/V) K m."""
    xc = sp.diags(-2.0 * pb.A / pb.fem.node_vol) @ pb.fem.stiff
    return xc @ m


def uniaxial_field(pb: Problem, m):
    """EffFieldCalc::uniaxialAnisotropyField (:71-84): 2 Ku (k.m) k."""
    km = np.sum(pb.ku_axis * m, axis=1)
    return (2.0 * pb.Ku * km)[:, None] * pb.ku_axis


def cubic_field(pb: Problem, m):
    """EffFieldCalc::cubicAnisotropyField (:249-272): alpha = C^T m (axes as columns of C),
    dE_j = -2 a_j (Kc1 (a_j+1^2 + a_j+2^2) + Kc2 a_j+1^2 a_j+2^2), H = C dE.
    pb.extra: Kc1, Kc2 (N,), cax (N, 3, 3) with the axes as rows."""
    cax = pb.extra["cax"]
    al = np.einsum("nkd,nd->nk", cax, m)
    k1, k2 = pb.extra["Kc1"], pb.extra["Kc2"]
    de = np.empty_like(al)
    for j in range(3):
        b1, b2 = al[:, (j + 1) % 3] ** 2, al[:, (j + 2) % 3] ** 2
        de[:, j] = -2.0 * al[:, j] * (k1 * (b1 + b2) + k2 * b1 * b2)
    return np.einsum("nkd,nk->nd", cax, de)


def surface_field(pb: Problem, m):
    """EffFieldCalc::surfaceAnisotropyField (:128-149) with Ksn = Ks * node area (:102-106):
    -2 Ksn nm (nm m - n) / V, nm = m . n.  pb.extra: Ks (N,)."""
    ksn = pb.extra["Ks"] * pb.bnd.node_area
    nv = pb.bnd.node_normal
    nm = np.sum(m * nv, axis=1)
    return (-2.0 * ksn * nm / pb.fem.node_vol)[:, None] * (nm[:, None] * m - nv)


def curl_m(pb: Problem, m):
    """EffFieldCalc::curlM (:280-298) with tGrad = -msh.tGrad (:43)."""
    tx, ty, tz = [-t for t in pb.fem.tgrad]
    c = np.empty_like(m)
    c[:, 0] = ty @ m[:, 2] - tz @ m[:, 1]
    c[:, 1] = tz @ m[:, 0] - tx @ m[:, 2]
    c[:, 2] = tx @ m[:, 1] - ty @ m[:, 0]
    return c


def dmi_field(pb: Problem, m):
    """Bulk DMI: EffFieldCalc::dmiField/surfIntDMI (:159-170):
    (nodeArea * (m x n) - 2 curl m) * D / V."""
    surf = pb.bnd.node_area[:, None] * np.cross(m, pb.bnd.node_normal)
    return (surf - 2.0 * curl_m(pb, m)) * (pb.D / pb.fem.node_vol)[:, None]


def interfacial_dmi_field(pb: Problem, m):
    """Interfacial DMI (not in the reference): variational derivative of
    E = sum_i V_i D_i [m_z div m - (m . grad) m_z]_i with the nodal gradient
    operators, H = -(1/V) dE/dm  (so that E = -1/2 sum V H.m per node-volume).

    The discrete energy uses g_d = grad_d (volume-averaged nodal gradient):
      e_i = mz_i (gx mx + gy my)_i - (mx_i (gx mz)_i + my_i (gy mz)_i)
    and the field is its exact negative gradient divided by the node volume.
    """
    V = pb.fem.node_vol
    w = V * pb.D
    gx, gy, _ = pb.fem.grad
    mx, my, mz = m[:, 0], m[:, 1], m[:, 2]
    dE = np.zeros_like(m)
    # d/dm of sum_i w_i mz_i (gx mx)_i
    dE[:, 2] += w * (gx @ mx + gy @ my)
    dE[:, 0] += gx.T @ (w * mz)
    dE[:, 1] += gy.T @ (w * mz)
    # d/dm of -sum_i w_i mx_i (gx mz)_i - w_i my_i (gy mz)_i
    dE[:, 0] -= w * (gx @ mz)
    dE[:, 1] -= w * (gy @ mz)
    dE[:, 2] -= gx.T @ (w * mx) + gy.T @ (w * my)
    return -dE / V[:, None]


def interfacial_dmi_energy(pb: Problem, m):
    V = pb.fem.node_vol
    gx, gy, _ = pb.fem.grad
    mx, my, mz = m[:, 0], m[:, 1], m[:, 2]
    e = mz * (gx @ mx + gy @ my) - (mx * (gx @ mz) + my * (gy @ mz))
    return float(np.sum(V * pb.D * e))


# --------------------------------------------------------------------------------------
# Demag  (main/DemagField.cpp)
# --------------------------------------------------------------------------------------
class DemagOracle:
    """DemagField with direct solves of the reference's row-pinned systems."""

    def __init__(self, pb: Problem):
        self.pb = pb
        n = pb.nx
        self.k = n // 2                                   # DemagField.cpp:80
        K = pb.fem.stiff.tolil(copy=True)
        # prepareNeumannMatrix (:204-220): row k -> e_k, prune zeros
        K.rows[self.k] = [self.k]
        K.data[self.k] = [1.0]
        neu = K.tocsr()
        neu.eliminate_zeros()
        # prepareDirichletMatrix (FEMprocessing.cpp:329-369): boundary rows -> identity
        D = pb.fem.stiff.tolil(copy=True)
        for b in pb.bnd.bnodes:
            D.rows[b] = [int(b)]
            D.data[b] = [1.0]
        dir_ = D.tocsr()
        dir_.eliminate_zeros()
        self.neumann = neu
        self.dirichlet = dir_
        self.lu_neu = spla.splu(neu.tocsc())
        self.lu_dir = spla.splu(dir_.tocsc())

    def rhs_poisson(self, m):
        """rhsPoisson (:124-136): sum_d tGrad_d (Js m_d) / mu0."""
        tg = self.pb.fem.tgrad
        Js = self.pb.Js
        return (tg[0] @ (m[:, 0] * Js) + tg[1] @ (m[:, 1] * Js) + tg[2] @ (m[:, 2] * Js)) / MU0

    def boundary_integral(self, u1):
        """boundaryIntegral (:184-201): gather, dense BEM product, scatter."""
        bn = self.pb.bnd.bnodes
        out = np.zeros(self.pb.nx)
        out[bn] = self.pb.B @ u1[bn]
        return out

    def potential(self, m):
        """calcPotential (:163-181)."""
        u1 = self.lu_neu.solve(self.rhs_poisson(m))
        u2 = self.lu_dir.solve(self.boundary_integral(u1))
        return u1 + u2, u1, u2

    def field(self, m):
        """calcField / calcGradientField (:92-113): -grad u."""
        u, _, _ = self.potential(m)
        g = self.pb.fem.grad
        return -np.stack([g[0] @ u, g[1] @ u, g[2] @ u], axis=1)

    def energy(self, m, H):
        """getDemagEnergy (:97-99)."""
        return float(-(self.pb.Js * self.pb.fem.node_vol) @ np.sum(H * m, axis=1) / 2.0)


# --------------------------------------------------------------------------------------
# Total field, LLG right-hand side, torque  (main/TheLLG.cpp)
# --------------------------------------------------------------------------------------
def inv_js(pb: Problem):
    with np.errstate(divide="ignore"):
        v = 1.0 / pb.Js
    v[~np.isfinite(v)] = 0.0
    return v


def local_field(pb: Problem, m, hdem):
    """totalEffectiveField (:238-254) with the terms this path uses."""
    h = exchange_field(pb, m)
    if np.any(pb.Ku != 0.0):
        h = h + uniaxial_field(pb, m)
    if np.any(pb.D != 0.0):
        h = h + (dmi_field(pb, m) if pb.dmi_kind == "bulk" else interfacial_dmi_field(pb, m))
    if "Kc1" in pb.extra:
        h = h + cubic_field(pb, m)
    if "Ks" in pb.extra:
        h = h + surface_field(pb, m)
    return h * inv_js(pb)[:, None] + pb.hext + hdem


def llg_rhs(pb: Problem, m, H, precession=True):
    """classicVersion / noPrecession (:150-199): -m x H - alpha m x (m x H); with pb.extra["eta"]
    ((N, 3): eta_jx, eta_jy, eta_jz) the spin-transfer term of sttDynamics (:201-220, U term
    calcUtermSTT :402-415): s [-(beta - alpha) m x U - (1 + alpha beta) m x (m x U)]."""
    mxh = np.cross(m, H)
    out = -pb.alpha * np.cross(m, mxh)
    if precession:
        out = out - mxh
    extra = getattr(pb, "extra", {})
    if "eta" in extra:
        eta, beta, s = extra["eta"], extra.get("beta", 0.0), extra.get("stt_scale", 1.0)
        g = pb.fem.grad
        U = sum(eta[:, d][:, None] * np.stack([g[d] @ m[:, c] for c in range(3)], axis=1) for d in range(3))
        mxu = np.cross(m, U)
        out = out + s * (-(beta - pb.alpha) * mxu - (1.0 + pb.alpha * beta) * np.cross(m, mxu))
    return out


def max_torque(m, H):
    """getMaxTorque (:426-439): mu0 * max |m x H|."""
    return float(np.max(np.linalg.norm(np.cross(m, H), axis=1)) * MU0)


def normalize(m):
    return m / np.linalg.norm(m, axis=1, keepdims=True)


# --------------------------------------------------------------------------------------
# Dormand-Prince 5(4) integrator with the freeze-demag outer loop
# --------------------------------------------------------------------------------------
# Butcher tableau of Dormand & Prince (1980), the stepper of TheLLG::IntegrateODEINT
# (main/TheLLG.cpp:517-524, boost::numeric::odeint::runge_kutta_dopri5).
DP_C = np.array([0.0, 1 / 5, 3 / 10, 4 / 5, 8 / 9, 1.0, 1.0])
DP_A = [
    [],
    [1 / 5],
    [3 / 40, 9 / 40],
    [44 / 45, -56 / 15, 32 / 9],
    [19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729],
    [9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656],
    [35 / 384, 0.0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84],
]
DP_B = np.array([35 / 384, 0.0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84, 0.0])
DP_BS = np.array([5179 / 57600, 0.0, 7571 / 16695, 393 / 640, -92097 / 339200, 187 / 2100, 1 / 40])
DP_E = DP_B - DP_BS


@dataclass
class StepControl:
    """Error control of odeint's controlled_runge_kutta (default_error_checker,
    default_step_adjuster): err = max_i |e_i| / (abs + rel (|y_i| + dt |f_i|));
    reject: dt *= max(0.9 err^(-1/3), 0.2); accept with err < 0.5:
    dt *= 0.9 max(err, 5^-5)^(-1/5)."""
    eps_abs: float = 1e-6
    eps_rel: float = 1e-6
    max_dt: float = np.inf


def dp45_segment(f, y, t0, t1, dt, ctl: StepControl = StepControl(), max_steps=10_000_000):
    """Integrate y' = f(t, y) from t0 to t1 (adaptive, FSAL).  Returns
    (y, dt_next, n_accepted, n_rejected, n_rhs)."""
    t = t0
    k1 = f(t, y)
    nrhs = 1
    acc = rej = 0
    while t < t1 and acc + rej < max_steps:
        last = False
        h = min(dt, ctl.max_dt)
        if t + h >= t1:
            h = t1 - t
            last = True
        ks = [k1]
        for s in range(1, 7):
            ys = y + h * sum(a * k for a, k in zip(DP_A[s], ks) if a != 0.0)
            ks.append(f(t + DP_C[s] * h, ys))
            nrhs += 1
        ynew = ys                                        # stage 7 input is the 5th-order solution
        err_vec = h * sum(e * k for e, k in zip(DP_E, ks) if e != 0.0)
        scale = ctl.eps_abs + ctl.eps_rel * (np.abs(y) + h * np.abs(k1))
        err = float(np.max(np.abs(err_vec) / scale))
        if not np.isfinite(err) or err > 1.0:
            dt = h * max(0.9 * (err if np.isfinite(err) else 1e30) ** (-1.0 / 3.0), 0.2)
            rej += 1
            continue
        t = t1 if last else t + h
        y = ynew
        k1 = ks[6]
        acc += 1
        e = max(err, 5.0 ** -5)
        if err < 0.5:
            dtn = h * 0.9 * e ** (-1.0 / 5.0)
        else:
            dtn = h
        if not last:
            dt = dtn
        else:
            dt = max(dt, dtn) if h < dt else dtn
    return y, dt, acc, rej, nrhs


def relax(pb: Problem, m0_soa, duration_ps, segment_ps=0.5, demag: Optional[DemagOracle] = None,
          ctl: StepControl = StepControl(), precession=True):
    """Outer loop of TheSimulation::start (main/TheSimulation.cpp:231-311) with
    frozen demag: per segment refresh H_dem, integrate, normalise, torque."""
    ts = pb.time_scale()
    m = normalize(soa_to_rows(m0_soa))
    dt = min(segment_ps * ts, ts)
    n = pb.nx
    stats = dict(accepted=0, rejected=0, rhs=0, segments=0)
    t_ps = 0.0
    while t_ps < duration_ps - 1e-12:
        hdem = demag.field(m) if demag is not None else np.zeros((n, 3))

        def f(t, y):
            mm = soa_to_rows(y)
            H = local_field(pb, mm, hdem)
            return rows_to_soa(llg_rhs(pb, mm, H, precession))

        seg = min(segment_ps, duration_ps - t_ps)
        y, dt, a, r, nr = dp45_segment(f, rows_to_soa(m), t_ps * ts, (t_ps + seg) * ts, dt, ctl)
        m = normalize(soa_to_rows(y))
        t_ps += seg
        stats["accepted"] += a
        stats["rejected"] += r
        stats["rhs"] += nr
        stats["segments"] += 1
    hdem = demag.field(m) if demag is not None else np.zeros((n, 3))
    H = local_field(pb, m, hdem)
    stats["max_torque"] = max_torque(m, H)
    return m, stats


def energies(pb: Problem, m, hdem):
    """TheSimulation::calculateEnergies (main/TheSimulation.cpp:385-396), energy densities:
    demag -1/2 sum Js V H_dem.m (DemagField.cpp:97-99), exchange -1/2 sum V H_ex.m with
    H_ex = -2 (A/V) K m (EffFieldCalc.cpp:65-69), uniaxial sum V Ku - sum V Ku (k.m)^2 (:86-95),
    Zeeman -sum Js V H_ext.m (TheLLG.cpp:345-348), cubic (EffFieldCalc.cpp:232-247), surface
    (:108-126), DMI -1/2 sum V H_dmi.m (the interfacial form: its own discrete energy), all divided
    by the total volume."""
    V = pb.fem.node_vol
    vt = V.sum()
    e_dem = -0.5 * np.sum(pb.Js * V * np.sum(hdem * m, axis=1)) / vt
    e_ex = -0.5 * np.sum(V * np.sum(exchange_field(pb, m) * m, axis=1)) / vt
    km = np.sum(pb.ku_axis * m, axis=1)
    e_uni = (np.sum(V * pb.Ku) - np.sum(V * pb.Ku * km * km)) / vt
    e_zee = -np.sum(pb.Js * V * np.sum(pb.hext * m, axis=1)) / vt
    if not np.any(pb.D != 0.0):
        e_dmi = 0.0
    elif pb.dmi_kind == "bulk":
        e_dmi = -0.5 * np.sum(V * np.sum(dmi_field(pb, m) * m, axis=1)) / vt
    else:
        e_dmi = interfacial_dmi_energy(pb, m) / vt
    e_cub = e_srf = 0.0
    if "Kc1" in pb.extra:
        al2 = np.einsum("nkd,nd->nk", pb.extra["cax"], m) ** 2
        e_cub = np.sum(V * (pb.extra["Kc1"] * (al2[:, 0] * al2[:, 1] + al2[:, 1] * al2[:, 2] + al2[:, 0] * al2[:, 2])
                            + pb.extra["Kc2"] * al2[:, 0] * al2[:, 1] * al2[:, 2])) / vt
    if "Ks" in pb.extra:
        ksn = pb.extra["Ks"] * pb.bnd.node_area
        nm = np.sum(m * pb.bnd.node_normal, axis=1)
        e_srf = (np.sum(ksn) - np.sum(ksn * nm * nm)) / vt
    tot = e_dem + e_ex + e_uni + e_zee + e_dmi + e_cub + e_srf
    return dict(total=tot, demag=e_dem, exchange=e_ex, uniaxial=e_uni, zeeman=e_zee, cubic=e_cub, surface=e_srf,
                dmi=e_dmi)


def mean_m(pb: Problem, m):
    """TheSimulation::getMeanM: volume-weighted average."""
    V = pb.fem.node_vol
    return (V @ m) / V.sum()


# --------------------------------------------------------------------------------------
# Analytic check: demagnetising factors of a rectangular prism (Aharoni 1998)
# --------------------------------------------------------------------------------------
def aharoni_nz(a, b, c):
    """Demagnetising factor along c of a prism with half-edges a, b, c
    (A. Aharoni, J. Appl. Phys. 83, 3432 (1998), eq. 1)."""
    r = np.sqrt
    abc = r(a * a + b * b + c * c)
    ab = r(a * a + b * b)
    bc = r(b * b + c * c)
    ac = r(a * a + c * c)
    t = ((b * b - c * c) / (2 * b * c) * np.log((abc - a) / (abc + a))
         + (a * a - c * c) / (2 * a * c) * np.log((abc - b) / (abc + b))
         + b / (2 * c) * np.log((ab + a) / (ab - a))
         + a / (2 * c) * np.log((ab + b) / (ab - b))
         + c / (2 * a) * np.log((bc - b) / (bc + b))
         + c / (2 * b) * np.log((ac - a) / (ac + a))
         + 2 * np.arctan(a * b / (c * abc))
         + (a ** 3 + b ** 3 - 2 * c ** 3) / (3 * a * b * c)
         + (a * a + b * b - 2 * c * c) / (3 * a * b * c) * abc
         + c / (a * b) * (ac + bc)
         - (ab ** 3 + bc ** 3 + ac ** 3) / (3 * a * b * c))
    return t / np.pi
