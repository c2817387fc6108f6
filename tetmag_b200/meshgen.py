"""Seeded synthetic meshes and initial states for the tetmag workloads.

tetmag reads its tetrahedral meshes from legacy VTK / gmsh files
(io/MeshReaderInterface.cpp:68-82) and its initial magnetisation from
specs/InitMag.cpp:44-247.  The workloads here are generated instead:

* ``kuhn_cuboid`` -- a structured cuboid whose cubic cells are each split into
  six tetrahedra around the (1,1,1) diagonal (Kuhn / Freudenthal split).  All
  cells use the same split, so the mesh is conforming.  Coordinates are in
  mesh units (nm for ``scale = 1e-9``), centred on the origin like the
  vortex initial state of specs/InitMag.cpp:203-225 expects.
* ``jittered_disk`` -- an unstructured disk from a seeded Delaunay triangulation of a
  jittered lattice, extruded in layers (the interfacial-DMI workload).
* initial states: uniform random on the unit sphere, and a vortex with a
  seeded core position.

Node numbering of the cuboid is ``i + nx*(j + ny*k)`` (x fastest).
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass

import numpy as np


@dataclass
class Mesh:
    xyz: np.ndarray      # (N, 3) float64, mesh units
    tets: np.ndarray     # (E, 4) int32
    scale: float = 1e-9  # metres per mesh unit (the ``scale`` key of simulation.cfg)
    name: str = "mesh"

    @property
    def nx(self) -> int:
        return int(self.xyz.shape[0])


def kuhn_cuboid(ncx: int, ncy: int, ncz: int, h: float, scale: float = 1e-9,
                name: str = "cuboid") -> Mesh:
    """Cuboid of ncx*ncy*ncz cubes of edge h, each cube split into 6 tets."""
    nx, ny, nz = ncx + 1, ncy + 1, ncz + 1
    gx = (np.arange(nx) - 0.5 * ncx) * h
    gy = (np.arange(ny) - 0.5 * ncy) * h
    gz = (np.arange(nz) - 0.5 * ncz) * h
    Z, Y, X = np.meshgrid(gz, gy, gx, indexing="ij")
    xyz = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1).astype(np.float64)

    ci, cj, ck = np.meshgrid(np.arange(ncx), np.arange(ncy), np.arange(ncz), indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()

    def node(di, dj, dk):
        return (ci + di) + nx * ((cj + dj) + ny * (ck + dk))

    tets = []
    for perm in itertools.permutations(range(3)):
        off = np.zeros(3, dtype=int)
        verts = [node(0, 0, 0)]
        for ax in perm:
            off[ax] = 1
            verts.append(node(*off))
        tets.append(np.stack(verts, axis=1))
    tets = np.concatenate(tets, axis=0).astype(np.int32)
    # order elements cell by cell (memory locality of the element loop)
    cell = np.tile(np.arange(ci.size), 6)
    order = np.argsort(cell, kind="stable")
    return Mesh(xyz=xyz, tets=np.ascontiguousarray(tets[order]), scale=scale, name=name)


def jittered_disk(diameter: float, thickness: float, h: float, seed: int,
                  jitter: float = 0.3, scale: float = 1e-9, name: str = "disk") -> Mesh:
    """Seeded disk: Delaunay triangulation of a jittered square lattice of spacing h inside the
    circle (plus a rim ring of about 2 pi R / h points), extruded through round(t / h) layers.

    Lattice points are jittered by up to +-jitter*h in x and y and kept if they lie more than
    h/2 inside the rim.  Each prism (triangle x layer) is split into three tetrahedra by the
    vertex-order rule (the diagonal of every side quad runs from the lower-numbered vertex's
    bottom node to the higher-numbered vertex's top node), so neighbouring prisms share their
    split faces and the mesh is conforming.  The 2D Delaunay step keeps every triangle well
    shaped, so the mesh has no slivers (a 3D Delaunay of a jittered lattice has many, and their
    stiffness sets the explicit time step).  All tetrahedra are positively oriented.
    """
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    R = 0.5 * diameter
    g = np.arange(-R, R + 1e-9, h)
    X, Y = np.meshgrid(g, g, indexing="ij")
    X = X.ravel() + jitter * h * rng.uniform(-1, 1, X.size)
    Y = Y.ravel() + jitter * h * rng.uniform(-1, 1, Y.size)
    keep = X * X + Y * Y < (R - 0.5 * h) ** 2
    n_ring = max(8, int(round(2 * np.pi * R / h)))
    phi = 2 * np.pi * np.arange(n_ring) / n_ring
    p2 = np.concatenate([np.stack([X[keep], Y[keep]], axis=1),
                         np.stack([R * np.cos(phi), R * np.sin(phi)], axis=1)], axis=0)
    tri = np.sort(Delaunay(p2).simplices.astype(np.int64), axis=1)
    e1, e2 = p2[tri[:, 1]] - p2[tri[:, 0]], p2[tri[:, 2]] - p2[tri[:, 0]]
    a2 = np.abs(e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]) * 0.5
    tri = tri[a2 > 1e-6 * h * h]
    nz = max(1, int(round(thickness / h)))
    zs = np.linspace(-0.5 * thickness, 0.5 * thickness, nz + 1)
    n2 = p2.shape[0]
    xyz = np.concatenate([np.concatenate([p2, np.full((n2, 1), z)], axis=1) for z in zs], axis=0)
    tets = []
    for k in range(nz):
        i, j, l = tri[:, 0], tri[:, 1], tri[:, 2]
        b, t = k * n2, (k + 1) * n2
        tets.append(np.stack([i + b, j + b, l + b, l + t], axis=1))
        tets.append(np.stack([i + b, j + b, j + t, l + t], axis=1))
        tets.append(np.stack([i + b, i + t, j + t, l + t], axis=1))
    tets = np.concatenate(tets, axis=0)
    p = xyz[tets]
    vol = np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0])
    neg = vol < 0
    tets[neg, 2], tets[neg, 3] = tets[neg, 3].copy(), tets[neg, 2].copy()
    return Mesh(xyz=np.ascontiguousarray(xyz), tets=np.ascontiguousarray(tets, dtype=np.int32), scale=scale,
                name=name)


def union(meshes, name: str = "union"):
    """Disjoint union of meshes (batched instances): nodes and elements stacked in order, element
    ids offset.  Returns the mesh and the node offsets of the components (length len(meshes)+1).
    The components keep their own coordinates (they may overlap in space; nothing couples them)."""
    off = np.zeros(len(meshes) + 1, dtype=np.int64)
    for i, m in enumerate(meshes):
        off[i + 1] = off[i] + m.nx
    xyz = np.concatenate([m.xyz for m in meshes], axis=0)
    tets = np.concatenate([m.tets.astype(np.int64) + off[i] for i, m in enumerate(meshes)], axis=0)
    if off[-1] >= 2 ** 31:
        raise ValueError("union too large for int32 node ids")
    return Mesh(xyz=xyz, tets=np.ascontiguousarray(tets, dtype=np.int32), scale=meshes[0].scale, name=name), off


def soa_stack(vectors) -> np.ndarray:
    """Concatenate per-component SoA nodal vectors (3 n_c each) into the union's SoA layout."""
    n = [v.size // 3 for v in vectors]
    return np.ascontiguousarray(np.concatenate([np.concatenate([v[d * k:(d + 1) * k] for v, k in zip(vectors, n)])
                                                for d in range(3)]))


def soa_split(v: np.ndarray, offsets) -> list:
    """Inverse of soa_stack for the union with node offsets `offsets`."""
    N = int(offsets[-1])
    return [np.concatenate([v[d * N + offsets[c]:d * N + offsets[c + 1]] for d in range(3)])
            for c in range(len(offsets) - 1)]


def interleave(vectors) -> np.ndarray:
    """R per-replica SoA vectors (3N each, one mesh) -> the interleaved replica layout of
    tmb_set_replicas: component d of node i of replica r at d * N * R + i * R + r."""
    R = len(vectors)
    n = vectors[0].size // 3
    a = np.stack([np.asarray(v, dtype=np.float64).reshape(3, n) for v in vectors], axis=2)  # (3, N, R)
    return np.ascontiguousarray(a.ravel())


def deinterleave(v: np.ndarray, R: int) -> list:
    """Inverse of interleave."""
    a = np.asarray(v).reshape(3, -1, R)
    return [np.ascontiguousarray(a[:, :, r].ravel()) for r in range(R)]


def random_state(n: int, seed: int) -> np.ndarray:
    """i.i.d. directions uniform on S^2 (normalised Gaussian triples), SoA (3N,)."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((n, 3))
    g /= np.linalg.norm(g, axis=1, keepdims=True)
    return np.ascontiguousarray(g.T.ravel())


def vortex_state(xyz: np.ndarray, seed: int, core_radius: float = 10.0,
                 polarity: float = 1.0, chirality: float = 1.0) -> np.ndarray:
    """In-plane vortex with a seeded core position in the central half.

    Follows the shape of the ``vortex`` initial state (specs/InitMag.cpp:203-225):
    curling in-plane magnetisation around the core; here the core has a smooth
    out-of-plane profile m_z = p*exp(-(r/rc)^2) instead of a hard disc.
    """
    rng = np.random.default_rng(seed)
    lo, hi = xyz[:, :2].min(axis=0), xyz[:, :2].max(axis=0)
    centre = 0.5 * (lo + hi) + 0.25 * (hi - lo) * rng.uniform(-1, 1, 2)
    d = xyz[:, :2] - centre
    r = np.linalg.norm(d, axis=1)
    mz = polarity * np.exp(-(r / core_radius) ** 2)
    inpl = np.sqrt(np.maximum(0.0, 1.0 - mz * mz))
    rs = np.where(r > 0, r, 1.0)
    mx = -chirality * d[:, 1] / rs * inpl
    my = chirality * d[:, 0] / rs * inpl
    m = np.stack([mx, my, mz], axis=1)
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    return np.ascontiguousarray(m.T.ravel()), centre


def skyrmion_state(xyz: np.ndarray, seed: int, radius: float = 20.0, wall: float = 5.0,
                   core_shift: float = 2.0, polarity: float = -1.0, helicity: float = 0.0) -> np.ndarray:
    """Neel skyrmion (helicity 0: radial in-plane rotation, the interfacial-DMI chirality) with a
    seeded core offset of at most ``core_shift`` from the xy centre of the mesh.

    theta(r) = 2 atan(exp((radius - r) / wall)) measured from the background direction
    -polarity * z, so the core points along polarity * z.  SoA (3N,), unit length.
    """
    rng = np.random.default_rng(seed)
    lo, hi = xyz[:, :2].min(axis=0), xyz[:, :2].max(axis=0)
    centre = 0.5 * (lo + hi) + core_shift * rng.uniform(-1, 1, 2)
    d = xyz[:, :2] - centre
    r = np.linalg.norm(d, axis=1)
    th = 2.0 * np.arctan(np.exp((radius - r) / wall))
    ph = np.arctan2(d[:, 1], d[:, 0]) + helicity
    mz = -polarity * np.cos(th)
    mx = np.sin(th) * np.cos(ph)
    my = np.sin(th) * np.sin(ph)
    m = np.stack([mx, my, mz], axis=1)
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    return np.ascontiguousarray(m.T.ravel())


def uniform_state(n: int, direction=(1.0, 0.0, 0.0)) -> np.ndarray:
    d = np.asarray(direction, dtype=np.float64)
    d = d / np.linalg.norm(d)
    return np.ascontiguousarray(np.repeat(d, n))


def field_from_angles(n: int, b_tesla: float, theta_deg: float, phi_deg: float) -> np.ndarray:
    """Uniform applied field in A/m, SoA (3N,): B/mu0 along (theta, phi).

    Same convention as fieldFromAngles (main/TheLLG.cpp:442-449).
    """
    mu0 = 1.256637061435917295376e-6
    th, ph = np.deg2rad(theta_deg), np.deg2rad(phi_deg)
    d = np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
    return np.ascontiguousarray(np.repeat(d * (b_tesla / mu0), n))
