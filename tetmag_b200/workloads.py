"""Seeded synthetic workloads of the tetmag field path and their device setup.

Each workload restates one measurement configuration: mesh, material,
applied field, initial state and run length.  ``setup_context`` drives the
library end to end: C++ preprocessing (MeshOps), device BEM assembly, material
and applied field.  Material units follow specs/SimulationData.cpp:45-57
(Js = mu0 Ms in T; A / scale^2; D / scale).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import meshgen
from .meshgen import Mesh

MU0 = 1.256637061435917295376e-6


@dataclass
class Workload:
    name: str
    mesh: Mesh
    Ms: float
    A: float
    alpha: float
    m0: np.ndarray                         # 3N SoA
    hext: np.ndarray                       # 3N SoA, A/m
    Ku: float = 0.0
    ku_axis: Optional[np.ndarray] = None   # 3N SoA
    D: float = 0.0
    duration_ps: float = 1000.0
    segment_ps: float = 0.5
    info: dict = field(default_factory=dict)
    components: Optional[np.ndarray] = None   # node offsets of batched instances (None: one mesh)
    shared_bem: bool = False                  # the components are replicas of one mesh
    dmi_kind: str = "bulk"                    # "bulk" (tetmag's) or "interfacial"
    replicas: int = 1                         # interleaved replicas of `mesh` (tmb_set_replicas)

    @property
    def n(self) -> int:
        return self.mesh.nx

    def material_arrays(self):
        n, s = self.n, self.mesh.scale
        Js = np.full(n, MU0 * self.Ms)
        A = np.full(n, self.A / s ** 2)
        Ku = np.full(n, self.Ku) if self.Ku != 0.0 else None
        D = np.full(n, self.D / s) if self.D != 0.0 else None
        return Js, A, Ku, self.ku_axis, D


def cuboid_random(ncx: int, ncy: int, ncz: int, h: float, seed: int = 1, alpha: float = 1.0,
                  name: str = "cuboid") -> Workload:
    mesh = meshgen.kuhn_cuboid(ncx, ncy, ncz, h, name=name)
    return Workload(name=name, mesh=mesh, Ms=8.0e5, A=1.3e-11, alpha=alpha,
                    m0=meshgen.random_state(mesh.nx, seed), hext=np.zeros(3 * mesh.nx))


def c1(seed: int = 1) -> Workload:
    """Permalloy cuboid 100x100x10 nm, 5 nm Kuhn cells (21x21x3 = 1323 nodes), dense BEM,
    alpha = 1, zero field, random initial state, relax 1 ns."""
    w = cuboid_random(20, 20, 2, 5.0, seed=seed, alpha=1.0, name="c1_cuboid_100x100x10nm_h5")
    w.duration_ps = 1000.0
    return w


def c2(seed: int = 2) -> Workload:
    """Permalloy cuboid 500x500x20 nm, 2.5 nm Kuhn cells (201x201x9 = 363609 nodes),
    alpha = 0.02, 20 mT at 10 deg in-plane, seeded vortex, 2 ns."""
    mesh = meshgen.kuhn_cuboid(200, 200, 8, 2.5, name="c2_cuboid_500x500x20nm_h2.5")
    m0, centre = meshgen.vortex_state(mesh.xyz, seed=seed, core_radius=10.0)
    return Workload(name=mesh.name, mesh=mesh, Ms=8.0e5, A=1.3e-11, alpha=0.02, m0=m0,
                    hext=meshgen.field_from_angles(mesh.nx, 0.020, 90.0, 10.0), duration_ps=2000.0,
                    info=dict(vortex_centre_nm=centre.tolist()))


def c4_replica(seed: int = 4, replica: int = 0) -> Workload:
    """Cuboid 200x200x40 nm, 4 nm Kuhn cells (51x51x11 = 28611 nodes, 7002 boundary nodes);
    one of 64 replicas: seeded random m0 and 0-50 mT at a random direction, alpha = 0.5, 1 ns."""
    mesh = meshgen.kuhn_cuboid(50, 50, 10, 4.0, name="c4_cuboid_200x200x40nm_h4")
    rng = np.random.default_rng([seed, replica])
    b = rng.uniform(0.0, 0.050)
    d = rng.standard_normal(3)
    d /= np.linalg.norm(d)
    th, ph = np.degrees(np.arccos(d[2])), np.degrees(np.arctan2(d[1], d[0]))
    return Workload(name=mesh.name, mesh=mesh, Ms=8.0e5, A=1.3e-11, alpha=0.5,
                    m0=meshgen.random_state(mesh.nx, int(rng.integers(1 << 31))),
                    hext=meshgen.field_from_angles(mesh.nx, b, th, ph), duration_ps=1000.0,
                    info=dict(replica=replica, b_tesla=b))


def c4_batch(replicas: int = 64, seed: int = 4, interleaved: bool = True) -> Workload:
    """The c4 cuboid as `replicas` replicas in one context, each with the m0 and applied field of
    c4_replica(seed, r).  interleaved: one mesh with interleaved replica vectors (tmb_set_replicas:
    every operator row applied to all replicas at once, the boundary product one GEMM); else the
    disjoint union of copies declared as shared-BEM components (tmb_set_components)."""
    reps = [c4_replica(seed=seed, replica=r) for r in range(replicas)]
    info = dict(replicas=replicas, b_tesla=[r.info["b_tesla"] for r in reps])
    if interleaved:
        base = reps[0].mesh
        mesh = meshgen.Mesh(xyz=base.xyz, tets=base.tets, scale=base.scale,
                            name=f"c4x{replicas}_cuboid_200x200x40nm_h4")
        return Workload(name=mesh.name, mesh=mesh, Ms=8.0e5, A=1.3e-11, alpha=0.5,
                        m0=meshgen.interleave([r.m0 for r in reps]), hext=meshgen.interleave([r.hext for r in reps]),
                        duration_ps=1000.0, replicas=replicas, info=info)
    mesh, off = meshgen.union([reps[0].mesh] * replicas, name=f"c4x{replicas}_union_cuboid_200x200x40nm_h4")
    return Workload(name=mesh.name, mesh=mesh, Ms=8.0e5, A=1.3e-11, alpha=0.5,
                    m0=meshgen.soa_stack([r.m0 for r in reps]), hext=meshgen.soa_stack([r.hext for r in reps]),
                    duration_ps=1000.0, components=off, shared_bem=True, info=info)


def c3_dots(ndots: int = 256, seed: int = 3, h_range=(2.0, 3.0)) -> Workload:
    """Batched uneven instances: ndots cuboid nanodots, sides Lx, Ly ~ U[20, 60] nm and thickness
    Lz ~ U[5, 20] nm at cell size h ~ U[h_range] nm (integer cell counts, at least one cell),
    each with its own dense BEM; Ku = 5e4 J/m^3 along a random unit axis per dot, alpha = 0.1,
    |B| ~ U[0, 100] mT in a random direction per dot, random m0; 0.5 ns."""
    meshes, m0, hext, axes, sizes = [], [], [], [], []
    for d in range(ndots):
        rng = np.random.default_rng([seed, d])
        h = rng.uniform(*h_range)
        L = np.array([rng.uniform(20, 60), rng.uniform(20, 60), rng.uniform(5, 20)])
        nc = np.maximum(1, np.rint(L / h).astype(int))
        m = meshgen.kuhn_cuboid(int(nc[0]), int(nc[1]), int(nc[2]), h, name=f"dot{d}")
        ax = rng.standard_normal(3)
        ax /= np.linalg.norm(ax)
        b = rng.uniform(0.0, 0.100)
        u = rng.standard_normal(3)
        u /= np.linalg.norm(u)
        th, ph = np.degrees(np.arccos(u[2])), np.degrees(np.arctan2(u[1], u[0]))
        meshes.append(m)
        m0.append(meshgen.random_state(m.nx, int(rng.integers(1 << 31))))
        hext.append(meshgen.field_from_angles(m.nx, b, th, ph))
        axes.append(np.ascontiguousarray(np.repeat(ax, m.nx)))
        sizes.append(m.nx)
    mesh, off = meshgen.union(meshes, name=f"c3_{ndots}dots")
    return Workload(name=mesh.name, mesh=mesh, Ms=8.0e5, A=1.3e-11, alpha=0.1, m0=meshgen.soa_stack(m0),
                    hext=meshgen.soa_stack(hext), Ku=5e4, ku_axis=meshgen.soa_stack(axes), duration_ps=500.0,
                    components=off, info=dict(dots=ndots, nodes_per_dot=sizes))


def instances(w: Workload) -> int:
    if w.replicas > 1:
        return w.replicas
    return 1 if w.components is None else len(w.components) - 1


def component(w: Workload, c: int) -> Workload:
    """Instance c of a batched workload as a single-mesh workload (its own mesh, m0, field)."""
    if w.replicas > 1:
        pick = lambda v: None if v is None else meshgen.deinterleave(v, w.replicas)[c]  # noqa: E731
        return Workload(name=f"{w.name}[{c}]", mesh=w.mesh, Ms=w.Ms, A=w.A, alpha=w.alpha, m0=pick(w.m0),
                        hext=pick(w.hext), Ku=w.Ku, ku_axis=w.ku_axis, D=w.D, duration_ps=w.duration_ps,
                        segment_ps=w.segment_ps, dmi_kind=w.dmi_kind)
    if w.components is None:
        return w
    off = w.components
    lo, hi = int(off[c]), int(off[c + 1])
    sel = (w.mesh.tets.min(axis=1) >= lo) & (w.mesh.tets.max(axis=1) < hi)
    mesh = meshgen.Mesh(xyz=w.mesh.xyz[lo:hi].copy(), tets=np.ascontiguousarray(w.mesh.tets[sel] - lo),
                        scale=w.mesh.scale, name=f"{w.name}[{c}]")
    split = lambda v: None if v is None else meshgen.soa_split(v, off)[c]  # noqa: E731
    return Workload(name=mesh.name, mesh=mesh, Ms=w.Ms, A=w.A, alpha=w.alpha, m0=split(w.m0), hext=split(w.hext),
                    Ku=w.Ku, ku_axis=split(w.ku_axis), D=w.D, duration_ps=w.duration_ps, segment_ps=w.segment_ps)


def c5_disk(seed: int = 5, diameter: float = 150.0, thickness: float = 10.0, h: float = 3.0, nsteps: int = 500,
            dt_ps: float = 1.0, n_bz: int = 100, ckpt_every: int = 10) -> Workload:
    """Interfacial-DMI disk (150 nm x 10 nm, seeded jittered 3 nm lattice: about 8.2k nodes) with a
    seeded Neel skyrmion (radius 20 nm); Ms = 3.84e5 A/m, A = 8.78e-12 J/m, D = 1.58e-3 J/m^2,
    alpha = 0.3, Ku = 0 along z (the differentiated parameter); nsteps steps of dt_ps under a
    piecewise-linear Bz(t) of n_bz samples over the run (seeded: a 50 mT Gaussian pulse centred
    at 30 % of the run plus 5 mT noise).  Each step is split into RK4 substeps that keep the
    exchange spectrum inside RK4's stability region (see stable_substeps)."""
    mesh = meshgen.jittered_disk(diameter, thickness, h, seed=seed, name=f"c5_disk_d{diameter:g}_t{thickness:g}_h{h:g}")
    rng = np.random.default_rng([seed, 55])
    t1 = nsteps * dt_ps
    ts = np.linspace(0.0, t1, n_bz)
    bz = 0.05 * np.exp(-((ts - 0.3 * t1) / (0.12 * t1)) ** 2) + 0.005 * rng.standard_normal(n_bz)
    m0 = meshgen.skyrmion_state(mesh.xyz, seed, radius=20.0 * diameter / 150.0, wall=5.0 * diameter / 150.0)
    axis = np.ascontiguousarray(np.concatenate([np.zeros(2 * mesh.nx), np.ones(mesh.nx)]))
    return Workload(name=mesh.name, mesh=mesh, Ms=3.84e5, A=8.78e-12, alpha=0.3, m0=m0, hext=np.zeros(3 * mesh.nx),
                    Ku=0.0, ku_axis=axis, D=1.58e-3, duration_ps=t1, dmi_kind="interfacial",
                    info=dict(nsteps=nsteps, dt_ps=dt_ps, bz=bz, bz_t0=0.0, bz_t1=t1, ckpt_every=ckpt_every))


def stable_substeps(w: Workload, mesh_ops, dt_ps: float, limit: float = 2.5) -> int:
    """RK4 substeps per step of dt_ps such that h * rho <= limit, with rho the spectral radius of the
    exchange operator diag(2 A / (V Js)) K in reduced time (gamma / (1 + alpha^2)), from the
    symmetric form D^1/2 K D^1/2 (Lanczos).  The linearised LLG has eigenvalues (-alpha +- i) rho,
    and RK4's stability region reaches about 2.8 along those directions; exchange dominates the
    spectrum on nm meshes (demag, DMI and anisotropy rates are two orders smaller here)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    op = mesh_ops.operators()
    n = w.n
    K = sp.csr_matrix((op["stiff"], op["col"], op["rowptr"]), shape=(n, n))
    d = np.sqrt(2.0 * (w.A / w.mesh.scale ** 2) / (op["node_vol"] * MU0 * w.Ms))
    S = sp.diags(d) @ K @ sp.diags(d)
    rho = float(spla.eigsh(S, k=1, which="LA", return_eigenvectors=False, tol=1e-3)[0]) * 1.02
    gamma0 = 221276.14886372426114160400
    per_ps = gamma0 / (1.0 + w.alpha ** 2) * 1e-12
    return max(1, int(np.ceil(dt_ps * per_ps * rho * np.sqrt(1.0 + w.alpha ** 2) / limit)))


WORKLOADS = {"c1": c1, "c2": c2, "c3": c3_dots, "c4": c4_replica, "c4x64": c4_batch, "c5": c5_disk}


def setup_context(w: Workload, device: int = 0, mixed: bool = False, tol: float = 1e-7, maxiter: int = 100,
                  mesh_ops=None, hmatrix: bool = False, keep_dense: bool = True, eps_mixed: float = 1e-6,
                  eps_fp64: float = 1e-7, kmax: int = 64, normal_split: bool = True, h2=None,
                  matrix_share: float = 0.0):
    """MeshOps + Context with operators, device-assembled BEM (dense, optionally compressed to the
    hierarchical form with leaf 32 and eta 2), material and applied field.  hmatrix="mesh" builds
    the hierarchical matrix from the mesh boundary; the dense matrix is then assembled only when
    keep_dense is set, in the far-field-accurate arithmetic the hierarchical matrix approximates.
    h2=(eps_fp64, eps_mixed) then recompresses the hierarchical matrix into nested cluster bases (H2)
    and selects the H2 matvec.  matrix_share > 0 builds the hierarchical matrix to matrix-relative
    accuracy (tmb_set_bem_accuracy)."""
    from .api import Context, MeshOps

    mo = mesh_ops if mesh_ops is not None else MeshOps(w.mesh.xyz, w.mesh.tets)
    ctx = Context(device)
    ctx.set_mesh(mo)
    if w.replicas > 1:
        ctx.set_replicas(w.replicas)
    if w.components is not None:
        ctx.set_components(w.components, shared_bem=w.shared_bem)
    if hmatrix:
        ctx.set_bem_accuracy(matrix_share)
    if hmatrix == "mesh":
        if keep_dense:
            ctx.bem_assemble(mo, accurate=True)
        ctx.bem_build_h(mo, leaf=32, eta=2.0, eps_mixed=eps_mixed, eps_fp64=eps_fp64, kmax=kmax)
    else:
        ctx.bem_assemble(mo)
    if hmatrix and hmatrix != "mesh":
        bd = mo.boundary()
        bn = bd["bnodes"]
        nrm = bd["node_normal"].reshape(3, -1).T[bn] if normal_split else None
        ctx.bem_compress(w.mesh.xyz[bn], bnormal=nrm, leaf=32, eta=2.0, eps_mixed=eps_mixed, eps_fp64=eps_fp64,
                         kmax=kmax, keep_dense=keep_dense)
    if h2 is not None and hmatrix:
        # h2: (eps_fp64, eps_mixed) of the recompression into nested cluster bases
        ctx.bem_h2(eps_fp64=h2[0], eps_mixed=h2[1], kmax=64)
    Js, A, Ku, axis, D = w.material_arrays()
    ctx.set_material(Js, A, Ku=Ku, ku_axis=axis, D=D, alpha=w.alpha)
    if w.dmi_kind == "interfacial":
        ctx.set_dmi_kind(True)
    ctx.set_applied_field(np.ascontiguousarray(w.hext, dtype=np.float64))
    ctx.set_precision(mixed)
    ctx.set_solver_params(tol, maxiter)
    return mo, ctx
