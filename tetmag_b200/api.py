"""Python host API over the C ABI, shaped like tetmag's own classes.

* ``MeshOps``     -- preprocessing (PreprocessMesh / MeshBoundary), C++ in libtmb
* ``Context``     -- one mesh on one GPU: operators, BEM, material, fields
* ``DemagField``  -- ``calcField(m)`` as main/DemagField.h:91
* ``TheLLG``      -- ``__call__(state, t)`` as TheLLG::operator() (main/TheLLG.h:148),
                     ``rhs(t, y, ydot)`` as the CVODE callback (main/TheLLG.h:141),
                     ``getMaxTorque(m)`` (main/TheLLG.cpp:426-439)
* ``SolverFactory.makeSolver("b200")`` -- the solver plugin
                     (main/SolverFactory.cpp:124-143), with setMatrix /
                     setLoadVector / setCGTolerance / compute / solve / result /
                     wasSuccessful / report.

Arrays: numpy float64 (host) or CUDA torch float64 tensors (device pointers,
ordered on the context stream).  Vectors of nodal 3-vectors are SoA, length 3N.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib as L
from ._lib import check, lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def _vec(a):
    """(void* address, ptr_kind, keepalive) for numpy or torch arrays."""
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
            raise TypeError("expected a C-contiguous float64 numpy array")
        return a.ctypes.data, L.TMB_PTR_HOST
    try:
        import torch
    except ImportError:  # pragma: no cover
        torch = None
    if torch is not None and isinstance(a, torch.Tensor):
        if a.dtype != torch.float64 or not a.is_contiguous():
            raise TypeError("expected a contiguous float64 tensor")
        if a.is_cuda:
            return a.data_ptr(), L.TMB_PTR_DEVICE
        return a.data_ptr(), L.TMB_PTR_HOST
    raise TypeError(f"unsupported array type {type(a)}")


class MeshOps:
    """Host mesh preprocessing in libtmb (tmb_mesh_*)."""

    def __init__(self, xyz: np.ndarray, tets: np.ndarray):
        self.xyz = _f64(xyz).reshape(-1, 3)
        self.tets = _i32(tets).reshape(-1, 4)
        h = C.c_void_p()
        check(lib().tmb_mesh_create(self.xyz.shape[0], self.tets.shape[0], _dptr(self.xyz), _iptr(self.tets),
                                    C.byref(h)))
        self.h = h
        self._L = lib()
        info = (C.c_longlong * 6)()
        check(lib().tmb_mesh_info(self.h, info))
        self.nx, self.ntet, self.nnz, self.nb, self.ntri = (int(info[i]) for i in range(5))

    def __del__(self):
        # the library handle taken at construction: at interpreter exit module globals may be gone
        h, L = getattr(self, "h", None), getattr(self, "_L", None)
        if h and L is not None:
            L.tmb_mesh_destroy(h)
            self.h = None

    def operators(self) -> dict:
        n, z = self.nx, self.nnz
        out = dict(rowptr=np.empty(n + 1, np.int32), col=np.empty(z, np.int32), stiff=np.empty(z),
                   gx=np.empty(z), gy=np.empty(z), gz=np.empty(z), tgx=np.empty(z), tgy=np.empty(z),
                   tgz=np.empty(z), node_vol=np.empty(n))
        check(lib().tmb_mesh_get_operators(self.h, _iptr(out["rowptr"]), _iptr(out["col"]), _dptr(out["stiff"]),
                                           _dptr(out["gx"]), _dptr(out["gy"]), _dptr(out["gz"]), _dptr(out["tgx"]),
                                           _dptr(out["tgy"]), _dptr(out["tgz"]), _dptr(out["node_vol"])))
        return out

    def boundary(self) -> dict:
        n, nb, nt = self.nx, self.nb, self.ntri
        out = dict(bnodes=np.empty(nb, np.int32), tri=np.empty(3 * nt, np.int32), tri_area=np.empty(nt),
                   tri_normal=np.empty(3 * nt), node_area=np.empty(n), node_normal=np.empty(3 * n),
                   solid_angle=np.empty(nb))
        check(lib().tmb_mesh_get_boundary(self.h, _iptr(out["bnodes"]), _iptr(out["tri"]), _dptr(out["tri_area"]),
                                          _dptr(out["tri_normal"]), _dptr(out["node_area"]),
                                          _dptr(out["node_normal"]), _dptr(out["solid_angle"])))
        return out


class Context:
    """One mesh on one device (tmb_ctx)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().tmb_ctx_create(device, C.byref(h)))
        self.h = h
        self._L = lib()
        self.n = 0
        self.nb = 0
        self.rep = 1

    def __del__(self):
        # the library handle taken at construction: at interpreter exit module globals may be gone
        h, L = getattr(self, "h", None), getattr(self, "_L", None)
        if h and L is not None:
            L.tmb_ctx_destroy(h)
            self.h = None

    # --- setup ---------------------------------------------------------------------------
    def set_mesh(self, mesh: MeshOps):
        check(lib().tmb_set_mesh(self.h, mesh.h))
        self.n, self.nb = mesh.nx, mesh.nb
        return self

    def set_operators(self, rowptr, col, stiff, grad, tgrad, node_vol, bnodes, node_area, node_normal_soa):
        rp, cl = _i32(rowptr), _i32(col)
        arrs = [_f64(stiff)] + [_f64(g) for g in grad] + [_f64(t) for t in tgrad]
        nv, bn, na, nn = _f64(node_vol), _i32(bnodes), _f64(node_area), _f64(node_normal_soa)
        n = rp.size - 1
        check(lib().tmb_set_operators(self.h, n, int(rp[-1]), _iptr(rp), _iptr(cl), *[_dptr(a) for a in arrs],
                                      _dptr(nv), bn.size, _iptr(bn), _dptr(na), _dptr(nn)))
        self.n, self.nb = n, bn.size
        return self

    def bem_assemble(self, mesh: MeshOps, accurate: bool = False):
        """Dense BEM on the device: tetmag's Lindholm arithmetic, or (accurate) the far-field-accurate
        form of the same weights."""
        check(lib().tmb_bem_assemble_ex(self.h, mesh.h, 1 if accurate else 0))
        return self

    def set_components(self, node_offsets, shared_bem: bool = False):
        """The mesh is a disjoint union of components (batched instances); see tmb_set_components."""
        off = _i32(node_offsets)
        check(lib().tmb_set_components(self.h, off.size - 1, _iptr(off), 1 if shared_bem else 0))
        return self

    def set_replicas(self, nrep: int):
        """nrep interleaved replicas of the mesh (tmb_set_replicas): state vectors become 3 N nrep long,
        node i of replica r at i * nrep + r in each component."""
        check(lib().tmb_set_replicas(self.h, int(nrep)))
        self.rep = int(nrep)
        return self

    def set_bem_gemm_kind(self, tensor_cores: bool):
        """Replicas' boundary GEMM on the mixed path: 3xTF32 tensor cores (default) or CUDA cores."""
        check(lib().tmb_set_bem_gemm_kind(self.h, 1 if tensor_cores else 0))
        return self

    def bem_gemm_info(self) -> dict:
        out = (C.c_double * 11)()
        check(lib().tmb_bem_gemm_info(self.h, out))
        return {"tensor_cores": bool(out[0]), "split": int(out[1]), "stages": int(out[10]),
                "tuned_ms": {k + 1: out[2 + k] for k in range(8) if out[2 + k] > 0}}

    def set_bem_dense(self, B: np.ndarray):
        Bc = np.asfortranarray(B, dtype=np.float64)
        check(lib().tmb_set_bem_dense(self.h, Bc.shape[0], Bc.ctypes.data_as(C.POINTER(C.c_double))))
        return self

    def get_bem_dense(self) -> np.ndarray:
        B = np.empty((self.nb, self.nb), order="F")
        check(lib().tmb_get_bem_dense(self.h, B.ctypes.data_as(C.POINTER(C.c_double))))
        return B

    def bem_compress(self, bxyz, bnormal=None, leaf=32, eta=2.0, eps_mixed=1e-6, eps_fp64=1e-7, kmax=64,
                     keep_dense=True):
        """Hierarchical BEM (cluster tree + ACA) from the device-assembled dense matrix."""
        b = _f64(bxyz).reshape(-1, 3)
        nrm = None if bnormal is None else _f64(bnormal).reshape(-1, 3)
        check(lib().tmb_bem_compress(self.h, _dptr(b), _dptr(nrm) if nrm is not None else None, int(leaf),
                                     float(eta), float(eps_mixed), float(eps_fp64), int(kmax),
                                     1 if keep_dense else 0))
        return self

    def bem_build_h(self, mesh: MeshOps, leaf=32, eta=2.0, eps_mixed=1e-6, eps_fp64=1e-7, kmax=64):
        """Hierarchical BEM built from the mesh boundary, no dense matrix needed."""
        check(lib().tmb_bem_build_h(self.h, mesh.h, int(leaf), float(eta), float(eps_mixed), float(eps_fp64),
                                    int(kmax)))
        return self

    def set_bem_accuracy(self, matrix_share: float):
        """Accuracy measure of the next hierarchical build: 0 block-relative cross approximation;
        s > 0 also lets a block stop at its share of a matrix-relative budget (tmb_set_bem_accuracy)."""
        check(lib().tmb_set_bem_accuracy(self.h, float(matrix_share)))
        return self

    def set_bem_mode(self, hierarchical):
        """False / 0: dense; True / 1: hierarchical; 2: H2 (nested cluster bases)."""
        check(lib().tmb_set_bem_mode(self.h, int(hierarchical)))
        return self

    def bem_h2(self, eps_fp64: float = 1e-8, eps_mixed: float = 1e-6, kmax: int = 64):
        """Recompress the hierarchical matrix into nested cluster bases (H2); selects the H2 matvec."""
        check(lib().tmb_bem_h2(self.h, float(eps_fp64), float(eps_mixed), int(kmax)))
        return self

    def bem_h2_info(self) -> dict:
        out = (C.c_double * 16)()
        check(lib().tmb_bem_h2_info(self.h, out))
        keys = ["built", "bytes", "coupling_bytes", "basis_bytes", "max_rank_row", "max_rank_col", "build_ms", "eps"]
        return {p: {k: out[8 * w + i] for i, k in enumerate(keys)} for w, p in enumerate(("fp64", "fp32"))}

    def bem_info(self) -> dict:
        st = (C.c_double * 12)()
        check(lib().tmb_bem_info(self.h, st))
        keys = ["mode", "dense_tiles", "lowrank_blocks", "terms_fp64", "terms_fp32", "bytes_fp64", "bytes_fp32",
                "dense_entries", "blocks_at_cap", "max_rank_fp64", "compress_ms", "built"]
        return {k: st[i] for i, k in enumerate(keys)}

    def bem_verify(self, per_block: bool = False):
        """Probe-vector accuracy of the low-rank blocks against the dense FP64 matrix.
        Returns a dict (rel_err_fp64, rel_err_fp32, worst_block_fp64, worst_block_fp32) and,
        with per_block, an (nblocks, 6) array: |A x|, FP64 error, FP32 error, ranks, cap flag."""
        out = (C.c_double * 4)()
        blk = None
        if per_block:
            blk = np.zeros((int(self.bem_info()["lowrank_blocks"]), 6))
        check(lib().tmb_bem_verify(self.h, _dptr(blk) if blk is not None else None, out))
        res = dict(zip(["rel_err_fp64", "rel_err_fp32", "worst_block_fp64", "worst_block_fp32"], list(out)))
        return (res, blk) if per_block else res

    def bem_apply(self, x, transpose: bool = False, out=None):
        """The boundary product alone (DemagField::mvp): B x or B^T x for a boundary vector in
        boundary-node order, with the current boundary matrix form and precision."""
        if out is None:
            if isinstance(x, np.ndarray):
                out = np.empty(x.size)
            else:
                import torch
                out = torch.empty(x.numel(), dtype=torch.float64, device=x.device)
        px, k = _vec(x)
        po, _ = _vec(out)
        check(lib().tmb_bem_apply(self.h, px, po, 1 if transpose else 0, k))
        return out

    def set_dmi_kind(self, interfacial: bool):
        """DMI form of the material's D: bulk (tetmag's) or interfacial."""
        check(lib().tmb_set_dmi_kind(self.h, 1 if interfacial else 0))
        return self

    def set_material(self, Js, A, Ku=None, ku_axis=None, D=None, alpha=1.0):
        n = self.n
        js, a = _f64(np.broadcast_to(Js, (n,))), _f64(np.broadcast_to(A, (n,)))
        ku = None if Ku is None else _f64(np.broadcast_to(Ku, (n,)))
        ax = None if ku_axis is None else _f64(ku_axis)
        d = None if D is None else _f64(np.broadcast_to(D, (n,)))
        check(lib().tmb_set_material(self.h, _dptr(js), _dptr(a), _dptr(ku) if ku is not None else None,
                                     _dptr(ax) if ax is not None else None, _dptr(d) if d is not None else None,
                                     float(alpha)))
        return self

    def set_applied_field(self, hext):
        p, k = _vec(hext)
        check(lib().tmb_set_applied_field(self.h, p, k))
        return self

    def set_precision(self, mixed: bool):
        check(lib().tmb_set_precision(self.h, L.TMB_MIXED if mixed else L.TMB_FP64))
        return self

    def set_solver_params(self, tol: float, maxiter: int = 100):
        check(lib().tmb_set_solver_params(self.h, float(tol), int(maxiter)))
        return self

    def set_llg_options(self, precession: bool = True):
        check(lib().tmb_set_llg_options(self.h, 1 if precession else 0))
        return self

    def set_stream(self, stream_handle: Optional[int]):
        check(lib().tmb_ctx_set_stream(self.h, C.c_void_p(stream_handle) if stream_handle else None))
        return self

    # --- evaluation ----------------------------------------------------------------------
    def _out_like(self, m):
        if isinstance(m, np.ndarray):
            return np.empty(3 * self.n * self.rep)
        import torch
        return torch.empty(3 * self.n * self.rep, dtype=torch.float64, device=m.device)

    def demag_field(self, m, out=None):
        out = self._out_like(m) if out is None else out
        pm, k = _vec(m)
        po, _ = _vec(out)
        check(lib().tmb_demag_field(self.h, pm, po, k))
        return out

    def field_eval(self, m, ydot=None, hdem=None):
        """Full field evaluation (demag chain + local field + LLG right-hand side)."""
        ydot = self._out_like(m) if ydot is None else ydot
        pm, k = _vec(m)
        py, _ = _vec(ydot)
        ph = _vec(hdem)[0] if hdem is not None else None
        check(lib().tmb_field_eval(self.h, pm, py, ph, k))
        return ydot

    def set_demag_frozen(self, hdem):
        p, k = _vec(hdem)
        check(lib().tmb_set_demag_frozen(self.h, p, k))

    def effective_field(self, m, out=None):
        out = self._out_like(m) if out is None else out
        pm, k = _vec(m)
        po, _ = _vec(out)
        check(lib().tmb_effective_field(self.h, pm, po, k))
        return out

    def llg_rhs(self, t, y, out=None):
        out = self._out_like(y) if out is None else out
        py, k = _vec(y)
        po, _ = _vec(out)
        check(lib().tmb_llg_rhs(self.h, float(t), py, po, k))
        return out

    def max_torque(self, m) -> float:
        v = C.c_double()
        pm, k = _vec(m)
        check(lib().tmb_max_torque(self.h, pm, C.byref(v), k))
        return v.value

    def normalize(self, m):
        pm, k = _vec(m)
        check(lib().tmb_normalize(self.h, pm, k))
        return m

    def relax(self, m, duration_ps, segment_ps=0.5, eps_abs=1e-6, eps_rel=1e-6) -> dict:
        st = (C.c_double * 12)()
        pm, k = _vec(m)
        check(lib().tmb_relax(self.h, pm, float(duration_ps), float(segment_ps), float(eps_abs), float(eps_rel),
                              st, k))
        keys = ["accepted", "rejected", "rhs", "demag", "cg_neumann", "cg_dirichlet", "max_torque", "dt",
                "segments"]
        return {kk: st[i] for i, kk in enumerate(keys)}

    def set_cubic_anisotropy(self, Kc1=None, Kc2=None, axes=None):
        """Cubic anisotropy: Kc1, Kc2 per node [J/m^3] (scalars broadcast), axes (N, 3, 3) or (3, 3) with
        the cubic axes as rows c1, c2, c3.  Kc1=None removes it."""
        if Kc1 is None:
            check(lib().tmb_set_cubic_anisotropy(self.h, None, None, None))
            return self
        n = self.n
        k1, k2 = _f64(np.broadcast_to(Kc1, (n,))), _f64(np.broadcast_to(0.0 if Kc2 is None else Kc2, (n,)))
        ax = _f64(np.broadcast_to(np.asarray(axes, np.float64), (n, 3, 3)).reshape(n, 9))
        check(lib().tmb_set_cubic_anisotropy(self.h, _dptr(k1), _dptr(k2), _dptr(ax)))
        return self

    def set_surface_anisotropy(self, Ks=None):
        """Surface anisotropy Ks per node [J/m^2, divided by the length scale]; None removes it."""
        if Ks is None:
            check(lib().tmb_set_surface_anisotropy(self.h, None))
            return self
        ks = _f64(np.broadcast_to(Ks, (self.n,)))
        check(lib().tmb_set_surface_anisotropy(self.h, _dptr(ks)))
        return self

    def set_stt(self, eta=None, beta: float = 0.0, scale: float = 1.0):
        """Zhang-Li spin-transfer torque: eta 3N SoA per node (or a 3-vector for all nodes), beta, pulse scale."""
        if eta is None:
            check(lib().tmb_set_stt(self.h, None, 0.0, 1.0))
            return self
        e = np.asarray(eta, np.float64)
        if e.size == 3:
            e = np.repeat(e, self.n)
        e = _f64(e)
        check(lib().tmb_set_stt(self.h, _dptr(e), float(beta), float(scale)))
        return self

    def energies(self, m) -> dict:
        """Energy densities [J/m^3] (tmb_energies): total, demag, exchange, uniaxial, zeeman, cubic, surface, dmi."""
        out = (C.c_double * 8)()
        pm, k = _vec(m)
        check(lib().tmb_energies(self.h, pm, out, k))
        keys = ["total", "demag", "exchange", "uniaxial", "zeeman", "cubic", "surface", "dmi"]
        return {kk: out[i] for i, kk in enumerate(keys)}

    def log_row(self, m, elapsed_ps: float, max_torque: float = -1.0) -> str:
        """One row of tetmag's .log file for state m (tmb_log_row)."""
        buf = C.create_string_buffer(1024)
        pm, k = _vec(m)
        check(lib().tmb_log_row(self.h, pm, k, float(elapsed_ps), float(max_torque), buf, len(buf)))
        return buf.value.decode()

    def set_bz_pulse(self, bz_tesla, t0_ps: float, t1_ps: float):
        """Piecewise-linear Bz(t) samples [T] over [t0_ps, t1_ps], added to the applied z field during
        step_rk4 / adjoint_rk4 (an empty sequence removes it)."""
        b = _f64(np.asarray(bz_tesla, dtype=np.float64).ravel())
        check(lib().tmb_set_bz_pulse(self.h, int(b.size), _dptr(b) if b.size else None, float(t0_ps), float(t1_ps)))
        return self

    def step_rk4(self, m, nsteps: int, dt_ps: float, nsub: int = 1, t0_ps: float = 0.0, normalize: bool = True):
        """Fixed-step RK4 (full field at every stage) in place on m; returns the evaluation counters."""
        st = (C.c_double * 8)()
        pm, k = _vec(m)
        check(lib().tmb_step_rk4(self.h, pm, int(nsteps), float(dt_ps), int(nsub), float(t0_ps), int(normalize), st, k))
        return {"rhs_evals": st[0], "cg_iters": st[3]}

    def adjoint_rk4(self, m0, w, nsteps: int, dt_ps: float, nsub: int = 1, ckpt_every: int = 10,
                    t0_ps: float = 0.0, normalize: bool = True, n_bz: int = 0):
        """Discrete adjoint of step_rk4 for J = sum(w * m_final).  m0, w: 3N float64 (numpy or CUDA
        tensors, both of one kind).  Returns dict(J, m_final, grad_m0, grad_ku, grad_bz, stats)."""
        n3 = 3 * self.n
        on_dev = not isinstance(m0, np.ndarray)
        if on_dev:
            import torch
            mk = lambda k: torch.empty(k, dtype=torch.float64, device=m0.device)  # noqa: E731
        else:
            mk = lambda k: np.empty(k)  # noqa: E731
        mf, gm, gk = mk(n3), mk(n3), mk(self.n)
        gb = np.zeros(max(int(n_bz), 1))
        J = C.c_double()
        st = (C.c_double * 8)()
        pm, k = _vec(m0)
        pw, kw = _vec(w)
        if kw != k:
            raise TypeError("m0 and w must both be host or both device arrays")
        check(lib().tmb_adjoint_rk4(self.h, pm, int(nsteps), float(dt_ps), int(nsub), int(ckpt_every), float(t0_ps),
                                    int(normalize), pw, _vec(mf)[0], _vec(gm)[0], _vec(gk)[0], _dptr(gb), C.byref(J),
                                    st, k))
        keys = ["fwd_evals", "recompute_evals", "vjp_evals", "cg_fwd", "cg_adj", "checkpoints", "storage_bytes"]
        return {"J": J.value, "m_final": mf, "grad_m0": gm, "grad_ku": gk, "grad_bz": gb[:int(n_bz)],
                "stats": {kk: st[i] for i, kk in enumerate(keys)}}

    def stats(self) -> dict:
        st = (C.c_double * 8)()
        check(lib().tmb_get_stats(self.h, st))
        keys = ["it_neumann", "it_dirichlet", "res_neumann", "res_dirichlet", "status_neumann",
                "status_dirichlet", "amg_levels", "amg_setup_ms"]
        return {kk: st[i] for i, kk in enumerate(keys)}


def write_vtu(path, xyz, tets, m, material=None, time_ps: float = 0.0, field=None, field_name: str = "Demag",
              binary: bool = True):
    """tetmag's .vtu output (tmb_write_vtu): xyz (N, 3), tets (E, 4), m and field 3N SoA."""
    x, t, mm = _f64(xyz).reshape(-1, 3), _i32(tets).reshape(-1, 4), _f64(m)
    n = x.shape[0]
    mat = None if material is None else _i32(np.broadcast_to(material, (n,)))
    f = None if field is None else _f64(field)
    check(lib().tmb_write_vtu(str(path).encode(), n, _dptr(x), t.shape[0], _iptr(t), _dptr(mm),
                              None if mat is None else _iptr(mat), float(time_ps),
                              None if f is None else _dptr(f), field_name.encode(), 1 if binary else 0))


def read_magnetization(path, nx: int):
    """VTKReader::readMag + getTime (tmb_read_magnetization): (m as 3N SoA, time in ps)."""
    m = np.empty(3 * nx)
    t = C.c_double(0.0)
    check(lib().tmb_read_magnetization(str(path).encode(), int(nx), _dptr(m), C.byref(t)))
    return m, t.value


def log_header(start_time: str, host: str, user: str) -> str:
    """The header of tetmag's .log file (tmb_log_header)."""
    buf = C.create_string_buffer(2048)
    check(lib().tmb_log_header(start_time.encode(), host.encode(), user.encode(), buf, len(buf)))
    return buf.value.decode()


def log_format(elapsed_ps: float, energies, max_torque: float, mean_m, mean_h_tesla) -> str:
    """A .log row from its values (tmb_log_format); energies in tmb_energies order (dict or 8 values)."""
    keys = ["total", "demag", "exchange", "uniaxial", "zeeman", "cubic", "surface", "dmi"]
    e = _f64([energies[k] for k in keys] if isinstance(energies, dict) else energies)
    mm, hh = _f64(mean_m), _f64(mean_h_tesla)
    buf = C.create_string_buffer(1024)
    check(lib().tmb_log_format(float(elapsed_ps), _dptr(e), float(max_torque), _dptr(mm), _dptr(hh), buf, len(buf)))
    return buf.value.decode()


def kernel_launches() -> int:
    v = C.c_longlong()
    check(lib().tmb_kernel_launches(C.byref(v)))
    return int(v.value)


PROFILE_IDS = ["local_llg", "divergence", "gradient", "bem_matvec", "solve_neumann", "solve_dirichlet",
               "cg_spmv", "demag_chain", "cg_update_smooth", "fine_post_smooth_rz", "fine_pre_smooth",
               "restriction", "prolongation", "coarse_smooth", "coarsest_solve", "cg_start", "cg_update"]
# ids that span several kernels (not candidates for a per-kernel roofline)
PROFILE_CONTAINERS = ("solve_neumann", "solve_dirichlet", "demag_chain")
# ids whose every record is one launch of one kernel (the others group the kernels of a product,
# or one kernel per AMG level)
PROFILE_SINGLE = ("local_llg", "divergence", "gradient", "cg_spmv", "cg_update_smooth", "fine_post_smooth_rz",
                  "fine_pre_smooth", "cg_update")


def profile_enable(ctx: "Context", on: bool = True):
    check(lib().tmb_profile_enable(ctx.h, 1 if on else 0))


def profile_read(ctx: "Context") -> dict:
    st = (C.c_double * (3 * len(PROFILE_IDS)))()
    check(lib().tmb_profile_read(ctx.h, st))
    return {k: dict(launches=st[3 * i], total_ms=st[3 * i + 1], bytes_per_launch=st[3 * i + 2])
            for i, k in enumerate(PROFILE_IDS)}


class DemagField:
    """DemagField::calcField (main/DemagField.cpp:92-94) on the device."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def calcField(self, m):
        return self.ctx.demag_field(m)


class TheLLG:
    """TheLLG's right-hand side with frozen demag (main/TheLLG.cpp:119-124, 670-711)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def setHdem(self, hdem):
        self.ctx.set_demag_frozen(hdem)

    def __call__(self, state, t: float = 0.0):
        return self.ctx.llg_rhs(t, state)

    def rhs(self, t: float, y, ydot) -> int:
        """CVODE-style callback: fills ydot, returns 0 on success and -1 on failure."""
        try:
            self.ctx.llg_rhs(t, y, out=ydot)
            return 0
        except L.TmbError:
            return -1

    def getMaxTorque(self, m) -> float:
        return self.ctx.max_torque(m)


class B200Solver:
    """The "b200" case of SolverFactory::makeSolver (main/SolverFactory.h:42-65)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        h = C.c_void_p()
        check(lib().tmb_solver_create(ctx.h, C.byref(h)))
        self.h = h
        self._L = lib()
        self.n = 0
        self.b = None
        self.x = None
        self.tol = 1e-7
        self.maxiter = 100
        self.preconditioner = "amg"
        self._ok = False

    def __del__(self):
        # the library handle taken at construction: at interpreter exit module globals may be gone
        h, L = getattr(self, "h", None), getattr(self, "_L", None)
        if h and L is not None:
            L.tmb_solver_destroy(h)
            self.h = None

    def setMatrix(self, A):
        import scipy.sparse as sp
        A = sp.csr_matrix(A)
        A.sort_indices()
        rp, cl, v = _i32(A.indptr), _i32(A.indices), _f64(A.data)
        self.n = A.shape[0]
        check(lib().tmb_solver_set_matrix(self.h, self.n, int(rp[-1]), _iptr(rp), _iptr(cl), _dptr(v)))

    def setLoadVector(self, b):
        self.b = _f64(b)

    def setCGTolerance(self, tol: float):
        self.tol = float(tol)

    def definePreconditioner(self, name: str):
        self.preconditioner = name

    def compute(self) -> bool:
        check(lib().tmb_solver_set_tolerance(self.h, self.tol, self.maxiter))
        check(lib().tmb_solver_compute(self.h))
        return True

    def solve(self):
        check(lib().tmb_solver_set_tolerance(self.h, self.tol, self.maxiter))
        x = np.empty(self.n)
        code = lib().tmb_solver_solve(self.h, self.b.ctypes.data, x.ctypes.data, L.TMB_PTR_HOST)
        self._ok = code == L.TMB_OK
        self.x = x
        if code not in (L.TMB_OK, L.TMB_ERR_NOCONVERGE):
            check(code)

    def result(self) -> np.ndarray:
        return self.x

    def info(self) -> dict:
        st = (C.c_double * 3)()
        check(lib().tmb_solver_info(self.h, st))
        return dict(iterations=int(st[0]), relres=st[1], status=int(st[2]))

    def wasSuccessful(self) -> bool:
        return self._ok and np.all(np.isfinite(self.x))

    def report(self):
        i = self.info()
        print(f"b200 PCG+AMG: {i['iterations']} iterations, relative residual {i['relres']:.3e}, "
              f"{'successful' if self.wasSuccessful() else 'FAILED'}")


class SolverFactory:
    @staticmethod
    def makeSolver(kind: str, ctx: Context) -> B200Solver:
        if kind.lower() != "b200":
            raise ValueError(f"solver option not understood: {kind}")
        return B200Solver(ctx)
