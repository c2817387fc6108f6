"""CPU tests of the FP64 oracle: the reference's own known-answer checks,
analytic identities, and the committed golden vectors."""
from pathlib import Path

import numpy as np
import pytest

from oracle import tetmag_oracle as O
from tetmag_b200 import meshgen

GOLDEN = Path(__file__).with_name("golden") / "oracle_small.npz"


@pytest.fixture(scope="module")
def c1():
    mesh = meshgen.kuhn_cuboid(20, 20, 2, 5.0)
    fem = O.fem_prepare(mesh.xyz, mesh.tets)
    bnd = O.extract_boundary(mesh.xyz, mesh.tets)
    return mesh, fem, bnd


def test_c1_sizes(c1):
    # 21x21x3 nodes, unpruned Kuhn pattern, 962 surface nodes
    mesh, fem, bnd = c1
    assert mesh.nx == 1323
    assert fem.stiff.nnz == 15487
    assert bnd.bnodes.size == 962
    assert bnd.tri.shape[0] == 1920
    assert np.isclose(bnd.tri_area.sum(), 2 * (100 * 100 + 2 * 100 * 10))


def test_gradient_operators_exact_on_linear_functions(c1):
    # PreprocessMesh::testGradientOperators (preproc/FEMprocessing.cpp:288-326), tol 1e-10
    mesh, fem, _ = c1
    x, y, z = mesh.xyz.T
    f = 0.5 * x - 17.0 * y + 13.0 * z + 42.0
    for d, c in enumerate((0.5, -17.0, 13.0)):
        g = fem.grad[d] @ f
        assert np.max(np.abs(g - c)) <= 1e-10 * abs(c)


def test_stiffness_and_divergence_annihilate_constants(c1):
    mesh, fem, _ = c1
    one = np.ones(mesh.nx)
    assert np.max(np.abs(fem.stiff @ one)) < 1e-12 * abs(fem.stiff).max()
    for t in fem.tgrad:  # sum_i grad(phi_i) = 0 per element
        assert np.max(np.abs(one @ t)) < 1e-12 * abs(t).max()


def test_dense_bem_rowsum_known_answer(c1):
    # BEMprocessing::testLaplaceMatrix (preproc/BEMprocessing.cpp:440-445, 55-72):
    # sum(B.(-1)) must equal Nb within 5e-3; each row of B sums to -1.
    mesh, _, bnd = c1
    B = O.dense_bem(mesh.xyz, mesh.tets, bnd)
    assert O.bem_rowsum_error(B) < 5e-3
    assert np.max(np.abs(B.sum(axis=1) + 1.0)) < 1e-9


def test_solid_angles_interior(c1):
    # face nodes see 2 pi, edge nodes pi, corner nodes pi/2
    mesh, _, bnd = c1
    sub = O.solid_angles(mesh.xyz, mesh.tets, bnd)
    assert np.allclose(np.sort(np.unique(np.round(sub / np.pi, 12))), [0.5, 1.0, 2.0])


@pytest.mark.parametrize("nc,tol", [(4, 0.03), (8, 0.012)])
def test_demag_factor_of_a_cube(nc, tol):
    # uniformly magnetised cube: N = 1/3 (Aharoni), FEM-BEM converges with h
    mesh = meshgen.kuhn_cuboid(nc, nc, nc, 10.0 / nc)
    pb = O.make_problem(mesh.xyz, mesh.tets, 1e-9, Ms=8e5, A=1.3e-11, alpha=1.0)
    dm = O.DemagOracle(pb)
    m = np.zeros((mesh.nx, 3))
    m[:, 2] = 1.0
    H = dm.field(m)
    Nz = dm.energy(m, H) / (0.5 * pb.Js[0] * 8e5 * pb.fem.node_vol.sum())
    assert abs(Nz - O.aharoni_nz(5.0, 5.0, 5.0)) < tol
    assert abs(O.aharoni_nz(5.0, 5.0, 5.0) - 1.0 / 3.0) < 1e-12


def test_llg_rhs_is_orthogonal_to_m():
    rng = np.random.default_rng(3)
    m = rng.standard_normal((50, 3))
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    H = rng.standard_normal((50, 3)) * 1e5

    class P:
        alpha = 0.5

    ydot = O.llg_rhs(P, m, H)
    assert np.max(np.abs(np.sum(ydot * m, axis=1))) < 1e-9


def test_dp45_on_linear_ode():
    f = lambda t, y: -y  # noqa: E731
    y, dt, acc, rej, nrhs = O.dp45_segment(f, np.array([1.0, 2.0]), 0.0, 3.0, 0.1,
                                          O.StepControl(eps_abs=1e-10, eps_rel=1e-10))
    assert np.allclose(y, np.exp(-3.0) * np.array([1.0, 2.0]), rtol=1e-8)
    assert acc > 0 and nrhs == 6 * (acc + rej) + 1


def test_golden_vectors():
    g = np.load(GOLDEN)
    n = g["xyz"].shape[0]
    pb = O.make_problem(g["xyz"], g["tets"], 1e-9, Ms=8e5, A=1.3e-11, alpha=0.3, Ku=5e4, ku_axis=g["axis"],
                        D=3e-3, hext=g["hext"])
    assert np.max(np.abs(pb.B - g["B"])) < 1e-13
    m = g["m"]
    hdem = O.DemagOracle(pb).field(m)
    assert np.linalg.norm(hdem - g["hdem"]) <= 1e-12 * np.linalg.norm(g["hdem"])
    H = O.local_field(pb, m, hdem)
    assert np.linalg.norm(H - g["H"]) <= 1e-12 * np.linalg.norm(g["H"])
    ydot = O.llg_rhs(pb, m, H)
    assert np.linalg.norm(ydot - g["ydot"]) <= 1e-12 * np.linalg.norm(g["ydot"])
    assert n == 210


def _lindholm_mp(x0, p, nv, dps=50):
    """Lindholm weights in 50-digit arithmetic (mpmath): the exact values both forms approximate."""
    mp = pytest.importorskip("mpmath")
    mp.mp.dps = dps
    X = [mp.mpf(float(v)) for v in x0]
    P = [[mp.mpf(float(v)) for v in q] for q in p]
    sub = lambda a, b: [a[i] - b[i] for i in range(3)]  # noqa: E731
    dot = lambda a, b: sum(a[i] * b[i] for i in range(3))  # noqa: E731
    cross = lambda a, b: [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]  # noqa: E731
    c = cross(sub(P[1], P[0]), sub(P[2], P[0]))
    cn = mp.sqrt(dot(c, c))
    chi = [v / cn for v in c]
    rv = [sub(P[i], X) for i in range(3)]
    xi = [sub(P[(i + 1) % 3], P[i]) for i in range(3)]
    s = [mp.sqrt(dot(v, v)) for v in xi]
    xi = [[v / s[i] for v in xi[i]] for i in range(3)]
    rho = [mp.sqrt(dot(v, v)) for v in rv]
    chi0 = dot(chi, rv[0])
    D = rho[0] * rho[1] * rho[2] + dot(rv[0], rv[1]) * rho[2] + dot(rv[0], rv[2]) * rho[1] + dot(rv[1], rv[2]) * rho[0]
    om = 2 * mp.atan2(cn * chi0, D)
    Pl = [mp.log((rho[i] + rho[(i + 1) % 3] + s[i]) / (rho[i] + rho[(i + 1) % 3] - s[i])) for i in range(3)]
    L = []
    for i in range(3):
        a = (i + 1) % 3
        gP = sum(dot(xi[a], xi[j]) * Pl[j] for j in range(3))
        L.append(s[a] / (8 * mp.pi * cn / 2) * (dot(cross(chi, xi[a]), rv[a]) * om - chi0 * gP))
    if dot([mp.mpf(float(v)) for v in nv], chi) < 0:
        L = [-v for v in L]
    return np.array([float(v) for v in L])


def test_far_field_lindholm_weights():
    # A 2.5 nm bottom-face triangle seen from the top face of a 20 nm film, 10-420 nm away:
    # the reference arithmetic (acos solid angle) loses accuracy with distance (about 10% at
    # 420 nm); the far-field form used for the low-rank blocks stays within 1e-9 relative.
    h = 2.5
    ref_err, acc_err = [], []
    for dist in (10.0, 50.0, 100.0, 200.0, 420.0):
        x0 = np.array([[0.0, 0.0, 10.0]])
        p = np.array([[dist, 0.0, -10.0], [dist + h, 0.0, -10.0], [dist, h, -10.0]])
        nv = np.array([[0.0, 0.0, -1.0]])
        area = np.array([h * h / 2])
        exact = _lindholm_mp(x0[0], p, nv[0])
        args = (x0, p[None, 0], p[None, 1], p[None, 2], area, nv)
        ref_err.append(np.max(np.abs(O.lindholm_weights(*args)[0] - exact)) / np.max(np.abs(exact)))
        acc_err.append(np.max(np.abs(O.lindholm_weights_accurate(*args)[0] - exact)) / np.max(np.abs(exact)))
    assert max(acc_err) < 1e-9
    assert ref_err[-1] > 1e-3                  # the reason the far blocks use the other form
    # random geometries, including observers close to the triangle's plane
    rng = np.random.default_rng(3)
    for trial in range(40):
        p0 = rng.uniform(-5, 5, 3)
        p = np.array([p0, p0 + 3 * rng.standard_normal(3), p0 + 3 * rng.standard_normal(3)])
        d = rng.standard_normal(3)
        x0 = p0 + 10 ** rng.uniform(0.5, 2.5) * d / np.linalg.norm(d)
        nv = np.cross(p[1] - p[0], p[2] - p[0])
        area = np.array([0.5 * np.linalg.norm(nv)])
        exact = _lindholm_mp(x0, p, nv)
        La = O.lindholm_weights_accurate(x0[None], p[None, 0], p[None, 1], p[None, 2], area, nv[None])[0]
        assert np.max(np.abs(La - exact)) <= 1e-9 * np.max(np.abs(exact))


def test_interfacial_dmi_field_is_energy_gradient():
    # the interfacial-DMI field (no reference counterpart) is -(1/V) dE/dm of its discrete energy:
    # checked by central differences of the energy on a small prism
    from tetmag_b200 import meshgen
    mesh = meshgen.kuhn_cuboid(4, 3, 2, 3.0)
    pb = O.make_problem(mesh.xyz, mesh.tets, 1e-9, Ms=3.84e5, A=8.78e-12, alpha=0.3, D=1.58e-3,
                        with_bem=False, dmi_kind="interfacial")
    m = O.soa_to_rows(meshgen.random_state(mesh.nx, 5))
    H = O.interfacial_dmi_field(pb, m)
    V = pb.fem.node_vol
    rng = np.random.default_rng(0)
    for _ in range(12):
        i, d = int(rng.integers(mesh.nx)), int(rng.integers(3))
        eps = 1e-6
        mp, mm = m.copy(), m.copy()
        mp[i, d] += eps
        mm[i, d] -= eps
        dE = (O.interfacial_dmi_energy(pb, mp) - O.interfacial_dmi_energy(pb, mm)) / (2 * eps)
        assert abs(-dE / V[i] - H[i, d]) <= 1e-7 * np.max(np.abs(H))


def _anisotropy_problem():
    from tetmag_b200 import meshgen
    mesh = meshgen.kuhn_cuboid(4, 3, 2, 3.0)
    rng = np.random.default_rng(11)
    k = rng.standard_normal(3)
    pb = O.make_problem(mesh.xyz, mesh.tets, 1e-9, Ms=8e5, A=1.3e-11, alpha=0.3, Ku=4e4,
                        ku_axis=k / np.linalg.norm(k), with_bem=False,
                        hext=rng.standard_normal((mesh.nx, 3)) * 1e4)
    q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    pb.extra.update(Kc1=np.full(mesh.nx, 4.5e4), Kc2=np.full(mesh.nx, -1.2e4),
                    cax=np.broadcast_to(q.T, (mesh.nx, 3, 3)).copy(), Ks=np.full(mesh.nx, 1e-3 / 1e-9))
    m = O.soa_to_rows(meshgen.random_state(mesh.nx, 7))
    return mesh, pb, m


def test_energy_terms_consistent_with_fields():
    # each energy density (TheSimulation::calculateEnergies) times the total volume is the discrete
    # energy whose gradient is -V_i Js H_i of its field term: exchange, uniaxial, Zeeman, cubic by
    # central differences; surface up to a component along m (tetmag's surface field drops the
    # constant part, main/EffFieldCalc.cpp:137-139); the parts add up to the total
    mesh, pb, m = _anisotropy_problem()
    V, vt = pb.fem.node_vol, pb.fem.node_vol.sum()
    hz = np.zeros_like(m)
    e0 = O.energies(pb, m, hz)
    assert np.isclose(e0["total"], sum(v for k, v in e0.items() if k != "total"), rtol=1e-14, atol=0)
    fields = dict(exchange=O.exchange_field(pb, m), uniaxial=O.uniaxial_field(pb, m),
                  zeeman=pb.Js[:, None] * pb.hext, cubic=O.cubic_field(pb, m), surface=O.surface_field(pb, m))
    rng = np.random.default_rng(3)
    for term, H in fields.items():
        scale = np.max(np.abs(H))
        for _ in range(8):
            i, d = int(rng.integers(mesh.nx)), int(rng.integers(3))
            eps = 1e-6
            mp, mm = m.copy(), m.copy()
            mp[i, d] += eps
            mm[i, d] -= eps
            dE = (O.energies(pb, mp, hz)[term] - O.energies(pb, mm, hz)[term]) * vt / (2 * eps)
            g = np.zeros(3)
            g[d] = -dE / V[i]
            if term == "surface":
                # compare only what is perpendicular to m: the rest of the gradient lies along the normal
                nv = pb.bnd.node_normal[i]
                nm = m[i] @ nv
                full = 2.0 * pb.extra["Ks"][i] * pb.bnd.node_area[i] * nm * nv / V[i]
                assert abs(full[d] - g[d]) <= 1e-6 * max(scale, 1.0)
                assert np.allclose(np.cross(m[i], H[i] - full), 0.0, atol=1e-9 * max(scale, 1.0))
            else:
                assert abs(H[i, d] - g[d]) <= 1e-6 * max(scale, 1.0)


def test_stt_term_of_a_uniform_state_vanishes():
    # U = sum_d eta_d grad_d m is zero for a uniform m (gradient operators annihilate constants)
    mesh, pb, _ = _anisotropy_problem()
    pb.extra.update(eta=np.tile([3.0, -1.0, 0.5], (mesh.nx, 1)), beta=0.04)
    m = np.tile([0.6, 0.0, 0.8], (mesh.nx, 1))
    H = O.local_field(pb, m, np.zeros_like(m))
    ref = O.llg_rhs(pb, m, H)
    del pb.extra["eta"]
    assert np.max(np.abs(ref - O.llg_rhs(pb, m, H))) <= 1e-10 * np.max(np.abs(ref))
