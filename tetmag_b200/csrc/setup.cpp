// Host mesh preprocessing: P1 FEM operators, boundary extraction, solid angles.
//
// Produces the same operators as tetmag's preprocessing so the device path can
// be driven end to end without the reference binary:
//   volumes and shape-function gradients  preproc/FEMprocessing.cpp:104-195
//   gradient / weak-divergence operators  preproc/FEMprocessing.cpp:228-253
//   stiffness matrix                      preproc/FEMprocessing.cpp:266-286
//   boundary triangles, normals, areas    preproc/Boundary.cpp:47-224
//   interior solid angles                 preproc/BEMprocessing.cpp:358-372,
//                                         preproc/Lindholm.cpp:41-61
// In a drop-in deployment tetmag's own MeshData supplies these arrays instead
// (tmb_set_operators in include/tmb.h).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <stdexcept>

#include "tmb_host.h"

namespace tmb {

namespace {

inline double det3(const double m[3][3]) {
  return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
         m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
         m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}

// det([[1,p1],[1,p2],[1,p3],[1,p4]]) = (p2-p1) . ((p3-p1) x (p4-p1))
inline double signed_volume6(const double* p1, const double* p2, const double* p3, const double* p4) {
  double a[3], b[3], c[3];
  for (int d = 0; d < 3; ++d) { a[d] = p2[d] - p1[d]; b[d] = p3[d] - p1[d]; c[d] = p4[d] - p1[d]; }
  return a[0] * (b[1] * c[2] - b[2] * c[1]) + a[1] * (b[2] * c[0] - b[0] * c[2]) +
         a[2] * (b[0] * c[1] - b[1] * c[0]);
}

inline void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

}  // namespace

void fem_prepare(MeshHost& m) {
  const int n = m.nx, ne = m.ntet;
  FemOperators& F = m.fem;
  F.nx = n;
  F.elem_vol.assign(ne, 0.0);
  F.node_vol.assign(n, 0.0);
  std::vector<double> sg(size_t(ne) * 12);  // shape-function gradients [el][node][dim]

  for (int e = 0; e < ne; ++e) {
    const int* t = &m.tets[size_t(e) * 4];
    const double* p[4];
    for (int k = 0; k < 4; ++k) p[k] = &m.xyz[size_t(t[k]) * 3];
    const double V6 = signed_volume6(p[0], p[1], p[2], p[3]);
    const double vol = std::fabs(V6) / 6.0;
    F.elem_vol[e] = vol;
    for (int k = 0; k < 4; ++k) F.node_vol[t[k]] += vol / 4.0;
    // Cofactor form of the P1 gradient, cyclic ordering of the other three
    // nodes (Zienkiewicz, "The Finite Element Method", sec. 4.11).
    for (int nn = 0; nn < 4; ++nn) {
      const double sign = (nn % 2 == 0) ? -1.0 : 1.0;  // (-1)^(nn+1)
      for (int d = 0; d < 3; ++d) {
        double g[3][3];
        for (int r = 0; r < 3; ++r) {
          const double* q = p[(nn + 1 + r) % 4];
          for (int c = 0; c < 3; ++c) g[r][c] = (c == d) ? 1.0 : q[c];
        }
        sg[size_t(e) * 12 + nn * 3 + d] = sign * det3(g) / V6;
      }
    }
  }

  // Shared CSR pattern: neighbours of every node through its elements.
  std::vector<int> deg(n + 1, 0);
  for (int e = 0; e < ne; ++e)
    for (int k = 0; k < 4; ++k) deg[m.tets[size_t(e) * 4 + k] + 1] += 4;
  std::vector<int64_t> start(n + 1, 0);
  for (int i = 0; i < n; ++i) start[i + 1] = start[i] + deg[i + 1];
  std::vector<int> buf(size_t(start[n]));
  std::vector<int64_t> fill(start.begin(), start.end() - 1);
  for (int e = 0; e < ne; ++e) {
    const int* t = &m.tets[size_t(e) * 4];
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) buf[size_t(fill[t[a]]++)] = t[b];
  }
  F.ptr.assign(n + 1, 0);
  std::vector<int> rowlen(n);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    int* b = &buf[size_t(start[i])];
    int len = int(start[i + 1] - start[i]);
    std::sort(b, b + len);
    rowlen[i] = int(std::unique(b, b + len) - b);
  }
  for (int i = 0; i < n; ++i) F.ptr[i + 1] = F.ptr[i] + rowlen[i];
  const int64_t nnz = F.ptr[n];
  if (nnz > std::numeric_limits<int>::max()) throw std::runtime_error("nnz exceeds int32");
  F.col.resize(size_t(nnz));
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i)
    std::memcpy(&F.col[F.ptr[i]], &buf[size_t(start[i])], sizeof(int) * rowlen[i]);
  buf.clear();
  buf.shrink_to_fit();

  F.stiff.assign(size_t(nnz), 0.0);
  for (int d = 0; d < 3; ++d) {
    F.grad[d].assign(size_t(nnz), 0.0);
    F.tgrad[d].assign(size_t(nnz), 0.0);
  }
  auto find = [&](int i, int j) -> int {
    const int* b = &F.col[F.ptr[i]];
    const int* e = &F.col[F.ptr[i + 1]];
    return F.ptr[i] + int(std::lower_bound(b, e, j) - b);
  };
  for (int e = 0; e < ne; ++e) {
    const int* t = &m.tets[size_t(e) * 4];
    const double vol = F.elem_vol[e];
    const double w = vol / 4.0;
    const double* g = &sg[size_t(e) * 12];
    for (int a = 0; a < 4; ++a) {
      const int gi = t[a];
      const double inv_v = 1.0 / F.node_vol[gi];
      for (int b = 0; b < 4; ++b) {
        const int pos = find(gi, t[b]);
        for (int d = 0; d < 3; ++d) {
          F.grad[d][pos] += g[b * 3 + d] * w * inv_v;
          F.tgrad[d][pos] += g[a * 3 + d] * w;
        }
        F.stiff[pos] += vol * (g[a * 3] * g[b * 3] + g[a * 3 + 1] * g[b * 3 + 1] + g[a * 3 + 2] * g[b * 3 + 2]);
      }
    }
  }
}

void extract_boundary(MeshHost& m) {
  const int n = m.nx, ne = m.ntet;
  BoundaryData& B = m.bnd;
  // Faces as sorted node triples; a face seen once is on the boundary.
  struct Face { int a, b, c, tet; };
  std::vector<Face> faces(size_t(ne) * 4);
  for (int e = 0; e < ne; ++e) {
    const int* t = &m.tets[size_t(e) * 4];
    for (int j = 0; j < 4; ++j) {
      int v[3], k = 0;
      for (int q = 0; q < 4; ++q)
        if (q != j) v[k++] = t[q];
      std::sort(v, v + 3);
      faces[size_t(e) * 4 + j] = Face{v[0], v[1], v[2], e};
    }
  }
  std::sort(faces.begin(), faces.end(), [](const Face& x, const Face& y) {
    if (x.a != y.a) return x.a < y.a;
    if (x.b != y.b) return x.b < y.b;
    return x.c < y.c;
  });
  B.tri.clear();
  B.tri_tet.clear();
  for (size_t i = 0; i < faces.size();) {
    size_t j = i + 1;
    while (j < faces.size() && faces[j].a == faces[i].a && faces[j].b == faces[i].b && faces[j].c == faces[i].c) ++j;
    if (j - i == 1) {
      B.tri.push_back(faces[i].a);
      B.tri.push_back(faces[i].b);
      B.tri.push_back(faces[i].c);
      B.tri_tet.push_back(faces[i].tet);
    }
    i = j;
  }
  const int nt = int(B.tri_tet.size());
  B.tri_area.assign(nt, 0.0);
  B.tri_normal.assign(size_t(nt) * 3, 0.0);
  B.node_area.assign(n, 0.0);
  B.node_normal.assign(size_t(n) * 3, 0.0);
  for (int t = 0; t < nt; ++t) {
    const double* p0 = &m.xyz[size_t(B.tri[t * 3]) * 3];
    const double* p1 = &m.xyz[size_t(B.tri[t * 3 + 1]) * 3];
    const double* p2 = &m.xyz[size_t(B.tri[t * 3 + 2]) * 3];
    double v12[3], v13[3], c[3];
    for (int d = 0; d < 3; ++d) { v12[d] = p0[d] - p1[d]; v13[d] = p0[d] - p2[d]; }
    cross3(v12, v13, c);
    const double cn = std::sqrt(dot3(c, c));
    const double area = 0.5 * cn;
    double nv[3] = {c[0] / cn, c[1] / cn, c[2] / cn};
    // orient away from the owning tetrahedron's centre (Boundary.cpp:119-121)
    const int* tt = &m.tets[size_t(B.tri_tet[t]) * 4];
    double ctr[3] = {0, 0, 0};
    for (int k = 0; k < 4; ++k)
      for (int d = 0; d < 3; ++d) ctr[d] += m.xyz[size_t(tt[k]) * 3 + d] / 4.0;
    double tc[3] = {ctr[0] - p0[0], ctr[1] - p0[1], ctr[2] - p0[2]};
    const double s = dot3(nv, tc);
    const double sg = (s > 0) ? 1.0 : ((s < 0) ? -1.0 : 0.0);
    for (int d = 0; d < 3; ++d) nv[d] = -nv[d] * sg;
    B.tri_area[t] = area;
    for (int d = 0; d < 3; ++d) B.tri_normal[size_t(t) * 3 + d] = nv[d];
    for (int k = 0; k < 3; ++k) {
      const int node = B.tri[t * 3 + k];
      B.node_area[node] += area / 3.0;
      for (int d = 0; d < 3; ++d) B.node_normal[size_t(node) * 3 + d] += nv[d] * area / 3.0;
    }
  }
  for (int i = 0; i < n; ++i) {
    double* v = &B.node_normal[size_t(i) * 3];
    const double nn = std::sqrt(dot3(v, v));
    for (int d = 0; d < 3; ++d) {
      const double q = v[d] / nn;
      v[d] = std::isfinite(q) ? q : 0.0;
    }
  }
  B.bnodes.assign(B.tri.begin(), B.tri.end());
  std::sort(B.bnodes.begin(), B.bnodes.end());
  B.bnodes.erase(std::unique(B.bnodes.begin(), B.bnodes.end()), B.bnodes.end());
  B.bindex.assign(n, -1);
  for (size_t i = 0; i < B.bnodes.size(); ++i) B.bindex[B.bnodes[i]] = int(i);
}

double solid_angle(const double* x, const double* t1, const double* t2, const double* t3) {
  double r1[3], r2[3], r3[3];
  for (int d = 0; d < 3; ++d) { r1[d] = t1[d] - x[d]; r2[d] = t2[d] - x[d]; r3[d] = t3[d] - x[d]; }
  const double r1n = std::sqrt(dot3(r1, r1)), r2n = std::sqrt(dot3(r2, r2)), r3n = std::sqrt(dot3(r3, r3));
  const double r23 = dot3(r2, r3), r12 = dot3(r1, r2), r31 = dot3(r3, r1);
  const double numer = r1n * r2n * r3n + r1n * r23 + r2n * r31 + r3n * r12;
  const double denom = std::sqrt(2.0 * (r2n * r3n + r23) * (r3n * r1n + r31) * (r1n * r2n + r12));
  double arg = numer / denom;
  // round-off can push arg just above 1; snap values within 100 ulp of 1
  const double eps = std::numeric_limits<double>::epsilon();
  if (std::fabs(arg - 1.0) < eps * std::fabs(arg + 1.0) * 100.0) arg = 1.0;
  return 2.0 * std::acos(arg);
}

void compute_solid_angles(MeshHost& m) {
  BoundaryData& B = m.bnd;
  B.solid_angle.assign(B.bnodes.size(), 0.0);
  for (int e = 0; e < m.ntet; ++e) {
    const int* t = &m.tets[size_t(e) * 4];
    for (int j = 0; j < 4; ++j) {
      const int bi = B.bindex[t[j]];
      if (bi < 0) continue;
      B.solid_angle[bi] += solid_angle(&m.xyz[size_t(t[j]) * 3], &m.xyz[size_t(t[(j + 1) % 4]) * 3],
                                       &m.xyz[size_t(t[(j + 2) % 4]) * 3], &m.xyz[size_t(t[(j + 3) % 4]) * 3]);
    }
  }
}

}  // namespace tmb
