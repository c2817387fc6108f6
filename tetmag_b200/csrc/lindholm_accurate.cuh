// Lindholm double-layer weights in a far-field-accurate arithmetic (device code).
//
// The weights are those of D.A. Lindholm, IEEE Trans. Magn. 20, 2025 (1984), as tetmag
// evaluates them (preproc/Lindholm.cpp:41-128): vertex i of triangle p seen from x0 gets
//   L_i = s_{i+1} / (8 pi A) (eta_{i+1} . rho_{i+1} Omega - chi0 sum_j gamma_{ij} P_j).
// The reference arithmetic takes the solid angle as 2 acos(arg) with arg -> 1 far away, which
// loses about (r / h)^2 ulps (and clamps arg to 1 within 100 ulps, i.e. Omega to 0 below
// ~6e-7 sr), and the two terms of a weight cancel by a factor ~r / h: several hundred nm from a
// nm-sized triangle the weights are off by ~10%, and on a 500 nm film row sums of the matrix
// miss -1 by up to ~1e-3.  Here the solid angle is 2 atan2(N, D) with the triple product taken
// as N = |e01 x e02| chi0 (Van Oosterom & Strackee, IEEE Trans. Biomed. Eng. 30, 125 (1983)),
// edges come from vertex differences and the edge logarithms use log1p, so the cancellation
// works on full-precision inputs (row sums -1 to ~1e-13).
#pragma once

#include <cmath>

namespace tmb {

__device__ __forceinline__ void lindholm_accurate(const double* x0, const double (*p)[3], double area,
                                                  const double* nv, double* L) {
  double xi[3][3], s[3], rv[3][3], rho[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const int i1 = (i + 1) % 3;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      xi[i][d] = p[i1][d] - p[i][d];
      rv[i][d] = p[i][d] - x0[d];
    }
    s[i] = sqrt(xi[i][0] * xi[i][0] + xi[i][1] * xi[i][1] + xi[i][2] * xi[i][2]);
    rho[i] = sqrt(rv[i][0] * rv[i][0] + rv[i][1] * rv[i][1] + rv[i][2] * rv[i][2]);
  }
  // (p1 - p0) x (p2 - p0) = xi0 x (-xi2)
  const double c[3] = {xi[2][1] * xi[0][2] - xi[2][2] * xi[0][1], xi[2][2] * xi[0][0] - xi[2][0] * xi[0][2],
                       xi[2][0] * xi[0][1] - xi[2][1] * xi[0][0]};
  const double cn = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
  const double chi[3] = {c[0] / cn, c[1] / cn, c[2] / cn};
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int d = 0; d < 3; ++d) xi[i][d] /= s[i];
  auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
  const double chi0 = dot(chi, rv[0]);
  const double D = rho[0] * rho[1] * rho[2] + dot(rv[0], rv[1]) * rho[2] + dot(rv[0], rv[2]) * rho[1] +
                   dot(rv[1], rv[2]) * rho[0];
  const double omega = 2.0 * atan2(cn * chi0, D);
  double P[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) P[j] = log1p(2.0 * s[j] / (rho[j] + rho[(j + 1) % 3] - s[j]));
  const double f = ((dot(nv, chi) < 0.0) ? -1.0 : 1.0) / (8.0 * 3.14159265358979323846 * area);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const int a = (i + 1) % 3;
    const double eta[3] = {chi[1] * xi[a][2] - chi[2] * xi[a][1], chi[2] * xi[a][0] - chi[0] * xi[a][2],
                           chi[0] * xi[a][1] - chi[1] * xi[a][0]};
    const double gP = dot(xi[a], xi[0]) * P[0] + dot(xi[a], xi[1]) * P[1] + dot(xi[a], xi[2]) * P[2];
    L[i] = f * s[a] * (dot(eta, rv[a]) * omega - chi0 * gP);
  }
}

}  // namespace tmb
