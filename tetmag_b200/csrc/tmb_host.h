// Host-side data structures of the tetmag B200 library (internal header).
//
// The mesh preprocessing here produces the operators that tetmag's
// PreprocessMesh / MeshBoundary / BEMprocessing hand to TheLLG and DemagField
// (MeshData, specs/MeshData.h:41-63): the stiffness matrix K, the nodal
// gradient operators grad_{x,y,z}, the weak-divergence operators
// tGrad_{x,y,z}, node volumes, boundary nodes, boundary triangles with
// outward normals, node areas and node normals, and the interior solid angle
// at every boundary node.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace tmb {

// Compressed sparse row matrix, int32 indices, sorted columns per row.
struct Csr {
  int nrows = 0, ncols = 0;
  std::vector<int> ptr, col;
  std::vector<double> val;
  int64_t nnz() const { return ptr.empty() ? 0 : ptr.back(); }
};

// All seven FEM operators share one sparsity pattern: every (i, j) node
// pair of every element (preproc/FEMprocessing.cpp:237-252, 256-286).
struct FemOperators {
  int nx = 0;
  std::vector<int> ptr, col;               // shared CSR pattern
  std::vector<double> stiff;               // K
  std::vector<double> grad[3];             // volume-averaged nodal gradient
  std::vector<double> tgrad[3];            // weak divergence (not negated)
  std::vector<double> node_vol;            // lumped node volume
  std::vector<double> elem_vol;
};

struct BoundaryData {
  std::vector<int> bnodes;                 // ascending global ids (Nb)
  std::vector<int> bindex;                 // N -> boundary index or -1
  std::vector<int> tri;                    // T x 3 global ids, ascending per triangle
  std::vector<int> tri_tet;                // owning tetrahedron
  std::vector<double> tri_area;            // T
  std::vector<double> tri_normal;          // T x 3 outward unit normal
  std::vector<double> node_area;           // N
  std::vector<double> node_normal;         // N x 3 (row-major), 0 off the boundary
  std::vector<double> solid_angle;         // Nb interior solid angle
};

struct MeshHost {
  int nx = 0, ntet = 0;
  std::vector<double> xyz;                 // N x 3 row-major
  std::vector<int> tets;                   // E x 4
  FemOperators fem;
  BoundaryData bnd;
};

// setup.cpp
void fem_prepare(MeshHost& m);
void extract_boundary(MeshHost& m);
void compute_solid_angles(MeshHost& m);
double solid_angle(const double* x, const double* t1, const double* t2, const double* t3);

// amg.cpp -- smoothed-aggregation hierarchy built on the host.
struct AmgLevel {
  Csr A;                                   // level operator
  Csr P;                                   // prolongation to this level from the next (n_l x n_{l+1})
  Csr R;                                   // restriction (P^T)
  std::vector<double> dinv;                // damped inverse diagonal for the Jacobi smoother
};

struct AmgParams {
  // strength threshold: AMGCL's default is 0.08; on Kuhn-split meshes 0.02 keeps the
  // face-diagonal couplings strong and cuts the Neumann PCG iterations about 3x (46 -> 15
  // on the 363,609-node film to 1e-7)
  double eps_strong = 0.02;
  // prolongation-smoother factor: tetmag gives AMGCL 0.75 (main/AMGCLSolver.cpp:40); 1.0 (Vanek's
  // 4/3 / rho) measured 3-17 % faster under the Jacobi V-cycle here (fewer PCG iterations)
  double relax = 1.0;
  // dense FP64 solve at or below this size: on the 363,609-node film the hierarchy then stops at
  // the 1,676-unknown level (one dense product instead of five latency-bound launches for the two
  // smallest levels per V-cycle)
  int coarse_enough = 2000;
  int max_levels = 12;
  // smoother damping, times 4 / (3 rho(D^-1 A)): 1.25 puts the weight at 1.67 / rho, below the 2 / rho
  // that keeps the symmetric V-cycle positive definite; measured fastest among 0.8-1.35 (fewer PCG
  // iterations; 1.35 gave more)
  double jacobi_omega = 1.25;
  bool singular = false;                   // operator annihilates constants (pure Neumann)
};

struct AmgHierarchy {
  std::vector<AmgLevel> levels;            // levels[0].A is the fine operator
  int ncoarse = 0;
  std::vector<double> coarse_inv;          // dense ncoarse x ncoarse inverse (row-major), FP64
  // when the coarsest level is too large for a dense inverse but only a few of its rows couple to
  // others (a row with no off-diagonal entry has a decoupled column too, the operator being
  // symmetric): coarse_inv inverts the submatrix of those rows, listed here (the level's row ids),
  // and every other row is solved exactly by its diagonal (coarse_diag_inv, one per level row).
  // Empty: coarse_inv covers all rows.
  std::vector<int> coarse_idx;
  std::vector<double> coarse_diag_inv;
  double setup_ms = 0.0;
};

void amg_build(const Csr& A, const AmgParams& prm, AmgHierarchy& H);

// hmatrix.cpp -- cluster tree and block partition of the boundary double-layer matrix.
struct HCluster {
  int begin, end;       // index range in the permuted boundary numbering
  double lo[3], hi[3];  // bounding box
  int child[2];         // -1 for leaves
};

struct HPartition {
  std::vector<int> perm;                     // permuted position -> boundary index
  std::vector<HCluster> clusters;            // clusters[0] is the root
  std::vector<std::pair<int, int>> near;     // inadmissible leaf pairs (row, col cluster)
  std::vector<std::pair<int, int>> far;      // admissible pairs -> low rank
};

// bnrm (Nb x 3 node normals, may be null) makes faces of different orientation separate first
void h_partition(const double* bxyz, const double* bnrm, int nb, int leaf, double eta, int max_block,
                 HPartition& P);
// h2.cpp -- recompression of the admissible blocks into nested cluster bases (H2).
struct H2Factors {                           // low-rank factors of P.far[q]: U (m x k), V (n x k)
  std::vector<const double*> U, V;           // column-major
  std::vector<int> ldu, ldv, rank;
};
struct H2Side {                              // cluster basis of one side (rows or columns)
  std::vector<int> k;                        // rank per cluster
  std::vector<std::vector<double>> leaf_basis;  // leaf clusters: |c| x k_c, column-major
  std::vector<std::vector<double>> transfer;    // non-root clusters: k_c x k_parent, column-major
};
struct H2Host {
  H2Side row, col;
  std::vector<std::vector<double>> coupling;    // per admissible block: k_row x k_col, column-major
};
// eps: relative truncation of each cluster's total matrix (H2Lib's releucl mode); kmax: rank cap
void h2_build_host(const HPartition& P, const H2Factors& F, double eps, int kmax, H2Host& out);

void csr_transpose(const Csr& A, Csr& T);
void csr_multiply(const Csr& A, const Csr& B, Csr& C);

}  // namespace tmb

namespace tmb {

// output.cpp -- run artefacts: VTU files, magnetisation restart files, .log columns.
int write_vtu(const std::string& path, int nx, const double* xyz, int ntet, const int* tets, const double* m,
              const int* material, double time_ps, const char* time_name, const double* field,
              const char* field_name, int binary, std::string& err);
int read_magnetization(const std::string& path, int nx, double* m, double* time_ps, std::string& err);
std::string log_header(const char* start_time, const char* host, const char* user);
std::string log_row(double t_ps, const double e[8], double torque, const double mean_m[3], const double mean_h_t[3]);

}  // namespace tmb
