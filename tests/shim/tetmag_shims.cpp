// The reference-side shims of INTEGRATION.md, compiled against include/tmb.h and linked to
// libtmb.so, with minimal stand-ins for the tetmag types they use (Eigen's RowMajor SpMat and
// VectorXd, the SolverFactory base class, SUNDIALS' N_Vector and CVODE's callback signature).
//
// Usage: tetmag_shims <input.bin> <output.bin>
//   input:  int32 nx, int32 ntet, nx*3 double xyz, ntet*4 int32 tets, 3*nx double m (SoA),
//           nx double load vector b
//   output: 3*nx double H_dem (DemagField::calcField through the C ABI),
//           3*nx double ydot (TheLLG::rhs, CVODE signature, host N_Vectors),
//           3*nx double ydot (TheLLG::rhs_d, CVODE signature, device N_Vectors),
//           nx double x (B200Solver on the row-pinned Neumann matrix, load b),
//           3 double solver info (iterations, relative residual, status)
// Exit code 0 when every call returned TMB_OK and every shim reported success.
//
// Test harness: tests/test_dropin.py compiles this file (CPU test) and runs it on a GPU, then
// checks the outputs against the FP64 oracle.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include "tmb.h"

// ---------------------------------------------------------------------------------------------
// Stand-ins for the tetmag / Eigen / SUNDIALS types the shims touch (only what they call).
// ---------------------------------------------------------------------------------------------
struct VectorXd {  // Eigen::VectorXd
  std::vector<double> v;
  void resize(long n) { v.assign(size_t(n), 0.0); }
  long size() const { return long(v.size()); }
  double* data() { return v.data(); }
  const double* data() const { return v.data(); }
  bool allFinite() const {
    for (double a : v)
      if (!std::isfinite(a)) return false;
    return true;
  }
};

struct SpMat {  // Eigen::SparseMatrix<double, RowMajor> (utils/typedefs.h:35), compressed
  int n = 0;
  std::vector<int> outer, inner;
  std::vector<double> val;
  int rows() const { return n; }
  int nonZeros() const { return int(val.size()); }
  const int* outerIndexPtr() const { return outer.data(); }
  const int* innerIndexPtr() const { return inner.data(); }
  const double* valuePtr() const { return val.data(); }
  void makeCompressed() {}
};

class SolverFactory {  // main/SolverFactory.h:42-65 (the members the b200 case uses)
 public:
  virtual ~SolverFactory() = default;
  void setMatrix(const SpMat& m) { A = m; }
  void setLoadVector(const VectorXd& v) { b = v; }
  void setCGTolerance(double t) { cgTol = t; }
  virtual bool compute() = 0;
  virtual void solve() = 0;
  virtual bool wasSuccessful() = 0;
  virtual void report() = 0;
  VectorXd result() const { return x; }

 protected:
  SpMat A, Ar;
  VectorXd b, x;
  double cgTol = 1e-7;
};

typedef double realtype;
struct NVectorContent {  // NVECTOR_SERIAL / NVECTOR_CUDA: one data pointer per vector
  double* host = nullptr;
  double* device = nullptr;
};
typedef NVectorContent* N_Vector;
static double* NV_DATA_S(N_Vector v) { return v->host; }
static double* N_VGetDeviceArrayPointer_Cuda(N_Vector v) { return v->device; }

struct UserData {  // main/TheLLG.h:177-181, with the library context added
  tmb_ctx* ctx;
};

// ---------------------------------------------------------------------------------------------
// the "b200" case of SolverFactory::makeSolver
// ---------------------------------------------------------------------------------------------
class B200Solver : public SolverFactory {
  tmb_ctx* ctx_;
  tmb_solver* s_ = nullptr;

 public:
  explicit B200Solver(tmb_ctx* ctx) : ctx_(ctx) { tmb_solver_create(ctx_, &s_); }
  ~B200Solver() override { tmb_solver_destroy(s_); }
  bool compute() override {
    Ar = A;
    Ar.makeCompressed();
    if (tmb_solver_set_matrix(s_, Ar.rows(), Ar.nonZeros(), Ar.outerIndexPtr(), Ar.innerIndexPtr(),
                              Ar.valuePtr()) != TMB_OK)
      return false;
    tmb_solver_set_tolerance(s_, cgTol, 300);
    return tmb_solver_compute(s_) == TMB_OK;
  }
  void solve() override {
    x.resize(b.size());
    last_ = tmb_solver_solve(s_, b.data(), x.data(), TMB_PTR_HOST);
  }
  bool wasSuccessful() override { return last_ == TMB_OK && x.allFinite(); }
  void report() override {
    double info[3];
    tmb_solver_info(s_, info);
    std::cout << "b200 PCG+AMG: " << info[0] << " iterations, residual " << info[1] << std::endl;
  }
  void info(double* out) { tmb_solver_info(s_, out); }

 private:
  int last_ = TMB_OK;
};

static std::shared_ptr<SolverFactory> makeSolver(const std::string& type, tmb_ctx* ctx) {
  if (type == "b200") return std::make_shared<B200Solver>(ctx);
  return nullptr;
}

// ---------------------------------------------------------------------------------------------
// the CVODE right-hand sides
// ---------------------------------------------------------------------------------------------
static int rhs(realtype t, N_Vector u, N_Vector u_dot, void* user_data) {  // TheLLG::rhs
  auto* d = static_cast<UserData*>(user_data);
  return tmb_llg_rhs(d->ctx, t, NV_DATA_S(u), NV_DATA_S(u_dot), TMB_PTR_HOST) == TMB_OK ? 0 : -1;
}

static int rhs_d(realtype t, N_Vector u, N_Vector u_dot, void* user_data) {  // TheLLG::rhs_d
  auto* d = static_cast<UserData*>(user_data);
  const double* y = N_VGetDeviceArrayPointer_Cuda(u);
  double* ydot = N_VGetDeviceArrayPointer_Cuda(u_dot);
  return tmb_llg_rhs(d->ctx, t, y, ydot, TMB_PTR_DEVICE) == TMB_OK ? 0 : -1;
}

// ---------------------------------------------------------------------------------------------
#define CHECK(call)                                                                   \
  do {                                                                                \
    const int rc_ = (call);                                                           \
    if (rc_ != TMB_OK) {                                                              \
      std::fprintf(stderr, "%s failed: %d %s\n", #call, rc_, tmb_last_error());       \
      return 2;                                                                       \
    }                                                                                 \
  } while (0)

template <typename T>
static bool read_n(FILE* f, T* p, size_t n) {
  return std::fread(p, sizeof(T), n, f) == n;
}

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
    return 1;
  }
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 1;
  int nx = 0, ntet = 0;
  if (!read_n(f, &nx, 1) || !read_n(f, &ntet, 1) || nx <= 0 || ntet <= 0) return 1;
  std::vector<double> xyz(size_t(3) * nx), m(size_t(3) * nx), bload(nx);
  std::vector<int> tets(size_t(4) * ntet);
  if (!read_n(f, xyz.data(), xyz.size()) || !read_n(f, tets.data(), tets.size()) ||
      !read_n(f, m.data(), m.size()) || !read_n(f, bload.data(), bload.size()))
    return 1;
  std::fclose(f);

  // tetmag's MeshData (specs/MeshData.h:41-63): K, grad*, tGrad* on one CSR pattern, node
  // volumes, boundary nodes, node areas and normals -- here from the library's preprocessing
  tmb_mesh* mesh = nullptr;
  CHECK(tmb_mesh_create(nx, ntet, xyz.data(), tets.data(), &mesh));
  long long info[6];
  CHECK(tmb_mesh_info(mesh, info));
  const int nnz = int(info[2]), nb = int(info[3]), ntri = int(info[4]);
  SpMat K;
  K.n = nx;
  K.outer.resize(nx + 1);
  K.inner.resize(nnz);
  K.val.resize(nnz);
  std::vector<double> gx(nnz), gy(nnz), gz(nnz), tgx(nnz), tgy(nnz), tgz(nnz), vol(nx);
  CHECK(tmb_mesh_get_operators(mesh, K.outer.data(), K.inner.data(), K.val.data(), gx.data(), gy.data(),
                               gz.data(), tgx.data(), tgy.data(), tgz.data(), vol.data()));
  std::vector<int> bnodes(nb), tri(size_t(3) * ntri);
  std::vector<double> area(nx), normal(size_t(3) * nx);
  CHECK(tmb_mesh_get_boundary(mesh, bnodes.data(), tri.data(), nullptr, nullptr, area.data(), normal.data(),
                              nullptr));

  // DemagField::initializeSolvers with solverType == "b200" 
  tmb_ctx* ctx = nullptr;
  CHECK(tmb_ctx_create(0, &ctx));
  CHECK(tmb_set_operators(ctx, nx, K.nonZeros(), K.outerIndexPtr(), K.innerIndexPtr(), K.valuePtr(), gx.data(),
                          gy.data(), gz.data(), tgx.data(), tgy.data(), tgz.data(), vol.data(), nb, bnodes.data(),
                          area.data(), normal.data()));
  CHECK(tmb_bem_assemble(ctx, mesh));
  const double mu0 = 1.256637061435917295376e-6;
  std::vector<double> Js(nx, mu0 * 8.0e5), A(nx, 1.3e-11 / 1e-18);
  CHECK(tmb_set_material(ctx, Js.data(), A.data(), nullptr, nullptr, nullptr, 0.5));
  CHECK(tmb_set_solver_params(ctx, 1e-13, 300));

  // DemagField::calcField (host matrices, column-major N x 3)
  std::vector<double> H(size_t(3) * nx), ydot_h(size_t(3) * nx), ydot_d(size_t(3) * nx);
  CHECK(tmb_demag_field(ctx, m.data(), H.data(), TMB_PTR_HOST));

  // CVODE callbacks, host and device N_Vectors
  UserData ud{ctx};
  NVectorContent y{m.data(), nullptr}, yd{ydot_h.data(), nullptr};
  if (rhs(0.0, &y, &yd, &ud) != 0) return 3;
  double *dy = nullptr, *dydot = nullptr;
  if (cudaMalloc(&dy, m.size() * sizeof(double)) != cudaSuccess) return 4;
  if (cudaMalloc(&dydot, m.size() * sizeof(double)) != cudaSuccess) return 4;
  cudaMemcpy(dy, m.data(), m.size() * sizeof(double), cudaMemcpyHostToDevice);
  NVectorContent yv{nullptr, dy}, ydv{nullptr, dydot};
  if (rhs_d(0.0, &yv, &ydv, &ud) != 0) return 3;
  cudaDeviceSynchronize();
  cudaMemcpy(ydot_d.data(), dydot, m.size() * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(dy);
  cudaFree(dydot);

  // SolverFactory::makeSolver("b200") on the Neumann matrix: K with row N/2 replaced by the
  // unit row (DemagField::prepareNeumannMatrix, main/DemagField.cpp:204-220)
  SpMat Kn;
  Kn.n = nx;
  Kn.outer.assign(1, 0);
  const int pin = nx / 2;
  for (int i = 0; i < nx; ++i) {
    if (i == pin) {
      Kn.inner.push_back(i);
      Kn.val.push_back(1.0);
    } else {
      for (int q = K.outer[i]; q < K.outer[i + 1]; ++q) {
        Kn.inner.push_back(K.inner[q]);
        Kn.val.push_back(K.val[q]);
      }
    }
    Kn.outer.push_back(int(Kn.inner.size()));
  }
  auto solver = makeSolver("b200", ctx);
  if (!solver) return 5;
  solver->setMatrix(Kn);
  solver->setCGTolerance(1e-13);
  if (!solver->compute()) return 5;
  VectorXd bv;
  bv.v = bload;
  solver->setLoadVector(bv);
  solver->solve();
  if (!solver->wasSuccessful()) return 6;
  solver->report();
  double sinfo[3];
  static_cast<B200Solver*>(solver.get())->info(sinfo);
  const VectorXd xs = solver->result();

  FILE* o = std::fopen(argv[2], "wb");
  if (!o) return 1;
  std::fwrite(H.data(), sizeof(double), H.size(), o);
  std::fwrite(ydot_h.data(), sizeof(double), ydot_h.size(), o);
  std::fwrite(ydot_d.data(), sizeof(double), ydot_d.size(), o);
  std::fwrite(xs.data(), sizeof(double), size_t(nx), o);
  std::fwrite(sinfo, sizeof(double), 3, o);
  std::fclose(o);
  solver.reset();
  tmb_ctx_destroy(ctx);
  tmb_mesh_destroy(mesh);
  return 0;
}
