// TEST INFRASTRUCTURE ONLY: C entry points that run the reference's own drivers with the
// CUDA adapter (calculixpp_b200/adapter/cxg_cxpp.cpp) in place of its CPU assembly, and
// the same drivers all on the CPU, on a Model built by ref_model_create (ref_shim.cpp).
// Built by `make -C oracle adapter` into oracle/_ref/libcxg_cxpp_test.so.
#include <cstring>
#include <stdexcept>
#include <string>

#include "calculixpp/fem/assembly.hpp"
#include "calculixpp/numerics/linear_static.hpp"
#include "cxg_cxpp.hpp"

extern "C" const cxpp::Model* ref_model_get(void* model);

namespace {
thread_local std::string g_err;

int fail(const std::exception& e) {
  g_err = e.what();
  return -1;
}

void copy_system(const cxpp::fem::LinearSystem& s, int32_t* rows, int32_t* cols, double* vals, double* rhs) {
  std::memcpy(rows, s.rows.data(), s.rows.size() * sizeof(int32_t));
  std::memcpy(cols, s.cols.data(), s.cols.size() * sizeof(int32_t));
  std::memcpy(vals, s.vals.data(), s.vals.size() * sizeof(double));
  std::memcpy(rhs, s.rhs.data(), s.rhs.size() * sizeof(double));
}
}  // namespace

extern "C" {

const char* cuda_last_error(void) { return g_err.c_str(); }

// numerics::solve_linear_static (gpu = 0: all on the CPU; 1: the assembly through the
// adapter; 2: the assembly and the solve on the GPU, through CudaBackend). solver 0
// direct, 1 CG. u[3N] displacement, stress[6N] averaged nodal stress.
int cuda_solve_linear_static(void* model, int gpu, int precision, int solver, double* u, double* stress) {
  try {
    const cxpp::Model& m = *ref_model_get(model);
    const auto kind = solver ? cxpp::numerics::SolverKind::CG : cxpp::numerics::SolverKind::Direct;
    const cxpp::StaticFields r =
        gpu ? cxg_cxpp::solve_linear_static_cuda(m, kind, static_cast<cxg_cxpp::Precision>(precision), gpu == 2)
            : cxpp::numerics::solve_linear_static(m, kind);
    for (std::size_t i = 0; i < r.displacement.size(); ++i)
      for (int d = 0; d < 3; ++d) u[3 * i + d] = r.displacement[i][static_cast<std::size_t>(d)];
    if (stress)
      for (std::size_t i = 0; i < r.stress.size(); ++i)
        for (int d = 0; d < 6; ++d) stress[6 * i + d] = r.stress[i][static_cast<std::size_t>(d)];
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// CudaBackend::solve_sparse on COO triplets (solver 0 direct, 1 CG).
int cuda_backend_solve(int32_t n, int64_t nnz, const int32_t* rows, const int32_t* cols, const double* vals,
                       const double* rhs, int solver, double* x) {
  try {
    const std::vector<cxpp::Index> r(rows, rows + nnz), c(cols, cols + nnz);
    const std::vector<cxpp::Real> v(vals, vals + nnz), b(rhs, rhs + n);
    const std::vector<cxpp::Real> sol = cxg_cxpp::cuda_backend().solve_sparse(
        r, c, v, n, b, solver ? cxpp::compute::SolverKind::CG : cxpp::compute::SolverKind::Direct);
    std::memcpy(x, sol.data(), sizeof(double) * static_cast<std::size_t>(n));
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// A CudaAssembler on the model; null on error (message in cuda_last_error).
void* cuda_assembler_create(void* model, int precision) {
  try {
    return new cxg_cxpp::CudaAssembler(*ref_model_get(model), static_cast<cxg_cxpp::Precision>(precision));
  } catch (const std::exception& e) {
    fail(e);
    return nullptr;
  }
}

void cuda_assembler_free(void* a) { delete static_cast<cxg_cxpp::CudaAssembler*>(a); }

// Triplet count and free-equation count of the assembler's systems.
int cuda_assembler_sizes(void* a, int64_t* nnz, int64_t* n_free) {
  cxg_plan_info info{};
  if (cxg_plan_get_info(static_cast<cxg_cxpp::CudaAssembler*>(a)->plan(), &info) != CXG_OK) {
    g_err = cxg_last_error();
    return -1;
  }
  *nnz = info.nnz;
  *n_free = info.n_free;
  return 0;
}

// assemble_linear_static through the adapter into arrays of cuda_assembler_sizes.
int cuda_assemble_linear(void* a, int32_t* rows, int32_t* cols, double* vals, double* rhs) {
  try {
    copy_system(static_cast<cxg_cxpp::CudaAssembler*>(a)->assemble_linear_static(), rows, cols, vals, rhs);
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// assemble_material_tangent through the adapter at the full displacement u[3 n_nodes];
// f_int[3 n_nodes]; commit != 0 commits the history afterwards. Arrays sized as
// cuda_assembler_sizes reports (the pattern is the same).
int cuda_assemble_tangent(void* a, int64_t n_nodes, const double* u, int32_t* rows, int32_t* cols, double* vals,
                          double* rhs, double* f_int, int commit) {
  try {
    auto* asmb = static_cast<cxg_cxpp::CudaAssembler*>(a);
    std::vector<cxpp::Vec3> uu(static_cast<std::size_t>(n_nodes));
    for (std::size_t i = 0; i < uu.size(); ++i) uu[i] = {u[3 * i], u[3 * i + 1], u[3 * i + 2]};
    std::vector<cxpp::Real> f;
    const cxpp::fem::LinearSystem s = asmb->assemble_material_tangent(uu, f);
    copy_system(s, rows, cols, vals, rhs);
    std::memcpy(f_int, f.data(), f.size() * sizeof(double));
    if (commit) asmb->commit();
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

}  // extern "C"
