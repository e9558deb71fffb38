// Test-infrastructure stand-in for the reference's compute backend (the reference's own
// src/compute/cpu_backend.cpp needs the SciPP/NumPP libraries, which are not available
// here). It provides the same functions that include/calculixpp/compute/backend.hpp
// declares, with a dense solve: Cholesky for the SPD reduced stiffness, falling back to
// partial-pivoting LU. Only meant for the small (<= a few thousand DOF) models the
// oracle drives through the reference's numerics drivers (sensitivity, Newton); both
// the reference operator and any operator compared against it use this same solve.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "calculixpp/compute/backend.hpp"

namespace cxpp::compute {
namespace {

std::vector<Real> dense_solve(std::vector<Real> A, std::vector<Real> b, std::size_t n) {
  // Cholesky attempt on a copy; LU with partial pivoting if a pivot is not positive.
  std::vector<Real> L = A;
  bool spd = true;
  for (std::size_t j = 0; j < n && spd; ++j) {
    Real d = L[j * n + j];
    for (std::size_t k = 0; k < j; ++k) d -= L[j * n + k] * L[j * n + k];
    if (!(d > 0.0)) { spd = false; break; }
    const Real ljj = std::sqrt(d);
    L[j * n + j] = ljj;
    for (std::size_t i = j + 1; i < n; ++i) {
      Real s = L[i * n + j];
      for (std::size_t k = 0; k < j; ++k) s -= L[i * n + k] * L[j * n + k];
      L[i * n + j] = s / ljj;
    }
  }
  if (spd) {
    std::vector<Real> y(n);
    for (std::size_t i = 0; i < n; ++i) {
      Real s = b[i];
      for (std::size_t k = 0; k < i; ++k) s -= L[i * n + k] * y[k];
      y[i] = s / L[i * n + i];
    }
    std::vector<Real> x(n);
    for (std::size_t ii = n; ii-- > 0;) {
      Real s = y[ii];
      for (std::size_t k = ii + 1; k < n; ++k) s -= L[k * n + ii] * x[k];
      x[ii] = s / L[ii * n + ii];
    }
    return x;
  }
  std::vector<std::size_t> piv(n);
  for (std::size_t i = 0; i < n; ++i) piv[i] = i;
  for (std::size_t j = 0; j < n; ++j) {
    std::size_t p = j;
    for (std::size_t i = j + 1; i < n; ++i)
      if (std::fabs(A[i * n + j]) > std::fabs(A[p * n + j])) p = i;
    if (A[p * n + j] == 0.0) throw std::runtime_error("singular reduced operator");
    if (p != j) {
      for (std::size_t k = 0; k < n; ++k) std::swap(A[j * n + k], A[p * n + k]);
      std::swap(b[j], b[p]);
    }
    for (std::size_t i = j + 1; i < n; ++i) {
      const Real f = A[i * n + j] / A[j * n + j];
      A[i * n + j] = f;
      for (std::size_t k = j + 1; k < n; ++k) A[i * n + k] -= f * A[j * n + k];
      b[i] -= f * b[j];
    }
  }
  std::vector<Real> x(n);
  for (std::size_t ii = n; ii-- > 0;) {
    Real s = b[ii];
    for (std::size_t k = ii + 1; k < n; ++k) s -= A[ii * n + k] * x[k];
    x[ii] = s / A[ii * n + ii];
  }
  return x;
}

class DenseStandInBackend final : public ComputeBackend {
 public:
  BackendKind kind() const override { return BackendKind::CPU; }
  std::vector<Real> solve_sparse(const std::vector<Index>& rows,
                                 const std::vector<Index>& cols,
                                 const std::vector<Real>& vals, Index n,
                                 const std::vector<Real>& rhs,
                                 SolverKind /*solver*/) const override {
    const std::size_t m = static_cast<std::size_t>(n);
    if (m > 6000) throw std::runtime_error("dense stand-in solve limited to 6000 DOF");
    std::vector<Real> A(m * m, 0.0);
    for (std::size_t k = 0; k < vals.size(); ++k)
      A[static_cast<std::size_t>(rows[k]) * m + static_cast<std::size_t>(cols[k])] += vals[k];
    return dense_solve(std::move(A), rhs, m);
  }
};

}  // namespace

std::string backend_name(BackendKind kind) {
  switch (kind) {
    case BackendKind::CPU: return "cpu";
    case BackendKind::CUDA: return "cuda";
    case BackendKind::OpenCL: return "opencl";
    case BackendKind::Metal: return "metal";
  }
  return "cpu";
}

BackendKind backend_kind(const std::string& name) {
  std::string s = name;
  for (char& c : s) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
  if (s == "cpu") return BackendKind::CPU;
  if (s == "cuda") return BackendKind::CUDA;
  if (s == "opencl") return BackendKind::OpenCL;
  if (s == "metal") return BackendKind::Metal;
  throw std::invalid_argument("unknown compute backend: '" + name + "'");
}

bool backend_available(BackendKind kind) { return kind == BackendKind::CPU; }
std::vector<BackendKind> available_backends() { return {BackendKind::CPU}; }

const ComputeBackend& cpu_backend() {
  static const DenseStandInBackend backend;
  return backend;
}

const ComputeBackend& select_backend(BackendKind /*requested*/) { return cpu_backend(); }

}  // namespace cxpp::compute
