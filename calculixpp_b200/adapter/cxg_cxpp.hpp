// CalculiX++ adapter over libcxg: the reference's assembly entry points with the element
// integration and CSR assembly on the GPU, returning the reference's own LinearSystem so
// its solve / expansion / recovery code consumes the result unchanged.
//
// A maintainer adds this header and cxg_cxpp.cpp to src/compute/ and links
// calculixpp_b200/_lib/libcxg.so. Replaces, for models the GPU path supports:
//   fem::assemble_linear_static      include/calculixpp/fem/assembly.hpp:42
//   fem::make_material_points        include/calculixpp/fem/assembly.hpp:93
//   fem::assemble_material_tangent   include/calculixpp/fem/assembly.hpp:105-108
//   numerics::solve_linear_static    include/calculixpp/numerics/linear_static.hpp
// Supported: one element type per model (C3D4/C3D10/C3D8/C3D8R/C3D20/C3D20R/C3D6/C3D15),
// per-element sections and materials (elastic, J2 plasticity), *BOUNDARY single-point
// constraints, *EQUATION and the other constraints the reference expands into linear
// equations (through its own constraint transform), *CLOAD/*DLOAD/*GRAV loads through
// external_load_vector, thermal strain (*EXPANSION with applied temperatures),
// deactivated elements (*MODEL CHANGE). Anything else (several element types, springs,
// hyperelastic or user materials) throws
// std::runtime_error naming the feature, before any GPU work.
#pragma once

#include <optional>
#include <vector>

#include "calculixpp/compute/backend.hpp"
#include "calculixpp/fem/assembly.hpp"
#include "calculixpp/numerics/linear_static.hpp"
#include "cxg.h"

namespace cxg_cxpp {

enum class Precision { FP64 = CXG_FP64, Mixed = CXG_MIXED };

// A model resident on the GPU: mesh, DOF map and CSR pattern built once; every
// assembly afterwards is two kernel passes plus the copies back to the host. The J2
// history of the material-point assembly lives in the plan (committed and trial).
class CudaAssembler {
 public:
  explicit CudaAssembler(const cxpp::Model& model, Precision precision = Precision::FP64);
  ~CudaAssembler();
  CudaAssembler(const CudaAssembler&) = delete;
  CudaAssembler& operator=(const CudaAssembler&) = delete;

  // assemble_linear_static (src/fem/assembly.cpp:225-257): K_ff as COO triplets in
  // (row, column) order with duplicates summed, rhs = T^T f_ext - K_fc u_c.
  cxpp::fem::LinearSystem assemble_linear_static();
  // assemble_material_tangent (src/fem/assembly.cpp:385-423) at the full nodal
  // displacement u; advances the trial history, fills f_int[3N].
  cxpp::fem::LinearSystem assemble_material_tangent(const std::vector<cxpp::Vec3>& u,
                                                    std::vector<cxpp::Real>& f_int);
  // MaterialPoints::commit (include/calculixpp/fem/assembly.hpp:84-87).
  void commit();
  // The history of every Gauss point in element order, 13 doubles each (committed or
  // trial), as MaterialState holds it (include/calculixpp/fem/material_model.hpp:38-64).
  std::vector<double> state(bool committed) const;

  cxg_plan* plan() const { return plan_; }

 private:
  cxpp::fem::LinearSystem system_from_csr(const std::vector<double>& vals, std::vector<double> rhs) const;

  const cxpp::Model& model_;
  cxg_plan* plan_ = nullptr;
  cxpp::fem::LinearSystem base_;      // DOF map, prescribed values, transform
  std::vector<double> f_ext_;         // external_load_vector(model)
  std::vector<int64_t> row_ptr_;
  std::vector<int32_t> col_idx_;
  std::vector<int64_t> active_;       // mesh element index of every plan element
};

// ComputeBackend (include/calculixpp/compute/backend.hpp:40-57) on the GPU: solve_sparse
// through cxg_solve_sparse, the COO triplets of a LinearSystem in, x out. SolverKind::Direct
// is a sparse Cholesky on the device; SolverKind::CG is the device's Jacobi-preconditioned
// CG to a relative residual of 1e-10 (the CPU backend uses IC0), throwing
// std::runtime_error("CG did not converge ...") like the CPU backend
// (src/compute/cpu_backend.cpp:57-62). select_backend(BackendKind::CUDA) would return it.
class CudaBackend : public cxpp::compute::ComputeBackend {
 public:
  cxpp::compute::BackendKind kind() const override { return cxpp::compute::BackendKind::CUDA; }
  std::vector<cxpp::Real> solve_sparse(const std::vector<cxpp::Index>& rows, const std::vector<cxpp::Index>& cols,
                                       const std::vector<cxpp::Real>& vals, cxpp::Index n,
                                       const std::vector<cxpp::Real>& rhs,
                                       cxpp::compute::SolverKind solver) const override;
};
const cxpp::compute::ComputeBackend& cuda_backend();

// One-shot form of CudaAssembler::assemble_linear_static with the reference's signature.
cxpp::fem::LinearSystem assemble_linear_static_cuda(const cxpp::Model& model,
                                                    Precision precision = Precision::FP64);

// numerics::solve_linear_static (src/numerics/linear_static.cpp:29-50) with the
// assembly on the GPU: the same solver choice, the solve through the compute backend
// (the selected one, as solve_reduced does, or cuda_backend() when gpu_solve), expansion
// through the constraint transform and field recovery.
cxpp::StaticFields solve_linear_static_cuda(const cxpp::Model& model,
                                            std::optional<cxpp::numerics::SolverKind> forced = std::nullopt,
                                            Precision precision = Precision::FP64, bool gpu_solve = false);

}  // namespace cxg_cxpp
