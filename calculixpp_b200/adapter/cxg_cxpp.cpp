// CalculiX++ adapter over libcxg (see cxg_cxpp.hpp).
#include "cxg_cxpp.hpp"

#include <cstring>
#include <stdexcept>
#include <string>

#include "calculixpp/fem/constraint_transform.hpp"
#include "calculixpp/fem/loads.hpp"
#include "calculixpp/fem/stress.hpp"

namespace cxg_cxpp {
namespace {

void check(int rc) {
  if (rc != CXG_OK) throw std::runtime_error(cxg_last_error());
}

void unsupported(const std::string& what) {
  throw std::runtime_error("CUDA assembly: " + what + " is not supported; use the CPU assembly");
}

// The DOF map of build_dof_map (src/fem/assembly.cpp:19-42): SPC flags and values in
// global-DOF order, then the reference's own constraint transform, so the free
// numbering, prescribed values and amplitudes are the reference's by construction.
void build_dof_map(const cxpp::Model& model, cxpp::fem::LinearSystem& sys) {
  const cxpp::Mesh& mesh = model.mesh;
  const std::size_t n_dof = mesh.num_nodes() * cxpp::kDofsPerNode;
  sys.prescribed.assign(n_dof, 0.0);
  sys.prescribed_amp.assign(n_dof, std::string{});
  std::vector<bool> constrained(n_dof, false);
  for (const cxpp::Spc& spc : model.spcs) {
    const cxpp::Index ni = mesh.node_index(spc.node_id);
    if (ni < 0) throw std::runtime_error("*BOUNDARY references unknown node");
    if (spc.comp < 1 || spc.comp > cxpp::kDofsPerNode) throw std::runtime_error("*BOUNDARY dof out of range");
    const std::size_t g = static_cast<std::size_t>(ni) * cxpp::kDofsPerNode + static_cast<std::size_t>(spc.comp - 1);
    constrained[g] = true;
    sys.prescribed[g] = spc.value;
    sys.prescribed_amp[g] = spc.amplitude;
  }
  sys.transform = cxpp::fem::build_constraint_transform(model, constrained, sys.prescribed);
  sys.dof_eq = sys.transform.dof_eq;
  sys.n_free = sys.transform.n_free;
  sys.rhs.assign(static_cast<std::size_t>(sys.n_free), 0.0);
}

bool same_table(const cxpp::Plastic& a, const cxpp::Plastic& b) {
  return a.hardening == b.hardening && a.kinematic_modulus == b.kinematic_modulus && a.eqplastic == b.eqplastic &&
         a.yield == b.yield;
}

}  // namespace

CudaAssembler::CudaAssembler(const cxpp::Model& model, Precision precision) : model_(model) {
  const cxpp::Mesh& mesh = model.mesh;
  build_dof_map(model, base_);
  // multi-point constraints: the slaves' expansions of the reference's own transform
  std::vector<int64_t> slave_dof, term_ptr(1, 0);
  std::vector<int32_t> term_eq;
  std::vector<double> term_coeff, constant;
  for (std::size_t g = 0; g < base_.transform.is_slave.size(); ++g) {
    if (!base_.transform.is_slave[g]) continue;
    const cxpp::fem::DofExpansion& ex = base_.transform.expansion[g];
    slave_dof.push_back(static_cast<int64_t>(g));
    for (const cxpp::fem::DofTerm& t : ex.terms) {
      term_eq.push_back(t.eq);
      term_coeff.push_back(t.coeff);
    }
    term_ptr.push_back(static_cast<int64_t>(term_eq.size()));
    constant.push_back(ex.constant);
  }
  if (!model.springs.empty()) unsupported("*SPRING connectors");

  const std::vector<bool> active = model.element_active_mask();
  const std::vector<cxpp::ElasticIso> elastic = model.element_elastic();
  const std::vector<std::optional<cxpp::Plastic>> plastic = model.element_plastic();
  const auto hyper = model.element_hyperelastic();
  const auto user = model.element_user_material();
  int type = -1;
  for (std::size_t e = 0; e < mesh.num_elements(); ++e) {
    if (!active[e]) continue;  // *MODEL CHANGE, REMOVE: no stiffness, no internal force
    const int t = static_cast<int>(mesh.elements()[e].type);
    if (type >= 0 && t != type) unsupported("a mesh of several element types");
    if (hyper[e] || user[e]) unsupported("a hyperelastic or user material");
    type = t;
    active_.push_back(static_cast<int64_t>(e));
  }
  if (type < 0) type = mesh.num_elements() ? static_cast<int>(mesh.elements()[0].type) : 2;
  if (cxg_nodes_per_element(type) <= 0) unsupported("this element type");
  const int npe = cxg_nodes_per_element(type);

  std::vector<double> coords(3 * mesh.num_nodes());
  for (std::size_t i = 0; i < mesh.num_nodes(); ++i)
    for (int d = 0; d < 3; ++d) coords[3 * i + d] = mesh.nodes()[i].x[static_cast<std::size_t>(d)];
  const std::size_t E = active_.size();
  std::vector<int32_t> conn(E * npe), elem_mat(E);
  std::vector<double> young(E), poisson(E);
  // materials: one per distinct *PLASTIC table (an elastic one first); E and nu come
  // per element from the sections (Model::element_elastic, src/core/model.cpp:33-87)
  std::vector<cxpp::Plastic> tables;
  std::vector<cxg_material> mats(1, cxg_material{1.0, 0.3, 0, nullptr, nullptr, 0, 0.0});
  for (std::size_t k = 0; k < E; ++k) {
    const std::size_t e = static_cast<std::size_t>(active_[k]);
    const cxpp::Element& el = mesh.elements()[e];
    if (static_cast<int>(el.nodes.size()) != npe) throw std::runtime_error("element has the wrong node count");
    for (int i = 0; i < npe; ++i) {
      const cxpp::Index ni = mesh.node_index(el.nodes[static_cast<std::size_t>(i)]);
      if (ni < 0) throw std::runtime_error("element references unknown node");
      conn[k * npe + i] = ni;
    }
    young[k] = elastic[e].E;
    poisson[k] = elastic[e].nu;
    int m = 0;
    if (plastic[e] && !plastic[e]->empty()) {
      m = -1;
      for (std::size_t j = 0; j < tables.size(); ++j)
        if (same_table(tables[j], *plastic[e])) m = static_cast<int>(j) + 1;
      if (m < 0) {
        tables.push_back(*plastic[e]);
        m = static_cast<int>(tables.size());
      }
    }
    elem_mat[k] = m;
  }
  for (const cxpp::Plastic& p : tables) {
    cxg_material cm{1.0, 0.3, static_cast<int32_t>(p.yield.size()), p.eqplastic.data(), p.yield.data(),
                    p.hardening == cxpp::Plastic::Hardening::Kinematic ? 1
                    : p.hardening == cxpp::Plastic::Hardening::Combined ? 2
                                                                        : 0,
                    p.kinematic_modulus};
    mats.push_back(cm);
  }
  std::vector<int32_t> dof_eq(base_.dof_eq.begin(), base_.dof_eq.end());
  cxg_mesh_desc desc{static_cast<int64_t>(mesh.num_nodes()), static_cast<int64_t>(E), type, coords.data(),
                     conn.data(), young.data(), poisson.data(), elem_mat.data(), static_cast<int32_t>(mats.size()),
                     mats.data()};
  cxg_dofmap_desc dmap{dof_eq.data(), base_.prescribed.data(), base_.n_free};
  const cxg_mpc_desc mpc{static_cast<int64_t>(slave_dof.size()), slave_dof.data(), term_ptr.data(), term_eq.data(),
                         term_coeff.data(), constant.data()};
  check(cxg_plan_create_mpc(&desc, &dmap, &mpc, static_cast<int32_t>(precision), &plan_));
  cxg_plan_info info{};
  check(cxg_plan_get_info(plan_, &info));
  row_ptr_.resize(static_cast<std::size_t>(info.n_free) + 1);
  col_idx_.resize(static_cast<std::size_t>(info.nnz));
  check(cxg_plan_get_pattern(plan_, row_ptr_.data(), col_idx_.data()));
  f_ext_ = cxpp::fem::external_load_vector(model);

  // thermal strain (*EXPANSION with applied temperatures): the reference's own inputs,
  // alpha evaluated at each element's mean temperature (the nodes without an applied
  // temperature counting as t_ref, element_alpha, src/fem/stress.cpp:97-105)
  if (model.has_thermal_strain()) {
    const std::size_t N = mesh.num_nodes();
    std::vector<double> node_temp(N, 0.0), alpha(E, 0.0), tref(E, 0.0);
    std::vector<uint8_t> applied(N, 0);
    for (const auto& [id, t] : model.applied_temperature) {
      const cxpp::Index ni = mesh.node_index(id);
      if (ni < 0) continue;
      node_temp[static_cast<std::size_t>(ni)] = t;
      applied[static_cast<std::size_t>(ni)] = 1;
    }
    const std::vector<std::optional<cxpp::Expansion>> expansion = model.element_expansion();
    for (std::size_t k = 0; k < E; ++k) {
      const std::optional<cxpp::Expansion>& ex = expansion[static_cast<std::size_t>(active_[k])];
      if (!ex || ex->empty()) continue;
      double tsum = 0.0;
      for (int i = 0; i < npe; ++i) {
        const std::size_t ni = static_cast<std::size_t>(conn[k * npe + i]);
        tsum += applied[ni] ? node_temp[ni] : ex->t_ref;
      }
      alpha[k] = ex->alpha.at(tsum / static_cast<double>(npe));
      tref[k] = ex->t_ref;
    }
    check(cxg_plan_set_thermal_strain(plan_, node_temp.data(), applied.data(), alpha.data(), tref.data()));
  }
}

CudaAssembler::~CudaAssembler() { cxg_plan_destroy(plan_); }

cxpp::fem::LinearSystem CudaAssembler::system_from_csr(const std::vector<double>& vals,
                                                       std::vector<double> rhs) const {
  cxpp::fem::LinearSystem sys = base_;
  const std::size_t nnz = col_idx_.size();
  sys.rows.resize(nnz);
  sys.cols.assign(col_idx_.begin(), col_idx_.end());
  sys.vals = vals;
  for (std::size_t r = 0; r + 1 < row_ptr_.size(); ++r)
    for (int64_t k = row_ptr_[r]; k < row_ptr_[r + 1]; ++k)
      sys.rows[static_cast<std::size_t>(k)] = static_cast<cxpp::Index>(r);
  sys.rhs = std::move(rhs);
  return sys;
}

cxpp::fem::LinearSystem CudaAssembler::assemble_linear_static() {
  std::vector<double> vals(col_idx_.size()), rhs(static_cast<std::size_t>(base_.n_free));
  check(cxg_assemble_linear(plan_, vals.data(), rhs.data(), f_ext_.data(), nullptr));
  int64_t bad = 0;
  check(cxg_plan_check(plan_, &bad));
  return system_from_csr(vals, std::move(rhs));
}

cxpp::fem::LinearSystem CudaAssembler::assemble_material_tangent(const std::vector<cxpp::Vec3>& u,
                                                                 std::vector<cxpp::Real>& f_int) {
  const std::size_t N = model_.mesh.num_nodes();
  if (u.size() != N) throw std::runtime_error("displacement size does not match the mesh");
  std::vector<double> uf(3 * N);
  for (std::size_t i = 0; i < N; ++i)
    for (int d = 0; d < 3; ++d) uf[3 * i + d] = u[i][static_cast<std::size_t>(d)];
  f_int.assign(3 * N, 0.0);
  std::vector<double> vals(col_idx_.size()), rhs(static_cast<std::size_t>(base_.n_free));
  check(cxg_assemble_tangent(plan_, uf.data(), vals.data(), f_int.data(), rhs.data(), f_ext_.data(), nullptr));
  int64_t bad = 0;
  check(cxg_plan_check(plan_, &bad));
  return system_from_csr(vals, std::move(rhs));
}

void CudaAssembler::commit() { check(cxg_state_commit(plan_, nullptr)); }

std::vector<double> CudaAssembler::state(bool committed) const {
  cxg_plan_info info{};
  check(cxg_plan_get_info(plan_, &info));
  std::vector<double> out(13 * static_cast<std::size_t>(info.n_gauss_points));
  check(cxg_state_get(plan_, committed ? CXG_STATE_COMMITTED : CXG_STATE_TRIAL, out.data()));
  return out;
}

cxpp::fem::LinearSystem assemble_linear_static_cuda(const cxpp::Model& model, Precision precision) {
  CudaAssembler a(model, precision);
  return a.assemble_linear_static();
}

std::vector<cxpp::Real> CudaBackend::solve_sparse(const std::vector<cxpp::Index>& rows,
                                                  const std::vector<cxpp::Index>& cols,
                                                  const std::vector<cxpp::Real>& vals, cxpp::Index n,
                                                  const std::vector<cxpp::Real>& rhs,
                                                  cxpp::compute::SolverKind solver) const {
  if (rows.size() != vals.size() || cols.size() != vals.size() || rhs.size() != static_cast<std::size_t>(n))
    throw std::invalid_argument("solve_sparse: inconsistent COO / rhs sizes");
  std::vector<cxpp::Real> x(static_cast<std::size_t>(n), 0.0);
  const bool cg = solver == cxpp::compute::SolverKind::CG;
  const int rc = cxg_solve_sparse(n, static_cast<int64_t>(vals.size()), rows.data(), cols.data(), vals.data(),
                                  rhs.data(), x.data(), cg ? CXG_SOLVER_IC0_CG : CXG_SOLVER_DIRECT, 1e-10,
                                  std::max<int32_t>(1000, 10 * n), nullptr, nullptr);
  if (rc != CXG_OK) throw std::runtime_error(cxg_last_error());
  return x;
}

const cxpp::compute::ComputeBackend& cuda_backend() {
  static const CudaBackend backend;
  return backend;
}

cxpp::StaticFields solve_linear_static_cuda(const cxpp::Model& model,
                                            std::optional<cxpp::numerics::SolverKind> forced, Precision precision,
                                            bool gpu_solve) {
  const cxpp::fem::LinearSystem sys = assemble_linear_static_cuda(model, precision);
  const cxpp::numerics::SolverKind kind =
      forced ? *forced : cxpp::numerics::resolve_solver_kind(model.solver, sys.n_free);
  const std::vector<cxpp::Real> uf =
      gpu_solve ? cuda_backend().solve_sparse(sys.rows, sys.cols, sys.vals, sys.n_free, sys.rhs, kind)
                : cxpp::numerics::solve_reduced(sys, kind);
  cxpp::StaticFields res;
  const std::size_t n_nodes = model.mesh.num_nodes();
  res.displacement.assign(n_nodes, cxpp::Vec3{0, 0, 0});
  for (std::size_t ni = 0; ni < n_nodes; ++ni)
    for (int c = 0; c < cxpp::kDofsPerNode; ++c) {
      const std::size_t g = ni * cxpp::kDofsPerNode + static_cast<std::size_t>(c);
      res.displacement[ni][static_cast<std::size_t>(c)] = sys.transform.displacement(g, uf, sys.prescribed);
    }
  cxpp::fem::recover_fields(model, res);
  return res;
}

}  // namespace cxg_cxpp
