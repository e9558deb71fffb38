// C-ABI shim over the reference's own C++ API (test infrastructure only).
//
// Compiled together with the reference's sources (oracle/Makefile) into
// oracle/_ref/libcxpp_ref.so, so that the Python tests and the CPU baseline can call
// the reference implementation itself:
//   element level  : gauss_rule / shape / physical_gradients / element_stiffness /
//                    element_tangent_force / J2PlasticMaterial::evaluate
//                    (src/fem/element.cpp:106-743, src/fem/plasticity.cpp:42-236)
//   assembly level : assemble_linear_static / make_material_points /
//                    assemble_material_tangent (src/fem/assembly.cpp:225-423)
//   drivers        : solve_sensitivity (src/numerics/sensitivity.cpp:112)
//   harness        : a threaded loop over element_stiffness with an exact CSR
//                    scatter ("harness-parallelized reference kernels"), used as the
//                    all-cores CPU baseline.
// Models are built through the reference's C++ API (Mesh::add_node/add_element,
// materials, sections, SPCs, CLOADs), with node id = index + 1 and element id =
// index + 1. Every entry point returns 0 on success and -1 after storing the
// exception text, readable through ref_last_error().
#include <algorithm>
#include <array>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <span>
#include <string>
#include <thread>
#include <vector>

#include "calculixpp/core/model.hpp"
#include "calculixpp/fem/assembly.hpp"
#include "calculixpp/fem/loads.hpp"
#include "calculixpp/fem/stress.hpp"
#include "calculixpp/fem/thermal.hpp"
#include "calculixpp/fem/element.hpp"
#include "calculixpp/fem/material_model.hpp"
#include "calculixpp/numerics/sensitivity.hpp"

using namespace cxpp;
using namespace cxpp::fem;

namespace {

thread_local std::string g_err;

int fail(const std::exception& e) {
  g_err = e.what();
  return -1;
}

}  // namespace

extern "C" {

// Material description used by every entry point below. n_plastic == 0 selects
// linear elasticity (ElasticIsoMaterial); otherwise a J2PlasticMaterial is built from
// the *PLASTIC table (eqplastic[i], yield[i]) with the given hardening kind
// (0 isotropic, 1 kinematic, 2 combined) and kinematic modulus.
typedef struct {
  double E;
  double nu;
  int32_t n_plastic;
  const double* eqplastic;
  const double* yield;
  int32_t hardening;
  double h_kin;
} ref_material;

const char* ref_last_error(void) { return g_err.c_str(); }

}  // extern "C"

namespace {

constexpr int kStateDoubles = 13;  // per Gauss point: eps_p[6], eqplastic, back_stress[6]

Material make_material(const ref_material& m, const std::string& name) {
  Material mat;
  mat.name = name;
  mat.elastic = ElasticIso{m.E, m.nu};
  if (m.n_plastic > 0) {
    Plastic p;
    p.hardening = m.hardening == 1   ? Plastic::Hardening::Kinematic
                  : m.hardening == 2 ? Plastic::Hardening::Combined
                                     : Plastic::Hardening::Isotropic;
    p.eqplastic.assign(m.eqplastic, m.eqplastic + m.n_plastic);
    p.yield.assign(m.yield, m.yield + m.n_plastic);
    p.kinematic_modulus = m.h_kin;
    mat.plastic = p;
  }
  return mat;
}

std::unique_ptr<MaterialModel> make_model(const ref_material& m) {
  if (m.n_plastic > 0) {
    const Material mat = make_material(m, "M");
    return std::make_unique<J2PlasticMaterial>(*mat.elastic, *mat.plastic);
  }
  return std::make_unique<ElasticIsoMaterial>(ElasticIso{m.E, m.nu});
}

void state_to_array(const MaterialState& s, bool committed, double* out) {
  const Voigt6& ep = committed ? s.committed_plastic_strain : s.plastic_strain;
  const Voigt6& al = committed ? s.committed_back_stress : s.back_stress;
  for (int i = 0; i < 6; ++i) out[i] = ep[static_cast<std::size_t>(i)];
  out[6] = committed ? s.committed_eqplastic : s.eqplastic;
  for (int i = 0; i < 6; ++i) out[7 + i] = al[static_cast<std::size_t>(i)];
}

void array_to_state(const double* in, bool committed, MaterialState& s) {
  Voigt6& ep = committed ? s.committed_plastic_strain : s.plastic_strain;
  Voigt6& al = committed ? s.committed_back_stress : s.back_stress;
  for (int i = 0; i < 6; ++i) ep[static_cast<std::size_t>(i)] = in[i];
  (committed ? s.committed_eqplastic : s.eqplastic) = in[6];
  for (int i = 0; i < 6; ++i) al[static_cast<std::size_t>(i)] = in[7 + i];
}

struct RefModel {
  Model model;
};

struct RefMp {
  MaterialPoints mp;
};

}  // namespace

extern "C" {

// ---- element level -----------------------------------------------------------------

// Gauss rule of `type`: writes {xi, et, ze, w} per point into out[4*i..]; returns the
// number of points.
int ref_gauss_rule(int type, double* out) {
  const auto rule = gauss_rule(static_cast<ElementType>(type));
  for (std::size_t i = 0; i < rule.size(); ++i) {
    out[4 * i + 0] = rule[i].xi;
    out[4 * i + 1] = rule[i].et;
    out[4 * i + 2] = rule[i].ze;
    out[4 * i + 3] = rule[i].w;
  }
  return static_cast<int>(rule.size());
}

// Shape functions N[k] and natural derivatives dN[3k+d]; returns the node count.
int ref_shape(int type, double xi, double et, double ze, double* N, double* dN) {
  const Shape s = shape(static_cast<ElementType>(type), xi, et, ze);
  for (int k = 0; k < s.n; ++k) {
    N[k] = s.N[static_cast<std::size_t>(k)];
    for (int d = 0; d < 3; ++d)
      dN[3 * k + d] = s.dNdxi[static_cast<std::size_t>(k)][static_cast<std::size_t>(d)];
  }
  return s.n;
}

// Physical gradients at a natural point; returns 0 and writes det(J), or -1 (det<=0).
int ref_physical_gradients(int type, double xi, double et, double ze,
                           const double* coords, double* grad, double* det_out) {
  try {
    const ElementType t = static_cast<ElementType>(type);
    const int n = nodes_per_element(t);
    std::vector<Vec3> x(static_cast<std::size_t>(n));
    for (int k = 0; k < n; ++k) x[static_cast<std::size_t>(k)] = {coords[3 * k], coords[3 * k + 1], coords[3 * k + 2]};
    const Shape s = shape(t, xi, et, ze);
    std::array<std::array<Real, 3>, kMaxNodes> g{};
    *det_out = physical_gradients(s, x, g);
    for (int k = 0; k < n; ++k)
      for (int d = 0; d < 3; ++d) grad[3 * k + d] = g[static_cast<std::size_t>(k)][static_cast<std::size_t>(d)];
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

int ref_element_volume(int type, const double* coords, double* vol) {
  try {
    const ElementType t = static_cast<ElementType>(type);
    const int n = nodes_per_element(t);
    std::vector<Vec3> x(static_cast<std::size_t>(n));
    for (int k = 0; k < n; ++k) x[static_cast<std::size_t>(k)] = {coords[3 * k], coords[3 * k + 1], coords[3 * k + 2]};
    *vol = element_volume(t, x);
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// Dense (3n)^2 row-major linear element stiffness.
int ref_element_stiffness(int type, const double* coords, double E, double nu,
                          double* Ke) {
  try {
    const ElementType t = static_cast<ElementType>(type);
    const int n = nodes_per_element(t);
    std::vector<Vec3> x(static_cast<std::size_t>(n));
    for (int k = 0; k < n; ++k) x[static_cast<std::size_t>(k)] = {coords[3 * k], coords[3 * k + 1], coords[3 * k + 2]};
    const std::vector<Real> K = element_stiffness(t, x, ElasticIso{E, nu});
    std::memcpy(Ke, K.data(), K.size() * sizeof(double));
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// One constitutive evaluation. committed[13] is the start-of-increment history;
// trial[13] receives the advanced history. stress[6], tangent[36] row-major.
int ref_material_evaluate(const ref_material* mat, const double* strain,
                          const double* committed, double* trial, double* stress,
                          double* tangent) {
  try {
    const auto model = make_model(*mat);
    MaterialState st;
    array_to_state(committed, true, st);
    array_to_state(committed, false, st);
    Voigt6 eps{};
    for (int i = 0; i < 6; ++i) eps[static_cast<std::size_t>(i)] = strain[i];
    const MaterialResponse r = model->evaluate(eps, st);
    for (int i = 0; i < 6; ++i) {
      stress[i] = r.stress[static_cast<std::size_t>(i)];
      for (int j = 0; j < 6; ++j)
        tangent[6 * i + j] = r.tangent[static_cast<std::size_t>(i)][static_cast<std::size_t>(j)];
    }
    state_to_array(st, false, trial);
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// Material-point element kernel. state_committed[13*ngp] in, state_trial[13*ngp] out.
int ref_element_tangent_force(int type, const double* coords, const double* ue,
                              const ref_material* mat, const double* state_committed,
                              double* state_trial, double* Ke, double* fe) {
  try {
    const ElementType t = static_cast<ElementType>(type);
    const int n = nodes_per_element(t);
    std::vector<Vec3> x(static_cast<std::size_t>(n)), u(static_cast<std::size_t>(n));
    for (int k = 0; k < n; ++k) {
      x[static_cast<std::size_t>(k)] = {coords[3 * k], coords[3 * k + 1], coords[3 * k + 2]};
      u[static_cast<std::size_t>(k)] = {ue[3 * k], ue[3 * k + 1], ue[3 * k + 2]};
    }
    const std::size_t ngp = gauss_rule(t).size();
    std::vector<MaterialState> st(ngp);
    for (std::size_t q = 0; q < ngp; ++q) {
      array_to_state(state_committed + kStateDoubles * q, true, st[q]);
      array_to_state(state_committed + kStateDoubles * q, false, st[q]);
    }
    const auto model = make_model(*mat);
    const ElementResponse r = element_tangent_force(t, x, u, *model, st);
    std::memcpy(Ke, r.Ke.data(), r.Ke.size() * sizeof(double));
    std::memcpy(fe, r.fe.data(), r.fe.size() * sizeof(double));
    for (std::size_t q = 0; q < ngp; ++q) state_to_array(st[q], false, state_trial + kStateDoubles * q);
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// ---- model / assembly level -----------------------------------------------------------

// Build a reference Model. conn_ptr[e]..conn_ptr[e+1] index into conn (0-based node
// indices). elem_mat[e] selects mats[]. SPC / CLOAD nodes are 0-based, comps 0..2.
void* ref_model_create(int64_t n_nodes, const double* coords, int64_t n_elems,
                       const int32_t* types, const int64_t* conn_ptr,
                       const int32_t* conn, const int32_t* elem_mat, int32_t n_mats,
                       const ref_material* mats, int64_t n_spc,
                       const int32_t* spc_node, const int32_t* spc_comp,
                       const double* spc_val, int64_t n_cload, const int32_t* cl_node,
                       const int32_t* cl_comp, const double* cl_val) {
  try {
    auto rm = std::make_unique<RefModel>();
    Model& m = rm->model;
    for (int64_t i = 0; i < n_nodes; ++i)
      m.mesh.add_node(static_cast<Index>(i + 1),
                      Vec3{coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]});
    std::vector<std::vector<Index>> sets(static_cast<std::size_t>(n_mats));
    for (int64_t e = 0; e < n_elems; ++e) {
      std::vector<Index> ids;
      for (int64_t p = conn_ptr[e]; p < conn_ptr[e + 1]; ++p) ids.push_back(conn[p] + 1);
      m.mesh.add_element(static_cast<Index>(e + 1), static_cast<ElementType>(types[e]), ids);
      sets[static_cast<std::size_t>(elem_mat[e])].push_back(static_cast<Index>(e + 1));
    }
    for (int32_t k = 0; k < n_mats; ++k) {
      const std::string name = "M" + std::to_string(k);
      if (sets[static_cast<std::size_t>(k)].empty()) continue;
      m.mesh.add_elset("E" + name, sets[static_cast<std::size_t>(k)]);
      m.materials[name] = make_material(mats[k], name);
      m.sections.push_back(SolidSection{"E" + name, name});
    }
    for (int64_t i = 0; i < n_spc; ++i) {
      Spc s;
      s.node_id = spc_node[i] + 1;
      s.comp = spc_comp[i] + 1;
      s.value = spc_val[i];
      m.spcs.push_back(s);
    }
    for (int64_t i = 0; i < n_cload; ++i) {
      Cload c;
      c.node_id = cl_node[i] + 1;
      c.comp = cl_comp[i] + 1;
      c.value = cl_val[i];
      m.cloads.push_back(c);
    }
    return rm.release();
  } catch (const std::exception& e) {
    fail(e);
    return nullptr;
  }
}

void ref_model_free(void* model) { delete static_cast<RefModel*>(model); }

// Adds a linear multi-point constraint (*EQUATION) sum coeff_i u(node_i, comp_i) = 0 to the
// model; the first term is the dependent DOF. Nodes 0-based, comps 0..2.
int ref_model_add_equation(void* model, int32_t n_terms, const int32_t* nodes, const int32_t* comps,
                           const double* coeffs) {
  try {
    Equation eq;
    eq.origin = "*EQUATION";
    for (int32_t i = 0; i < n_terms; ++i) eq.terms.push_back(EquationTerm{nodes[i] + 1, comps[i] + 1, coeffs[i]});
    static_cast<RefModel*>(model)->model.equations.push_back(eq);
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// *EXPANSION of material k (Material::expansion): an alpha(T) table of n_points[k] rows
// (alpha_vals / alpha_temps, rows of all materials concatenated) and the reference
// temperature tref[k]; n_points[k] == 0 leaves material k without expansion.
int ref_model_set_expansion(void* model, int32_t n_mats, const int32_t* n_points, const double* alpha_vals,
                            const double* alpha_temps, const double* tref) {
  try {
    Model& m = static_cast<RefModel*>(model)->model;
    int64_t off = 0;
    for (int32_t k = 0; k < n_mats; ++k) {
      const auto it = m.materials.find("M" + std::to_string(k));
      const int32_t np = n_points[k];
      if (it != m.materials.end() && np > 0) {
        Expansion ex;
        for (int32_t r = 0; r < np; ++r) {
          ex.alpha.value.push_back(alpha_vals[off + r]);
          ex.alpha.temp.push_back(alpha_temps[off + r]);
        }
        ex.t_ref = tref[k];
        it->second.expansion = ex;
      }
      off += np;
    }
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// A *FILM face (Model::films): element 0-based, face 1-based.
int ref_model_add_film(void* model, int64_t elem, int32_t face, double h, double sink) {
  try {
    Film f;
    f.elem_id = static_cast<Index>(elem + 1);
    f.face = face;
    f.h = h;
    f.sink_temp = sink;
    static_cast<RefModel*>(model)->model.films.push_back(f);
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// Applied temperatures (Model::applied_temperature): nodes 0-based.
int ref_model_set_temperature(void* model, int64_t n, const int32_t* nodes, const double* temps) {
  try {
    Model& m = static_cast<RefModel*>(model)->model;
    m.applied_temperature.clear();
    for (int64_t i = 0; i < n; ++i) m.applied_temperature[static_cast<Index>(nodes[i] + 1)] = temps[i];
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// thermal_strain_load_vector (loads.cpp:515-560): out[3N].
int ref_thermal_strain_load_vector(void* model, double* out) {
  try {
    const Model& m = static_cast<RefModel*>(model)->model;
    const std::vector<Real> f = thermal_strain_load_vector(m);
    std::copy(f.begin(), f.end(), out);
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// The Model behind a handle, for other harness translation units (ref_cuda_shim.cpp).
const cxpp::Model* ref_model_get(void* model) { return &static_cast<RefModel*>(model)->model; }

// element_mass (lumped = 0) / element_mass_lumped (lumped = 1), element.hpp:93-102.
int ref_element_mass(int type, const double* coords, double rho, int lumped, double* Me) {
  try {
    const ElementType t = static_cast<ElementType>(type);
    const int n = nodes_per_element(t);
    std::vector<Vec3> x(static_cast<std::size_t>(n));
    for (int k = 0; k < n; ++k) x[static_cast<std::size_t>(k)] = {coords[3 * k], coords[3 * k + 1], coords[3 * k + 2]};
    const std::vector<Real> M = lumped ? element_mass_lumped(t, x, rho) : element_mass(t, x, rho);
    std::memcpy(Me, M.data(), M.size() * sizeof(double));
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// element_geometric_stiffness, element.hpp:117-119; gp_stress[6 * points] (Voigt6).
int ref_element_geometric_stiffness(int type, const double* coords, const double* gp_stress, double* Ke) {
  try {
    const ElementType t = static_cast<ElementType>(type);
    const int n = nodes_per_element(t);
    std::vector<Vec3> x(static_cast<std::size_t>(n));
    for (int k = 0; k < n; ++k) x[static_cast<std::size_t>(k)] = {coords[3 * k], coords[3 * k + 1], coords[3 * k + 2]};
    const std::size_t ng = gauss_rule(t).size();
    std::vector<Voigt6> sg(ng);
    for (std::size_t q = 0; q < ng; ++q)
      for (int c = 0; c < 6; ++c) sg[q][static_cast<std::size_t>(c)] = gp_stress[6 * q + c];
    const std::vector<Real> K = element_geometric_stiffness(t, x, sg);
    std::memcpy(Ke, K.data(), K.size() * sizeof(double));
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// Per-material density (Material::density) of a model built by ref_model_create.
int ref_model_set_density(void* model, int32_t n_mats, const double* rho) {
  try {
    Model& m = static_cast<RefModel*>(model)->model;
    for (int32_t k = 0; k < n_mats; ++k) {
      auto it = m.materials.find("M" + std::to_string(k));
      if (it != m.materials.end()) it->second.density = rho[k];
    }
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// assemble_mass (assembly.cpp:259-298).
void* ref_assemble_mass(void* model, int lumped) {
  try {
    return new LinearSystem(assemble_mass(static_cast<RefModel*>(model)->model, lumped != 0));
  } catch (const std::exception& e) {
    fail(e);
    return nullptr;
  }
}

// assemble_geometric_stiffness (assembly.cpp:300-331); gp_stress[6 * G], element order.
void* ref_assemble_geometric(void* model, const double* gp_stress) {
  try {
    const Model& m = static_cast<RefModel*>(model)->model;
    std::vector<std::vector<Voigt6>> sg(m.mesh.num_elements());
    std::size_t off = 0;
    for (std::size_t e = 0; e < m.mesh.num_elements(); ++e) {
      const std::size_t ng = gauss_rule(m.mesh.elements()[e].type).size();
      sg[e].resize(ng);
      for (std::size_t q = 0; q < ng; ++q, ++off)
        for (int c = 0; c < 6; ++c) sg[e][q][static_cast<std::size_t>(c)] = gp_stress[6 * off + c];
    }
    return new LinearSystem(assemble_geometric_stiffness(m, sg));
  } catch (const std::exception& e) {
    fail(e);
    return nullptr;
  }
}

// recover_gauss_stress (stress.cpp:147-187): out[6 G] in element order.
int ref_recover_gauss_stress(void* model, const double* u, double* out) {
  try {
    const Model& m = static_cast<RefModel*>(model)->model;
    std::vector<Vec3> uu(m.mesh.num_nodes());
    for (std::size_t i = 0; i < uu.size(); ++i) uu[i] = {u[3 * i], u[3 * i + 1], u[3 * i + 2]};
    const auto sg = recover_gauss_stress(m, uu);
    std::size_t off = 0;
    for (const auto& e : sg)
      for (const auto& v : e) {
        for (int c = 0; c < 6; ++c) out[6 * off + c] = v[static_cast<std::size_t>(c)];
        ++off;
      }
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// recover_fields (stress.cpp:189-271): nodal strain/stress [6N], reaction [3N].
int ref_recover_fields(void* model, const double* u, double* strain, double* stress, double* reaction) {
  try {
    const Model& m = static_cast<RefModel*>(model)->model;
    StaticFields f;
    f.displacement.resize(m.mesh.num_nodes());
    for (std::size_t i = 0; i < f.displacement.size(); ++i) f.displacement[i] = {u[3 * i], u[3 * i + 1], u[3 * i + 2]};
    recover_fields(m, f);
    for (std::size_t i = 0; i < f.displacement.size(); ++i) {
      for (int c = 0; c < 6; ++c) {
        strain[6 * i + c] = f.strain[i][static_cast<std::size_t>(c)];
        stress[6 * i + c] = f.stress[i][static_cast<std::size_t>(c)];
      }
      for (int c = 0; c < 3; ++c) reaction[3 * i + c] = f.reaction[i][static_cast<std::size_t>(c)];
    }
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// element_conduction (element.hpp:73-74): Kt[n * n].
int ref_element_conduction(int type, const double* coords, double k, double* Kt) {
  try {
    const ElementType t = static_cast<ElementType>(type);
    const int n = nodes_per_element(t);
    std::vector<Vec3> x(static_cast<std::size_t>(n));
    for (int i = 0; i < n; ++i) x[static_cast<std::size_t>(i)] = {coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]};
    const std::vector<Real> K = element_conduction(t, x, k);
    std::memcpy(Kt, K.data(), K.size() * sizeof(double));
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// assemble_conduction (thermal.cpp:92-141) on a model built by ref_model_create, with
// per-material conductivity and prescribed temperatures (0-based nodes).
void* ref_assemble_conduction(void* model, int32_t n_mats, const double* k, int64_t n_tbc, const int32_t* tbc_node,
                              const double* tbc_val) {
  try {
    Model& m = static_cast<RefModel*>(model)->model;
    for (int32_t i = 0; i < n_mats; ++i) {
      auto it = m.materials.find("M" + std::to_string(i));
      if (it == m.materials.end()) continue;
      Thermal th;
      th.conductivity = PropertyTable(k[i]);
      it->second.thermal = th;
    }
    m.temp_bcs.clear();
    for (int64_t i = 0; i < n_tbc; ++i) {
      TempBc bc;
      bc.node_id = tbc_node[i] + 1;
      bc.value = tbc_val[i];
      m.temp_bcs.push_back(bc);
    }
    return new LinearSystem(assemble_conduction(m));
  } catch (const std::exception& e) {
    fail(e);
    return nullptr;
  }
}

void* ref_assemble_linear_static(void* model) {
  try {
    auto* sys = new LinearSystem(assemble_linear_static(static_cast<RefModel*>(model)->model));
    return sys;
  } catch (const std::exception& e) {
    fail(e);
    return nullptr;
  }
}

int ref_sys_info(void* sys, int64_t* n_free, int64_t* nnz) {
  const auto* s = static_cast<LinearSystem*>(sys);
  *n_free = s->n_free;
  *nnz = static_cast<int64_t>(s->vals.size());
  return 0;
}

// COO triplets in the reference's (hash-map) order, the reduced rhs and dof_eq[3N].
int ref_sys_copy(void* sys, int32_t* rows, int32_t* cols, double* vals, double* rhs,
                 int32_t* dof_eq) {
  const auto* s = static_cast<LinearSystem*>(sys);
  std::memcpy(rows, s->rows.data(), s->rows.size() * sizeof(int32_t));
  std::memcpy(cols, s->cols.data(), s->cols.size() * sizeof(int32_t));
  std::memcpy(vals, s->vals.data(), s->vals.size() * sizeof(double));
  std::memcpy(rhs, s->rhs.data(), s->rhs.size() * sizeof(double));
  std::memcpy(dof_eq, s->dof_eq.data(), s->dof_eq.size() * sizeof(int32_t));
  return 0;
}

void ref_sys_free(void* sys) { delete static_cast<LinearSystem*>(sys); }

void* ref_mp_create(void* model) {
  try {
    auto* mp = new RefMp{make_material_points(static_cast<RefModel*>(model)->model)};
    return mp;
  } catch (const std::exception& e) {
    fail(e);
    return nullptr;
  }
}

void ref_mp_free(void* mp) { delete static_cast<RefMp*>(mp); }

int64_t ref_mp_num_points(void* mp) {
  int64_t n = 0;
  for (const auto& es : static_cast<RefMp*>(mp)->mp.state) n += static_cast<int64_t>(es.size());
  return n;
}

// State of every Gauss point in element order, 13 doubles each.
int ref_mp_get_state(void* mp, int committed, double* out) {
  int64_t k = 0;
  for (const auto& es : static_cast<RefMp*>(mp)->mp.state)
    for (const MaterialState& s : es) state_to_array(s, committed != 0, out + kStateDoubles * (k++));
  return 0;
}

int ref_mp_set_state(void* mp, int committed, const double* in) {
  int64_t k = 0;
  for (auto& es : static_cast<RefMp*>(mp)->mp.state)
    for (MaterialState& s : es) array_to_state(in + kStateDoubles * (k++), committed != 0, s);
  return 0;
}

void ref_mp_commit(void* mp) { static_cast<RefMp*>(mp)->mp.commit(); }

// Material tangent + internal force at the full nodal displacement u[3N].
void* ref_assemble_material_tangent(void* model, void* mp, const double* u, double* f_int) {
  try {
    const Model& m = static_cast<RefModel*>(model)->model;
    std::vector<Vec3> uu(m.mesh.num_nodes());
    for (std::size_t i = 0; i < uu.size(); ++i) uu[i] = {u[3 * i], u[3 * i + 1], u[3 * i + 2]};
    std::vector<Real> f;
    auto* sys = new LinearSystem(assemble_material_tangent(m, uu, static_cast<RefMp*>(mp)->mp, f));
    std::memcpy(f_int, f.data(), f.size() * sizeof(double));
    return sys;
  } catch (const std::exception& e) {
    fail(e);
    return nullptr;
  }
}

// Compliance sensitivity over coordinate design variables (node 0-based, comp 0..2),
// through the reference's solve_sensitivity (semi-analytic central differences).
int ref_sensitivity_compliance(void* model, int64_t n_vars, const int32_t* var_node,
                               const int32_t* var_comp, double h, double* dgdx,
                               double* objective) {
  try {
    Model m = static_cast<RefModel*>(model)->model;
    m.procedure = Procedure::Sensitivity;
    m.design_variables.clear();
    for (int64_t i = 0; i < n_vars; ++i)
      m.design_variables.push_back(DesignVariable{var_node[i] + 1, var_comp[i] + 1});
    DesignResponse r;
    r.name = "C";
    r.kind = DesignResponse::Kind::Compliance;
    m.design_responses = {r};
    const numerics::SensitivityReport rep = numerics::solve_sensitivity(m, h);
    const auto& res = rep.responses.front();
    for (int64_t i = 0; i < n_vars; ++i) dgdx[i] = res.dgdx[static_cast<std::size_t>(i)];
    *objective = res.objective;
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// ---- harness-parallelized reference kernels (all-cores CPU baseline) -----------------

// Runs the reference's element_stiffness over elements [0, n_elems) on `nthreads`
// threads and scatters each K_e into a prebuilt CSR (row_ptr int64, col_idx int32,
// sorted columns) of the reduced free system with atomic adds, skipping exact zeros
// like the reference scatter; prescribed columns with a nonzero value go into rhs as
// -K_fc u_c. Uniform element type; conn is n_elems x nodes_per_element.
int ref_assemble_csr_threads(int type, const double* coords, int64_t n_elems,
                             const int32_t* conn, const double* young,
                             const double* poisson, const int32_t* dof_eq,
                             const double* prescribed, const int64_t* row_ptr,
                             const int32_t* col_idx, double* vals, double* rhs,
                             int nthreads) {
  try {
    const ElementType t = static_cast<ElementType>(type);
    const int n = nodes_per_element(t);
    const int ndof = 3 * n;
    std::atomic<int> failed{0};
    auto work = [&](int64_t e0, int64_t e1) {
      std::vector<Vec3> x(static_cast<std::size_t>(n));
      std::vector<int32_t> eq(static_cast<std::size_t>(ndof));
      std::vector<int64_t> gd(static_cast<std::size_t>(ndof));
      try {
        for (int64_t e = e0; e < e1; ++e) {
          const int32_t* c = conn + e * n;
          for (int k = 0; k < n; ++k) {
            x[static_cast<std::size_t>(k)] = {coords[3 * c[k]], coords[3 * c[k] + 1], coords[3 * c[k] + 2]};
            for (int d = 0; d < 3; ++d) {
              gd[static_cast<std::size_t>(3 * k + d)] = 3 * static_cast<int64_t>(c[k]) + d;
              eq[static_cast<std::size_t>(3 * k + d)] = dof_eq[3 * static_cast<int64_t>(c[k]) + d];
            }
          }
          const std::vector<Real> K = element_stiffness(t, x, ElasticIso{young[e], poisson[e]});
          for (int a = 0; a < ndof; ++a) {
            const int32_t r = eq[static_cast<std::size_t>(a)];
            if (r < 0) continue;
            const int32_t* cb = col_idx + row_ptr[r];
            const int32_t* ce = col_idx + row_ptr[r + 1];
            for (int b = 0; b < ndof; ++b) {
              const double kab = K[static_cast<std::size_t>(a * ndof + b)];
              if (kab == 0.0) continue;
              const int32_t cc = eq[static_cast<std::size_t>(b)];
              if (cc >= 0) {
                const int32_t* p = std::lower_bound(cb, ce, cc);
                std::atomic_ref<double>(vals[p - col_idx]).fetch_add(kab, std::memory_order_relaxed);
              } else {
                const double u = prescribed[gd[static_cast<std::size_t>(b)]];
                if (u != 0.0)
                  std::atomic_ref<double>(rhs[r]).fetch_sub(kab * u, std::memory_order_relaxed);
              }
            }
          }
        }
      } catch (const std::exception& ex) {
        g_err = ex.what();
        failed = 1;
      }
    };
    if (nthreads < 1) nthreads = 1;
    std::vector<std::thread> pool;
    const int64_t chunk = (n_elems + nthreads - 1) / nthreads;
    for (int i = 0; i < nthreads; ++i) {
      const int64_t e0 = std::min<int64_t>(n_elems, i * chunk);
      const int64_t e1 = std::min<int64_t>(n_elems, e0 + chunk);
      pool.emplace_back(work, e0, e1);
    }
    for (auto& th : pool) th.join();
    return failed ? -1 : 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

}  // extern "C"
