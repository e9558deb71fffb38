/* cxo — CPU restatement of CalculiX++'s element-integration / J2 / assembly path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker the parity tests, smoke()
 * and the bench's cpu_baseline leg compare the CUDA path against; the product path
 * (calculixpp_b200) never links, loads or calls it.
 *
 * Parity is pinned: tests/test_oracle_vs_reference.py checks this restatement
 * bit-for-bit against the reference itself (oracle/_ref/libcxpp_ref.so, compiled from
 * the reference's own sources) on element matrices, J2 updates and assembled systems,
 * and tests/test_oracle_golden.py checks it against committed fixtures generated from
 * the reference (tests/golden/make_golden.py) plus the reference's analytic
 * known-answer tests (tests/test_element.cpp, tests/test_plasticity.cpp).
 *
 * Element type codes are the ordinals of cxpp::ElementType
 * (include/calculixpp/core/element.hpp:13-22): C3D8=2, C3D8R=3, C3D20=4, C3D20R=5,
 * C3D6=6, C3D15=7. Arrays are row-major; DOF order is node-major [u1,v1,w1,u2,...];
 * Voigt order xx,yy,zz,xy,xz,yz with engineering shear. The per-Gauss-point history
 * is 13 doubles: plastic strain[6], equivalent plastic strain, back stress[6].
 */
#ifndef CXO_H
#define CXO_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as the shim's ref_material and the product's cxg_material. */
typedef struct {
  double E;
  double nu;
  int32_t n_plastic; /* 0: linear elastic; else *PLASTIC table length */
  const double* eqplastic;
  const double* yield;
  int32_t hardening; /* 0 isotropic, 1 kinematic, 2 combined */
  double h_kin;
} cxo_material;

int cxo_nodes_per_element(int type);
int cxo_gauss_rule(int type, double* out4);
int cxo_shape(int type, double xi, double et, double ze, double* N, double* dN);
int cxo_physical_gradients(int type, double xi, double et, double ze,
                           const double* coords, double* grad, double* det);
int cxo_element_volume(int type, const double* coords, double* vol);
int cxo_element_stiffness(int type, const double* coords, double E, double nu,
                          double* Ke);
int cxo_material_evaluate(const cxo_material* mat, const double* strain,
                          const double* committed, double* trial, double* stress,
                          double* tangent);
int cxo_element_tangent_force(int type, const double* coords, const double* ue,
                              const cxo_material* mat, const double* state_committed,
                              double* state_trial, double* Ke, double* fe);

/* Reduced system in canonical CSR (rows ascending, columns ascending, duplicates summed
 * in element order). */
typedef struct cxo_system cxo_system;

/* Free-DOF numbering from single-point constraints (constraint_transform.cpp:78-82):
 * dof_eq[3N] (free equation or -1), prescribed[3N]. Returns n_free. */
int32_t cxo_dof_map(int64_t n_nodes, int64_t n_spc, const int32_t* spc_node,
                    const int32_t* spc_comp, const double* spc_val, int32_t* dof_eq,
                    double* prescribed);

/* assemble_linear_static for SPC-only models. conn_ptr has n_elems+1 offsets into conn
 * (0-based node indices); elem_mat selects mats[] (elastic part used). f_ext[3N] may be
 * NULL. */
cxo_system* cxo_assemble_linear(int64_t n_nodes, const double* coords, int64_t n_elems,
                                const int32_t* types, const int64_t* conn_ptr,
                                const int32_t* conn, const int32_t* elem_mat,
                                const cxo_material* mats, const int32_t* dof_eq,
                                const double* prescribed, int32_t n_free,
                                const double* f_ext);

/* assemble_material_tangent: u[3N] full displacement, state_committed[13*G] in,
 * state_trial[13*G] and f_int[3N] out (G = total Gauss points, element order). */
cxo_system* cxo_assemble_tangent(int64_t n_nodes, const double* coords, int64_t n_elems,
                                 const int32_t* types, const int64_t* conn_ptr,
                                 const int32_t* conn, const int32_t* elem_mat,
                                 const cxo_material* mats, const int32_t* dof_eq,
                                 const double* prescribed, int32_t n_free,
                                 const double* f_ext, const double* u,
                                 const double* state_committed, double* state_trial,
                                 double* f_int);

/* element_mass / element_mass_lumped / element_geometric_stiffness
 * (include/calculixpp/fem/element.hpp:93-118): dense 3n x 3n. gp_stress[6 * points]. */
int cxo_element_mass(int type, const double* coords, double rho, double* Me);
int cxo_element_mass_lumped(int type, const double* coords, double rho, double* Ml);
int cxo_element_geometric_stiffness(int type, const double* coords, const double* gp_stress, double* Ke);

/* assemble_mass (kind 1 consistent, 2 lumped) and assemble_geometric_stiffness (kind 3),
 * src/fem/assembly.cpp:259-331; the rhs of the returned system is zero. */
cxo_system* cxo_assemble_scalar(int kind, int64_t n_nodes, const double* coords, int64_t n_elems,
                                const int32_t* types, const int64_t* conn_ptr, const int32_t* conn,
                                const double* density, const double* gp_stress, const int32_t* dof_eq,
                                const double* prescribed, int32_t n_free);

/* recover_gauss_stress / recover_fields (src/fem/stress.cpp:147-271), elastic without
 * thermal strain: gp_stress[6 G]; nodal strain/stress [6N] averaged over incident
 * elements; reaction[3N] = f_int - f_ext (f_ext may be NULL). */
int cxo_recover_gauss_stress(int64_t n_nodes, const double* coords, int64_t n_elems, const int32_t* types,
                             const int64_t* conn_ptr, const int32_t* conn, const double* young,
                             const double* poisson, const double* u, double* gp_stress);
int cxo_recover_fields(int64_t n_nodes, const double* coords, int64_t n_elems, const int32_t* types,
                       const int64_t* conn_ptr, const int32_t* conn, const double* young, const double* poisson,
                       const double* u, const double* f_ext, double* strain, double* stress, double* reaction);
/* Thermal strain (loads.cpp:515-560, stress.cpp:76-271): node_temp[n_nodes] applied
 * temperatures, node_applied[n_nodes] 0/1 (NULL: every node), elem_alpha[n_elems] the
 * expansion coefficient at the element's mean temperature (0: none), elem_tref[n_elems];
 * NULL node_temp: no thermal strain. */
int cxo_thermal_strain_load(int64_t n_nodes, const double* coords, int64_t n_elems, const int32_t* types,
                            const int64_t* conn_ptr, const int32_t* conn, const double* young, const double* poisson,
                            const double* node_temp, const uint8_t* node_applied, const double* elem_alpha,
                            const double* elem_tref, double* f);
int cxo_recover_gauss_stress_th(int64_t n_nodes, const double* coords, int64_t n_elems, const int32_t* types,
                                const int64_t* conn_ptr, const int32_t* conn, const double* young,
                                const double* poisson, const double* node_temp, const uint8_t* node_applied,
                                const double* elem_alpha, const double* elem_tref, const double* u, double* out);
int cxo_recover_fields_th(int64_t n_nodes, const double* coords, int64_t n_elems, const int32_t* types,
                          const int64_t* conn_ptr, const int32_t* conn, const double* young, const double* poisson,
                          const double* node_temp, const uint8_t* node_applied, const double* elem_alpha,
                          const double* elem_tref, const double* u, const double* f_ext, double* strain_out,
                          double* stress_out, double* reaction);

/* element_conduction (n x n) and assemble_conduction without films (src/fem/thermal.cpp:
 * 92-141): t_dof_eq[N] / t_prescribed[N] scalar temperature DOF map, flux[N] may be NULL. */
int cxo_element_conduction(int type, const double* coords, double k, double* Kt);
cxo_system* cxo_assemble_conduction(int64_t n_nodes, const double* coords, int64_t n_elems, const int32_t* types,
                                    const int64_t* conn_ptr, const int32_t* conn, const double* conductivity,
                                    const int32_t* t_dof_eq, const double* t_prescribed, int32_t n_free,
                                    const double* flux);
/* assemble_conduction with *FILM faces (thermal.cpp:113-126): film f on face film_face[f]
 * (1-based) of element film_elem[f], coefficient film_h[f], sink temperature film_sink[f]. */
cxo_system* cxo_assemble_conduction_films(int64_t n_nodes, const double* coords, int64_t n_elems,
                                          const int32_t* types, const int64_t* conn_ptr, const int32_t* conn,
                                          const double* conductivity, const int32_t* t_dof_eq,
                                          const double* t_prescribed, int32_t n_free, const double* flux,
                                          int64_t n_films, const int64_t* film_elem, const int32_t* film_face,
                                          const double* film_h, const double* film_sink);

int cxo_system_info(const cxo_system* s, int32_t* n_free, int64_t* nnz);
int cxo_system_copy(const cxo_system* s, int64_t* row_ptr, int32_t* col_idx,
                    double* vals, double* rhs);
void cxo_system_free(cxo_system* s);

/* Per-element compliance derivative by central differences of K_e in the nodal
 * coordinates: dcdX[3n] = -u_e^T (K_e(x+h) - K_e(x-h))/(2h) u_e, the element-level
 * form of the reference's semi-analytic design sensitivity
 * (src/numerics/sensitivity.cpp:77-108). */
int cxo_element_compliance_grad_fd(int type, const double* coords, const double* ue,
                                   double E, double nu, double h, double* dcdX);

const char* cxo_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
