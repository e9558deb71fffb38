/* cxg — B200-native element integration and CSR assembly for CalculiX++.
 *
 * C ABI of libcxg.so (calculixpp_b200/_lib/libcxg.so). Plain pointers and sizes only.
 * Every pointer argument may point to host or device memory; the library asks the
 * CUDA driver which one it is and stages host buffers through device memory. Device
 * pointers must belong to the current device. All entry points return a cxg_status;
 * cxg_last_error() returns the thread's last error message.
 *
 * Conventions (identical to the reference, include/calculixpp/core/types.hpp:9-13 and
 * include/calculixpp/fem/element.hpp:12-61):
 *   - element type codes are the ordinals of cxpp::ElementType
 *     (include/calculixpp/core/element.hpp:13-22): C3D8=2, C3D8R=3, C3D20=4,
 *     C3D20R=5, C3D6=6, C3D15=7, and the tetrahedra C3D4=0, C3D10=1;
 *   - node indices are 0-based int32; DOF g = 3*node + component;
 *   - element DOF order node-major [u1,v1,w1,u2,...]; Voigt xx,yy,zz,xy,xz,yz with
 *     engineering shear;
 *   - per-Gauss-point material history: 13 doubles {plastic strain[6], equivalent
 *     plastic strain, back stress[6]} (include/calculixpp/fem/material_model.hpp:38-64),
 *     Gauss points in element order then the element's Gauss-rule order.
 *
 * Reduced system: the free/free stiffness K_ff in CSR with int64 row_ptr and int32
 * col_idx, rows and columns in free-equation order, columns ascending. It replaces
 * the reference's COO LinearSystem (include/calculixpp/fem/assembly.hpp:18-38); the
 * same triplets sorted by (row, col) give exactly this CSR.
 */
#ifndef CXG_H
#define CXG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CXG_ABI_VERSION 1

#if defined(__GNUC__)
#define CXG_API __attribute__((visibility("default")))
#else
#define CXG_API
#endif

typedef enum {
  CXG_OK = 0,
  CXG_ERR_INVALID_ARGUMENT = 1,
  CXG_ERR_CUDA = 2,
  CXG_ERR_OUT_OF_MEMORY = 3,
  /* det(J) <= 0 at a Gauss point: the reference throws
   * "non-positive element Jacobian (bad connectivity?)" (src/fem/element.cpp:86-88). */
  CXG_ERR_NEGATIVE_JACOBIAN = 4,
  CXG_ERR_UNSUPPORTED = 5,
  /* an element references a node index outside [0, n_nodes)
   * (src/fem/assembly.cpp:53-54 "element references unknown node"). */
  CXG_ERR_UNKNOWN_NODE = 6,
  CXG_ERR_NO_GPU = 7,
  /* cxg_solve_cg stopped at max_iter above the tolerance (the reference's CG path
   * throws "CG did not converge", src/compute/cpu_backend.cpp:57-62). */
  CXG_ERR_NOT_CONVERGED = 8
} cxg_status;

typedef enum { CXG_FP64 = 0, CXG_MIXED = 1 } cxg_precision;

typedef enum { CXG_STATE_COMMITTED = 0, CXG_STATE_TRIAL = 1 } cxg_state_slot;

/* Material of one element family. n_plastic == 0: linear isotropic elasticity
 * (ElasticIsoMaterial, include/calculixpp/fem/material_model.hpp:84-93). Otherwise J2
 * plasticity with a piecewise-linear *PLASTIC table (eqplastic[i], yield[i]) and
 * hardening 0 = isotropic, 1 = kinematic, 2 = combined, kinematic modulus h_kin
 * (J2PlasticMaterial, material_model.hpp:108-126). Table pointers are host memory. */
typedef struct {
  double E;
  double nu;
  int32_t n_plastic;
  const double* eqplastic;
  const double* yield;
  int32_t hardening;
  double h_kin;
} cxg_material;

/* One mesh of a single element type. young/poisson (per element) override the
 * material's E and nu when non-NULL; elem_mat (per element) selects materials[],
 * NULL means every element uses materials[0]. */
typedef struct {
  int64_t n_nodes;
  int64_t n_elems;
  int32_t elem_type;
  const double* coords;   /* [3*n_nodes] */
  const int32_t* conn;    /* [n_elems * nodes_per_element] */
  const double* young;    /* [n_elems] or NULL */
  const double* poisson;  /* [n_elems] or NULL */
  const int32_t* elem_mat;  /* [n_elems] or NULL */
  int32_t n_materials;
  const cxg_material* materials; /* host array [n_materials] */
} cxg_mesh_desc;

/* Free-DOF map of an SPC-constrained model (ConstraintTransform::dof_eq and
 * LinearSystem::prescribed, include/calculixpp/fem/constraint_transform.hpp:38-47):
 * dof_eq[g] = free equation or -1; free equations numbered in increasing g.
 * prescribed[g] = SPC value (0 for free DOFs). */
typedef struct {
  const int32_t* dof_eq;     /* [3*n_nodes] */
  const double* prescribed;  /* [3*n_nodes] */
  int32_t n_free;
} cxg_dofmap_desc;

/* Multi-point constraints (*EQUATION and the constraints expanded into equations) as the
 * reference's constraint transform holds them (ConstraintTransform::expansion,
 * include/calculixpp/fem/constraint_transform.hpp:28-47, built by
 * src/fem/constraint_transform.cpp:25-131): every slave DOF g = 3*node + comp (ascending)
 * expands onto free equations with coefficients, plus a constant (the full-magnitude
 * prescribed values of SPC masters). In the cxg_dofmap_desc of such a model, slaves have
 * dof_eq -1 and prescribed 0; the free numbering is the reference's. */
typedef struct {
  int64_t n_slaves;
  const int64_t* slave_dof;   /* [n_slaves] ascending */
  const int64_t* term_ptr;    /* [n_slaves + 1] offsets into term_eq / term_coeff */
  const int32_t* term_eq;     /* free equation of each term */
  const double* term_coeff;   /* its coefficient */
  const double* constant;     /* [n_slaves] */
} cxg_mpc_desc;

typedef struct cxg_plan cxg_plan;

typedef struct {
  int64_t n_nodes;
  int64_t n_elems;
  int32_t elem_type;
  int32_t n_free;
  int64_t nnz;
  int64_t n_gauss_points;
  int32_t precision;
  int32_t device;
  int64_t device_bytes; /* device memory owned by the plan */
} cxg_plan_info;

CXG_API const char* cxg_last_error(void);
CXG_API int cxg_abi_version(void);
CXG_API int cxg_nodes_per_element(int32_t elem_type);
CXG_API int cxg_gauss_points_per_element(int32_t elem_type);

/* ---- plan: mesh + DOF map resident in device memory, CSR pattern built on device ---
 * Replaces the per-call build_dof_map + hash-map scatter set-up of
 * assemble_linear_static / assemble_material_tangent (src/fem/assembly.cpp:19-42,
 * 76-110, 211-221): the pattern is built once and reused by every assembly. */
CXG_API int cxg_plan_create(const cxg_mesh_desc* mesh, const cxg_dofmap_desc* dofs,
                    int32_t precision, cxg_plan** out);
/* A plan for a model with multi-point constraints. The element pass and row gather
 * assemble the system on an extended numbering in which slave DOFs are equations too;
 * a reduction then forms K_ff = T^T K_x T and rhs = T^T (rhs_x - K_x c), the congruence
 * transform of scatter_block (src/fem/assembly.cpp:76-101) and add_external_load
 * (assembly.cpp:200-208), each CSR value summed in a fixed order. cxg_plan_get_info,
 * the pattern calls, cxg_assemble_linear, cxg_assemble_tangent, cxg_spmv and
 * cxg_solve_cg then work on the reduced free system; f_int stays per global DOF. The
 * other operators return CXG_ERR_UNSUPPORTED on such a plan. */
CXG_API int cxg_plan_create_mpc(const cxg_mesh_desc* mesh, const cxg_dofmap_desc* dofs, const cxg_mpc_desc* mpc,
                                int32_t precision, cxg_plan** out);
CXG_API int cxg_plan_destroy(cxg_plan* plan);
CXG_API int cxg_plan_get_info(const cxg_plan* plan, cxg_plan_info* info);
CXG_API int cxg_plan_set_precision(cxg_plan* plan, int32_t precision);
/* Copy the CSR pattern out (host or device destinations). */
CXG_API int cxg_plan_get_pattern(const cxg_plan* plan, int64_t* row_ptr, int32_t* col_idx);
/* Borrow the plan's device copies of the pattern (valid until destroy). */
CXG_API int cxg_plan_pattern_device(const cxg_plan* plan, const int64_t** row_ptr,
                            const int32_t** col_idx);
/* Replace nodal coordinates [3*n_nodes] (same topology, e.g. design updates). */
CXG_API int cxg_plan_update_coords(cxg_plan* plan, const double* coords);
/* Replace per-element Young's moduli [n_elems]. */
CXG_API int cxg_plan_update_young(cxg_plan* plan, const double* young);
/* Launch shape of the plan's two passes for the current precision; mode 0 = linear
 * assembly, 1 = material-point (tangent) assembly. tile: node-pair tile of the element
 * pass, 0 = 2x4 (default), 1 = 2x2, 2 = 4x4 (linear, mixed precision only);
 * p1_blocks_per_sm: persistent grid of the element pass (0 = all resident);
 * p2_warps: warps per row-gather block, 1 to 8 (0 = up to 8 as shared memory allows). Results
 * do not depend on the shape. */
CXG_API int cxg_plan_set_launch_config(cxg_plan* plan, int32_t mode, int32_t tile, int32_t p1_blocks_per_sm,
                                       int32_t p2_warps);
/* No counterpart in the reference. Mixed-precision material-point assembly: enable != 0
 * runs the J2 return (src/fem/plasticity.cpp:90-236: trial stress, local Newton on the
 * plastic multiplier, stress and history update, tangent parameters) in FP32, with the
 * FP64 return for points whose consistency scalar lies within 1e-3 sigma_y of the yield
 * surface and for points whose FP32 Newton does not settle; 0 (default) keeps the FP64
 * return with FP32 tangent blocks, which measured faster on the B200 (the element pass
 * is not bound by its arithmetic) and keeps the history bit-for-bit FP64. */
CXG_API int cxg_plan_set_j2_fp32_return(cxg_plan* plan, int32_t enable);
/* No counterpart in the reference (a tuning knob of this library). Device-memory
 * budget of the element buffers that carry K_e blocks from the element pass to the
 * row gather. The assembly runs in windows of consecutive elements, each followed by
 * the row gather of the nodes it completes, with the buffers holding only as many
 * elements as the budget allows, so that they stay in L2 between the two passes.
 * 0 (default) or < 0 = one window over the whole mesh (buffers for every element);
 * > 0 = windows whose buffers fit that many bytes. The windows follow from the element ordering: a node
 * waits for its last incident element, so the ring must also hold the largest
 * distance between a node's first and last element; when the budget cannot, the
 * assembly runs as one window. Results do not depend on the budget. */
CXG_API int cxg_plan_set_ring_bytes(cxg_plan* plan, int64_t bytes);
/* The reference's own sparsity pattern for the linear assembly. The reference's scatter
 * skips every element contribution that is exactly 0.0 (src/fem/assembly.cpp:86-90), so
 * an entry whose every contribution is exactly zero in its FP64 arithmetic is absent from
 * its LinearSystem (straight, axis-aligned C3D20 / C3D20R / C3D6 elements have such
 * entries). enable != 0: evaluates every K_e once in the reference's operation order
 * (element.cpp:10-102, 160-462, 529-610; no multiply-add contraction), keeps the CSR
 * entries with at least one nonzero contribution, and from then on cxg_plan_get_info,
 * cxg_plan_get_pattern, cxg_plan_pattern_device, cxg_assemble_linear, cxg_spmv and
 * cxg_solve_cg use that pattern (each assembly runs on the topological pattern and copies
 * the kept entries). The values of the dropped entries are zero to rounding. While it is
 * on, the other operators, CXG_ACCUMULATE and coordinate / modulus updates return
 * CXG_ERR_UNSUPPORTED; enable = 0 returns to the topological pattern. */
CXG_API int cxg_plan_use_reference_pattern(cxg_plan* plan, int32_t enable);
/* Windows of the current precision's linear (mode 0) or tangent (mode 1) assembly and
 * the elements its buffers hold (both from the last assembly of that mode; 0 before). */
CXG_API int cxg_plan_get_windows(const cxg_plan* plan, int32_t mode, int32_t* n_windows, int64_t* ring_elems);
/* Synchronise the stream of the last launch and report the first in-kernel error
 * (CXG_ERR_NEGATIVE_JACOBIAN, CXG_ERR_UNKNOWN_NODE) with the offending element. */
CXG_API int cxg_plan_check(cxg_plan* plan, int64_t* bad_element);

/* ---- assembly ------------------------------------------------------------------
 * Linear static: vals[nnz] = K_ff; rhs[n_free] = T^T f_ext - K_fc u_c
 * (assemble_linear_static, src/fem/assembly.cpp:225-257). f_ext[3*n_nodes] may be
 * NULL. Asynchronous on `stream` (a cudaStream_t, NULL = legacy default stream). */
CXG_API int cxg_assemble_linear(cxg_plan* plan, double* vals, double* rhs, const double* f_ext,
                        void* stream);

/* Flags of the _ex variants. CXG_ACCUMULATE adds this plan's element contributions
 * to the values already in vals (and rhs, f_int) instead of overwriting them, e.g. to
 * sum several meshes that share one DOF numbering and pattern; f_ext is then ignored. */
#define CXG_ACCUMULATE 1
CXG_API int cxg_assemble_linear_ex(cxg_plan* plan, double* vals, double* rhs, const double* f_ext,
                                   int32_t flags, void* stream);

/* Material-point tangent (assemble_material_tangent, src/fem/assembly.cpp:385-423):
 * u[3*n_nodes] full displacement; vals = consistent tangent K_ff; f_int[3*n_nodes] =
 * internal force; rhs = T^T f_ext - K_fc(tangent) u_c where u_c are the plan's
 * prescribed values. Reads the committed state, writes the trial state. f_int, rhs
 * and f_ext may be NULL. */
CXG_API int cxg_assemble_tangent(cxg_plan* plan, const double* u, double* vals, double* f_int,
                         double* rhs, const double* f_ext, void* stream);

/* Consistent (lumped = 0) or lumped (row-sum) mass matrix M_ff on the plan's pattern
 * (assemble_mass, src/fem/assembly.cpp:259-298; element_mass / element_mass_lumped,
 * include/calculixpp/fem/element.hpp:93-102): M_e[3a+i][3b+j] = delta_ij sum_q rho_e
 * detJ w N_a N_b. density[n_elems] per element (Model::element_density). Entries the
 * reference omits as exact zeros (all off-diagonal entries when lumped) are present
 * here as 0.0. *MASS point masses are not part of this entry point. */
CXG_API int cxg_assemble_mass(cxg_plan* plan, const double* density, int32_t lumped, double* vals,
                              void* stream);
/* Geometric (initial-stress) stiffness K_geo on the plan's pattern
 * (assemble_geometric_stiffness, src/fem/assembly.cpp:300-331; element_geometric_stiffness,
 * element.hpp:104-119): K_e[3a+i][3b+j] = delta_ij sum_q detJ w g_a . sigma_q . g_b.
 * gp_stress[6 * n_gauss_points] Voigt {xx,yy,zz,xy,xz,yz} per Gauss point, element
 * order then the Gauss rule's order; NULL means a zero field. */
CXG_API int cxg_assemble_geometric(cxg_plan* plan, const double* gp_stress, double* vals, void* stream);

/* ---- heat conduction (assemble_conduction, src/fem/thermal.cpp:92-141)
 * A temperature plan carries one DOF per node: t_dof_eq[n_nodes] (free equation or -1,
 * free nodes numbered in node order, build_thermal_dof_map, thermal.cpp:71-90) and
 * t_prescribed[n_nodes]; its pattern is the scalar conduction pattern. The mesh's
 * materials are not used. cxg_assemble_conduction writes Kt_ff (element_conduction,
 * element.cpp:745-765: k detJ w g_a . g_b) and rhs = q_f - Kt_fc T_c; conductivity is
 * per element, flux[n_nodes] (may be NULL) is added at the free nodes. */
CXG_API int cxg_thermal_plan_create(const cxg_mesh_desc* mesh, const int32_t* t_dof_eq, const double* t_prescribed,
                                    int32_t n_free, cxg_plan** out);
CXG_API int cxg_assemble_conduction(cxg_plan* plan, const double* conductivity, const double* flux, double* vals,
                                    double* rhs, void* stream);
/* *FILM faces of a temperature plan (Model::films; assemble_conduction, thermal.cpp:
 * 113-126): film f is face face[f] (1-based: tet 1..4, hex 1..6, wedge 1..5, the
 * reference's face numbering, src/fem/loads.cpp:13-46) of element elem[f] (0-based),
 * coefficient h[f], sink temperature sink[f]; host or device arrays, copied. From then on
 * cxg_assemble_conduction adds h int N_a N_b dA to the matrix and h T_sink int N_a dA to
 * the free rows of the rhs (3-point triangle / 2x2 quad face rules). n_films = 0 clears. */
CXG_API int cxg_thermal_plan_set_films(cxg_plan* plan, int64_t n_films, const int64_t* elem, const int32_t* face,
                                       const double* h, const double* sink);

/* ---- thermal strain (*EXPANSION with an applied temperature field) ---------------------
 * Inputs of the reference's thermal-strain path (Material::expansion,
 * Model::applied_temperature; element_temp_change / element_alpha, src/fem/stress.cpp:
 * 76-105): node_temp[n_nodes] the applied temperature of every node, node_applied[n_nodes]
 * 1 where a temperature is applied (NULL: every node), elem_alpha[n_elems] the expansion
 * coefficient of the element's material at the element's mean temperature (nodes without
 * an applied temperature counting as t_ref; 0 for elements without *EXPANSION),
 * elem_tref[n_elems] the material's reference temperature. Host or device arrays, copied.
 * node_temp = NULL clears. Once set, cxg_assemble_linear(_ex) adds the thermal-strain load
 * to the rhs as assemble_linear_static does (src/fem/assembly.cpp:251-253; not with
 * CXG_ACCUMULATE), and the field recovery uses sigma = D (eps - eps_th) and
 * f_int = K u - f_th (stress.cpp:147-271). The material-point assembly ignores it, as the
 * reference's does. */
CXG_API int cxg_plan_set_thermal_strain(cxg_plan* plan, const double* node_temp, const uint8_t* node_applied,
                                        const double* elem_alpha, const double* elem_tref);
/* thermal_strain_load_vector (src/fem/loads.cpp:515-560): f_th[3*n_nodes] = sum_e
 * int B^T D eps_th dV, eps_th = alpha sum_k N_k te_k on the normal components (zeros when
 * no thermal strain is set). */
CXG_API int cxg_thermal_strain_load(cxg_plan* plan, double* f_th, void* stream);

/* ---- field recovery from a displacement field u[3*n_nodes] (linear elasticity) -------
 * recover_gauss_stress (src/fem/stress.cpp:147-187): gp_stress[6 * n_gauss_points],
 * sigma = D (B u_e - eps_th) per Gauss point (Voigt, engineering shear; eps_th = 0 unless
 * cxg_plan_set_thermal_strain), element order. */
CXG_API int cxg_recover_gauss_stress(cxg_plan* plan, const double* u, double* gp_stress, void* stream);
/* recover_fields (stress.cpp:189-271): nodal strain (mechanical, B u) and stress
 * [6 * n_nodes]: each incident element's Gauss-point values extrapolated to the node
 * (the mean for hexahedra, wedges and C3D4; the corner matrix and midside averages for
 * C3D10, include/calculixpp/fem/extrapolation.hpp:26-55), averaged over the elements;
 * reaction[3 * n_nodes] = f_int - f_ext with f_int = sum_e (K_e u_e - f_th_e). Any output
 * and f_ext may be NULL. C3D8R (hourglass forces) is rejected with CXG_ERR_UNSUPPORTED. */
CXG_API int cxg_recover_fields(cxg_plan* plan, const double* u, const double* f_ext, double* strain,
                               double* stress, double* reaction, void* stream);

/* ---- per-Gauss-point history (MaterialPoints, include/calculixpp/fem/assembly.hpp:76-88)
 * committed/trial buffers, 13 doubles per Gauss point. */
CXG_API int cxg_state_get(const cxg_plan* plan, int32_t slot, double* out);
CXG_API int cxg_state_set(cxg_plan* plan, int32_t slot, const double* in);
/* trial -> committed (MaterialPoints::commit, assembly.hpp:84-87). */
CXG_API int cxg_state_commit(cxg_plan* plan, void* stream);

/* ---- element level (element_stiffness / element_tangent_force,
 * include/calculixpp/fem/element.hpp:64-65, 156-164), batched over elements whose
 * coordinates are given per element: coords[n_elems][n][3]. Dense outputs
 * Ke[n_elems][3n][3n], fe[n_elems][3n]. */
CXG_API int cxg_element_stiffness(int32_t elem_type, int64_t n_elems, const double* coords,
                          const double* young, const double* poisson, int32_t precision,
                          double* Ke, void* stream);
CXG_API int cxg_element_tangent_force(int32_t elem_type, int64_t n_elems, const double* coords,
                              const double* ue, const cxg_material* material,
                              const double* state_committed, double* state_trial,
                              int32_t precision, double* Ke, double* fe, void* stream);

/* ---- reduced-system products and solve on the device ------------------------------
 * The device counterpart of ComputeBackend::solve_sparse (include/calculixpp/compute/
 * backend.hpp:51-56; CPU: SciPP spsolve / IC0-CG, src/compute/cpu_backend.cpp:24-72),
 * on the plan's CSR pattern: y = K_ff x, and Jacobi-preconditioned conjugate gradients
 * for K_ff x = rhs from the initial guess in x, stopping at ||r|| <= rtol ||rhs|| or
 * max_iter. Returns CXG_ERR_NOT_CONVERGED (with the reached residual) when the
 * tolerance is not met, as the reference's CG path throws (cpu_backend.cpp:57-62). */
CXG_API int cxg_spmv(cxg_plan* plan, const double* vals, const double* x, double* y, void* stream);
/* ComputeBackend::solve_sparse (include/calculixpp/compute/backend.hpp:51-56) on the
 * device: A x = rhs for A given as COO triplets (rows[k], cols[k], vals[k]) of an n x n
 * SPD matrix, duplicate entries summed; host or device arrays. solver CXG_SOLVER_DIRECT:
 * sparse Cholesky on the device (the reference's spsolve); CXG_SOLVER_IC0_CG: CG
 * preconditioned with a zero-fill incomplete Cholesky factor of A, the reference's CG
 * kind (cpu_backend.cpp:52-63; on a non-positive pivot the factor is retried on
 * A + alpha diag(A), alpha = 1e-4 .. 1e-1, CXG_ERR_NOT_CONVERGED past that);
 * CXG_SOLVER_CG: Jacobi-preconditioned CG (more iterations, no factorisation, no
 * triangular solves). The CG kinds stop at ||r|| <= rtol ||rhs|| and return
 * CXG_ERR_NOT_CONVERGED past max_iter, as the reference throws (cpu_backend.cpp:57-62).
 * iterations / rel_residual may be NULL. */
#define CXG_SOLVER_DIRECT 0
#define CXG_SOLVER_CG 1
#define CXG_SOLVER_IC0_CG 2
CXG_API int cxg_solve_sparse(int32_t n, int64_t nnz, const int32_t* rows, const int32_t* cols, const double* vals,
                             const double* rhs, double* x, int32_t solver, double rtol, int32_t max_iter,
                             int32_t* iterations, double* rel_residual);
CXG_API int cxg_solve_cg(cxg_plan* plan, const double* vals, const double* rhs, double* x, double rtol,
                         int32_t max_iter, int32_t* iterations, double* rel_residual, void* stream);

/* ---- element_tangent_force for callers that cannot allocate device memory --------
 * No counterpart in the reference. Same computation and argument meaning as
 * cxg_element_tangent_force, but the library allocates nothing: code that runs inside
 * another framework's memory pool, a real-time loop or a caller-managed arena may not
 * call cudaMalloc/cudaFree (or any allocating routine). Every array argument must be a
 * device pointer the caller owns; the material table is read from host memory.
 * The J2 history staging, per-element constants and the error word live in one
 * statically sized device buffer of this library (CXG_NOALLOC_SCRATCH_BYTES, held by
 * every GPU that loads the library until the process exits), so one call handles at
 * most CXG_NOALLOC_MAX_GAUSS_POINTS Gauss points (n_elems x points per element);
 * larger batches are rejected with CXG_ERR_INVALID_ARGUMENT. All calls share that
 * buffer: calls whose work overlaps on the GPU (different streams, or different host
 * threads on one device) race with each other and must be serialised by the caller.
 * The first call on each device looks up the buffer's device address; make that first
 * call before any stream capture. The call synchronises `stream` before returning. */
#define CXG_NOALLOC_MAX_GAUSS_POINTS 8192
#define CXG_NOALLOC_SCRATCH_BYTES (2 * 13 * 8 * CXG_NOALLOC_MAX_GAUSS_POINTS + 2 * 8 * CXG_NOALLOC_MAX_GAUSS_POINTS + 4096)
CXG_API int cxg_element_tangent_force_noalloc(int32_t elem_type, int64_t n_elems, const double* coords,
                                              const double* ue, const cxg_material* material,
                                              const double* state_committed, double* state_trial,
                                              int32_t precision, double* Ke, double* fe, void* stream);

/* ---- adjoint of the compliance c = f^T u for K u = f with load independent of the
 * design: dc/dE_e = -(1/E_e) u_e^T K_e u_e and dc/dX = -sum_e u_e^T dK_e/dX u_e,
 * evaluated in closed form per Gauss point. Full-integration families (C3D8, C3D20,
 * C3D20R, C3D6, C3D15) and linear elasticity. The reference computes the coordinate
 * part by central differences of the reduced operator
 * (src/numerics/sensitivity.cpp:77-108). dc_dE[n_elems], dc_dX[3*n_nodes]; either may
 * be NULL. */
CXG_API int cxg_adjoint_compliance(cxg_plan* plan, const double* u, double* dc_dE, double* dc_dX,
                           void* stream);

/* ---- batches: many independent models (elastic or J2) per launch ---------------------
 * No counterpart in the reference, whose drivers assemble one model per call
 * (assemble_linear_static, src/fem/assembly.cpp:225-257); per model the results are
 * those of cxg_assemble_linear on that model alone. A batch groups its models by
 * element type. Each group is one block-diagonal system (the models' meshes and DOF
 * maps concatenated in input order) that one element pass and one row gather
 * assemble. All models' outputs share one vals and one rhs buffer at the offsets that
 * cxg_batch_get_model_info reports, and the load vector is read at 3 * node_offset.
 * Groups are ordered by element type code. Models may be elastic or J2 (materials with a
 * *PLASTIC table); cxg_batch_assemble_tangent assembles the material-point tangent of
 * every model at once. */
typedef struct cxg_batch cxg_batch;

typedef struct {
  int32_t elem_type;
  int32_t group;
  int64_t n_nodes;
  int64_t n_elems;
  int32_t n_free;
  int64_t nnz;
  int64_t vals_offset;  /* first K_ff value of the model in the batch's vals */
  int64_t rhs_offset;   /* first equation of the model in the batch's rhs */
  int64_t node_offset;  /* first node of the model in the batch's node order */
} cxg_batch_model_info;

typedef struct {
  int32_t n_models;
  int32_t n_groups;
  int64_t n_nodes;
  int64_t n_elems;
  int64_t n_free;
  int64_t nnz;
  int64_t device_bytes;
} cxg_batch_info;

CXG_API int cxg_batch_create(int32_t n_models, const cxg_mesh_desc* meshes, const cxg_dofmap_desc* dofs,
                             int32_t precision, cxg_batch** out);
CXG_API int cxg_batch_destroy(cxg_batch* batch);
CXG_API int cxg_batch_get_info(const cxg_batch* batch, cxg_batch_info* info);
CXG_API int cxg_batch_get_model_info(const cxg_batch* batch, int32_t model, cxg_batch_model_info* info);
/* The model's own CSR pattern: row_ptr[n_free + 1] from 0, col_idx[nnz] in the
 * model's equation numbers. */
CXG_API int cxg_batch_get_pattern(const cxg_batch* batch, int32_t model, int64_t* row_ptr, int32_t* col_idx);
CXG_API int cxg_batch_set_precision(cxg_batch* batch, int32_t precision);
/* How one assembly of the batch is launched. CXG_BATCH_PER_GROUP (the default): one
 * element pass and one row gather per element-type group, the groups as independent
 * branches of the graph form. CXG_BATCH_ONE_LAUNCH: one element pass and one row
 * gather for the whole batch (at most 8 groups, one window each), every group a slot
 * of the same persistent grid with a share of its blocks in proportion to the group's
 * pass time as cxg_batch_tune measures it (estimated from the element counts until
 * then). Its element pass takes 2x2 tiles, and 2x4 in mixed precision; the kernel
 * holds the register count of its largest family. Results are the same bit for bit in
 * both modes. Applies to cxg_batch_assemble, cxg_batch_graph_launch,
 * cxg_batch_assemble_tangent and cxg_batch_tune; cxg_batch_group_config and
 * cxg_batch_set_group_config read and pin the current mode's shapes (in the one-launch
 * mode the row gather's warps per block are one value for the whole batch, the last one
 * set, and the element-pass blocks per SM are not used). */
#define CXG_BATCH_PER_GROUP 0
#define CXG_BATCH_ONE_LAUNCH 1
CXG_API int cxg_batch_set_launch(cxg_batch* batch, int32_t mode);
CXG_API int cxg_batch_get_launch(const cxg_batch* batch, int32_t* mode);
/* Assemble every model on `stream` (vals, rhs, f_ext host or device; f_ext may be
 * NULL). */
CXG_API int cxg_batch_assemble(cxg_batch* batch, double* vals, double* rhs, const double* f_ext, void* stream);
/* The same work as one CUDA graph, the groups as independent branches. The first
 * call for a set of buffers and a precision captures the graph; later calls replay it.
 * Device pointers only. */
CXG_API int cxg_batch_graph_launch(cxg_batch* batch, double* vals, double* rhs, const double* f_ext,
                                   void* stream);
/* Synchronise and report the first in-kernel error of any group. */
CXG_API int cxg_batch_check(cxg_batch* batch);
/* Material-point (J2) assembly of every model of the batch at once: per model
 * assemble_material_tangent (src/fem/assembly.cpp:385-423) at its slice of u[3 n_nodes]
 * (batch node order), K_ff into its vals slice, f_int[3 n_nodes] and rhs as
 * cxg_assemble_tangent writes them; each model's history lives in the batch. Device
 * buffers only. Per model the results equal cxg_assemble_tangent on a plan of that model. */
CXG_API int cxg_batch_assemble_tangent(cxg_batch* batch, const double* u, double* vals, double* f_int, double* rhs,
                                       const double* f_ext, void* stream);
/* MaterialPoints::commit (include/calculixpp/fem/assembly.hpp:84-87) for every model. */
CXG_API int cxg_batch_commit(cxg_batch* batch, void* stream);
/* Model `model`'s history (committed or trial), 13 doubles per Gauss point in its element
 * order, as cxg_state_get returns a plan's. */
CXG_API int cxg_batch_get_state(const cxg_batch* batch, int32_t model, int32_t slot, double* out);
/* Autotuner. For every group and the current precision it times each candidate launch
 * shape on the batch's own data with CUDA events: the element-pass node-pair tile
 * (2x4, 2x2 and, in mixed precision, 4x4), its persistent grid (blocks per SM) and
 * the row gather's warps per block. It keeps the fastest of each pass. vals and rhs
 * (device memory) serve as scratch and hold a complete assembly on return. Results are
 * looked up in and added to the JSON file cache_path (NULL: no cache), keyed by SM
 * count, element type, precision and element-count bucket. */
CXG_API int cxg_batch_tune(cxg_batch* batch, double* vals, double* rhs, const double* f_ext,
                           const char* cache_path, void* stream);
/* Read or pin a group's launch shape (tile 0 = 2x4, 1 = 2x2, 2 = 4x4; 0 for a count
 * means the default). */
CXG_API int cxg_batch_group_config(const cxg_batch* batch, int32_t group, int32_t* elem_type, int32_t* tile,
                                   int32_t* p1_blocks_per_sm, int32_t* p2_warps);
CXG_API int cxg_batch_set_group_config(cxg_batch* batch, int32_t group, int32_t tile, int32_t p1_blocks_per_sm,
                                       int32_t p2_warps);

#ifdef __cplusplus
}
#endif
#endif /* CXG_H */
