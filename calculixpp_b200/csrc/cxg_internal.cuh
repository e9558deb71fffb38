// Internal declarations shared by the kernels (cxg_kernels.cu, cxg_pattern.cu) and
// the C-ABI layer (cxg_api.cu).
#pragma once

#include <cuda_runtime.h>

#include <functional>

#include <cstdint>

#include "cxg_elements.hpp"

namespace cxg {

constexpr int kStateDoubles = 13;  // plastic strain[6], eq. plastic strain, back stress[6]
constexpr int kMaxTable = 64;      // *PLASTIC table points per material

// Device record of one material (J2PlasticMaterial, src/fem/plasticity.cpp:42-65, with
// the kinematic-hardening table adjustment of its constructor already applied).
struct J2Mat {
  int32_t plastic;  // 0: linear elastic
  int32_t n;        // table length
  double h_kin;
  double ep[kMaxTable];
  double sy[kMaxTable];
};

// In-kernel error reporting: first error code and the smallest offending element.
struct DevStatus {
  int32_t code;
  int32_t pad;
  unsigned long long bad_elem;
};

enum KernelMode : int { MODE_LINEAR = 0, MODE_TANGENT = 1 };

// Constant tables (defined in cxg_kernels.cu, filled by ensure_tables): natural
// derivatives dN[k][d][q] (Gauss point fastest) and weights of every family.
constexpr int dn_size(int t) { return nodes_of(t) * 3 * gauss_of(t); }
constexpr int dn_offset(int t) {
  int off = 0;
  for (int u = kFirstType; u < t; ++u) off += dn_size(u);
  return off;
}
constexpr int kDnTotal = dn_offset(C3D15) + dn_size(C3D15);
extern __constant__ double c_dN[kDnTotal];
// Shape-function values N[k][q] (Gauss point fastest) of every family.
constexpr int nn_size(int t) { return nodes_of(t) * gauss_of(t); }
constexpr int nn_offset(int t) {
  int off = 0;
  for (int u = kFirstType; u < t; ++u) off += nn_size(u);
  return off;
}
constexpr int kNTotal = nn_offset(C3D15) + nn_size(C3D15);
extern __constant__ double c_N[kNTotal];
extern __constant__ double c_w[8][kMaxGauss];

// Everything an element-integration launch reads or writes. Pointers are device
// pointers; optional ones may be null.
struct ElemArgs {
  int64_t n_elems;
  int64_t n_nodes;
  // geometry: either a mesh (coords + conn) or per-element coordinates (dense mode)
  const double* coords;     // [3N]
  const int32_t* conn;      // [E*n]
  const double* elem_coords;  // [E*n*3] (dense element-level mode)
  const double* young;      // [E]
  const double* poisson;    // [E]
  const int32_t* elem_mat;  // [E] or null -> material 0
  const J2Mat* mats;        // [n_mats]
  // DOF map / CSR addressing (scatter mode)
  const int64_t* node_base;   // [N] CSR offset of the node's first free row
  const int32_t* node_rowlen; // [N] length of each of the node's rows
  const uint8_t* node_mask;   // [N] bit i: component i free
  const int32_t* node_eq0;    // [N] first free equation of the node (or -1)
  const double* prescribed;   // [3N]
  const uint16_t* slot;       // [E*n*n] position of node b in node a's adjacency list
  const uint16_t* adj_len;    // [N] adjacency list length (row gather)
  const int64_t* bnd_ptr;     // [N+1] adjacency of the compressed-row nodes
  const int32_t* bnd_node;
  // state (tangent mode), SoA [13][G]
  const double* state_c;
  double* state_t;
  int64_t n_gauss;
  // history components the element pass reads and writes: 13, or 7 (plastic strain and
  // equivalent plastic strain) when the back stress is zero in both buffers and no
  // material moves it (every kinematic modulus is 0); components 7..12 are then zero
  // and left untouched
  int state_comps;
  // thermal strain (null th_temp: none): applied temperature per node, whether it is
  // applied (null: every node), expansion coefficient and reference temperature per
  // element (alpha 0: no expansion)
  const double* th_temp;      // [N]
  const uint8_t* th_applied;  // [N]
  const double* th_alpha;     // [E]
  const double* th_tref;      // [E]
  // displacement (tangent mode)
  const double* u;           // [3N] (mesh) or [E*n*3] (dense)
  // outputs
  double* vals;   // [nnz]
  double* rhs;    // [n_free]
  double* f_int;  // [3N]
  double* Ke;     // dense [E*(3n)^2]
  double* fe;     // dense [E*3n]
  DevStatus* status;
};

// Extra arguments of the two-pass assembly (cxg_v2.cu).
struct V2Args {
  void* edata;              // per-element upper 3x3 blocks, FP32 (mixed) or FP64
  double* fdata;            // per-element internal force [E*3n] (material-point mode)
  const int64_t* inc_ptr;   // node -> incident elements
  const int32_t* inc_code;
  const double* f_ext;      // [3N] load vector for the rhs, or null
  int64_t max_adj;          // longest adjacency list of any node
  int64_t row_stride;       // set by the launcher: doubles per row-buffer copy
  int accumulate;           // add into vals / rhs / f_int instead of overwriting
  // The window of one element-pass + row-gather pair: the element pass integrates
  // elements [e_begin, e_end), the row gather the nodes node_order[n_begin..n_end)
  // (node_order null: nodes n_begin..n_end in mesh order). The element buffers hold
  // `ring` elements; element e lives in slot e mod ring.
  int64_t e_begin, e_end, ring, ring_base;
  const int32_t* node_order;
  int64_t n_begin, n_end;
  // Window schedule read by the launcher (host arrays): n_win windows with element
  // offsets win_e[0..n_win] and node-list offsets win_n[0..n_win]; n_win <= 1 runs the
  // whole mesh as one window.
  int32_t n_win;
  const int64_t* win_e;
  const int64_t* win_n;
};
// Launch shape of the two passes. tile: element-pass node-pair tile (0 = 2x4, 1 = 2x2,
// 2 = 4x4, the last in the linear pass with FP32 accumulators only);
// *_blocks_per_sm: persistent grid per SM (0 = as many as are resident); p2_warps:
// warps per row-gather block, at most 8 (0 = up to 8 as shared memory allows); passes: bit 0 the
// element pass, bit 1 the row gather.
struct LaunchCfg {
  int tile = 0;
  int p1_blocks_per_sm = 0;
  int p2_warps = 0;
  int p2_blocks_per_sm = 0;
  int passes = 3;
  // mixed-precision material-point pass: the J2 return in FP32 (j2_point_mixed) instead
  // of FP64
  int j2_fp32 = 0;
};
// One element pass and one row gather for a whole batch of element-type groups: slot k
// is group k's arguments (one window, mesh node order), its element type and launch
// shape; the weights share the persistent grid of each pass between the slots.
constexpr int kMaxBatchSlots = 8;
struct BatchSlotIn {
  ElemArgs a;
  V2Args v;
  int32_t type = 0;
  LaunchCfg cfg;
  double p1_weight = 1.0, p2_weight = 1.0;
};
cudaError_t launch_v2_batch(int mode, int precision, const BatchSlotIn* slots, int n_slots, int passes,
                            cudaStream_t s);
// Tiles the batch kernels take (2x2; 2x4 in the mixed-precision linear pass).
bool batch_tile_ok(int mode, int precision, int tile);
size_t v2_edata_bytes(int elem_type, int64_t n_elems, int precision);
// Bytes of element buffer per element (blocks, plus the internal force in tangent mode).
size_t v2_bytes_per_element(int elem_type, int precision, bool tangent);
// Element pass of the scalar-block operators (every 3x3 block is a scalar times I):
// kind 1 consistent mass rho N_a N_b, 2 lumped mass (row sums on the diagonal), 3
// geometric stiffness g_a . sigma . g_b, 4 conduction k g_a . g_b. Writes FP64 blocks
// for the FP64 row gather. density[E] is rho (kinds 1, 2) or k (kind 4), gp_stress[6 G]
// (kind 3).
cudaError_t launch_scalar_pass(int elem_type, int kind, const ElemArgs& a, const V2Args& v, const double* density,
                               const double* gp_stress, cudaStream_t s);
cudaError_t launch_v2(int elem_type, int mode, int precision, const ElemArgs& a, const V2Args& v, cudaStream_t s,
                      const LaunchCfg& cfg = LaunchCfg{});

// The reference's own pattern (cxg_refpattern.cu): launch_refmask writes, per element and
// in the FP64 element-buffer layout, 1.0 where the reference's K_e (its operation order)
// is nonzero and 0.0 where it is exactly zero; compact_pattern keeps the CSR entries whose
// gathered count is positive (row_ptr_c, col_idx_c, and src = their topological index);
// gather_values copies a topological assembly onto the kept entries.
cudaError_t launch_refmask(int elem_type, const ElemArgs& a, double* out, cudaStream_t s);
cudaError_t compact_pattern(const int64_t* row_ptr, const int32_t* col_idx, int32_t n_rows, int64_t nnz,
                            const double* counts, int64_t** row_ptr_c, int32_t** col_idx_c, int64_t** src,
                            int64_t* nnz_c, cudaStream_t s);
cudaError_t gather_values(const int64_t* src, const double* topo, int64_t nnz_c, double* out, cudaStream_t s);

// Multi-point constraints (cxg_mpc.cu): the reduced CSR of K_ff = T^T K_x T and, per
// reduced entry, the list of (extended entry, weight) pairs it sums (tgt_ptr / src / w);
// per free equation, the list of (extended row, weight) pairs of T^T (rhs_ptr / rhs_src /
// rhs_w).
struct MpcLists {
  int64_t nnz = 0;
  int64_t* row_ptr = nullptr;
  int32_t* col_idx = nullptr;
  int64_t* tgt_ptr = nullptr;
  int64_t* src = nullptr;
  double* w = nullptr;
  int64_t* rhs_ptr = nullptr;
  int64_t* rhs_src = nullptr;
  double* rhs_w = nullptr;
};
// ext_map[x]: free equation of extended equation x, or -1 - s for slave s whose terms are
// [term_ptr[s], term_ptr[s+1]) of term_eq / term_coeff.
cudaError_t build_mpc_reduce(const int64_t* x_row_ptr, const int32_t* x_col, int64_t n_x, int64_t nnz_x,
                             const int32_t* ext_map, const int64_t* term_ptr, const int32_t* term_eq,
                             const double* term_coeff, int32_t n_free, MpcLists* out, cudaStream_t s);
cudaError_t mpc_reduce_values(const MpcLists& m, const double* vals_x, double* vals, cudaStream_t s);
// rhs = T^T (rhs_x - kc), kc = K_x c (null when every constant is zero); tmp_x[n_x] scratch.
cudaError_t mpc_reduce_rhs(const MpcLists& m, const double* rhs_x, const double* kc, int64_t n_x, double* tmp_x,
                           int32_t n_free, double* rhs, cudaStream_t s);

// Launchers (cxg_kernels.cu). `precision` 0 = FP64, 1 = mixed.
cudaError_t launch_element_kernel(int elem_type, int mode, bool dense, int precision,
                                  const ElemArgs& a, cudaStream_t s);
cudaError_t launch_rhs_init(const int32_t* dof_eq, const double* f_ext, int64_t ndof,
                            double* rhs, cudaStream_t s);
cudaError_t launch_state_transpose(const double* src, double* dst, int64_t G, bool to_soa,
                                   cudaStream_t s);
// Field recovery (cxg_recover.cu): a.u is the full displacement. gp_stress[6G] may be
// null; emean[12E] and felem[3nE] are scratch for the node pass (both null: Gauss-point
// stress only); strain/stress[6N], reaction[3N] outputs.
cudaError_t launch_recover(int elem_type, const ElemArgs& a, const int64_t* inc_ptr, const int32_t* inc_code,
                           double* gp_stress, double* emean, double* felem, const double* f_ext, double* strain,
                           double* stress, double* reaction, bool thermal_load, cudaStream_t s);
// *FILM faces of a temperature plan (cxg_film.cu), device arrays built once per film set:
// films grouped by element (felem[g] owns flist[fptr[g] .. fptr[g+1]), in film order),
// and per face node the (film, face-local index) entries film * 8 + i it receives
// (fnode[g] owns fnlist[fnptr[g] .. fnptr[g+1]), in film order); load[8 * n_films] holds
// h T_sink int N_i dA between the two passes.
struct FilmArgs {
  int64_t n_films = 0, n_felem = 0, n_fnode = 0;
  const int64_t* felem = nullptr;
  const int32_t* fptr = nullptr;
  const int32_t* flist = nullptr;
  const int32_t* face = nullptr;
  const double* h = nullptr;
  const double* sink = nullptr;
  const int64_t* fnode = nullptr;
  const int32_t* fnptr = nullptr;
  const int32_t* fnlist = nullptr;
  double* load = nullptr;
};
cudaError_t launch_films(int elem_type, const ElemArgs& a, const FilmArgs& f, double* edata, double* f_ext3,
                         cudaStream_t s);
cudaError_t launch_adjoint(int elem_type, const ElemArgs& a, double* dc_dE, double* dc_dX,
                           cudaStream_t s);
cudaError_t launch_spmv(int32_t nrows, const int64_t* rp, const int32_t* ci, const double* v, const double* x,
                        double* y, cudaStream_t s);
// Jacobi-preconditioned CG on CSR; work holds 5*n + 2056 doubles.
cudaError_t cg_solve(int32_t n, const int64_t* rp, const int32_t* ci, const double* v, const double* b, double* x,
                     double rtol, int max_iter, double* work, int* iters_out, double* rel_out, cudaStream_t s);
// The same CG loop with z = M^-1 r given by `precond` (launched on the loop's stream);
// work holds 5*n + 2056 doubles, the fifth n-vector unused by the loop.
using Preconditioner = std::function<cudaError_t(const double* r, double* z)>;
cudaError_t pcg_solve(int32_t n, const int64_t* rp, const int32_t* ci, const double* v, const double* b, double* x,
                      double rtol, int max_iter, double* work, int* iters_out, double* rel_out, cudaStream_t s,
                      const Preconditioner& precond);
// Element tables (constant memory) are uploaded once per device.
cudaError_t ensure_tables();

// Pattern construction (cxg_pattern.cu).
struct PatternOut {
  int64_t nnz = 0;
  int64_t* row_ptr = nullptr;   // [n_free+1]
  int32_t* col_idx = nullptr;   // [nnz]
  int64_t* node_base = nullptr;
  int32_t* node_rowlen = nullptr;
  uint8_t* node_mask = nullptr;
  int32_t* node_eq0 = nullptr;
  uint16_t* slot = nullptr;     // [E*n*n] position of node b in node a's adjacency list
  // node adjacency (neighbours of a node, itself included, ascending): the list length
  // of every node, and the list itself for the nodes with a neighbour that is not fully
  // free (bnd_node[bnd_ptr[a] .. bnd_ptr[a+1]); empty for the others)
  uint16_t* adj_len = nullptr;  // [N]
  int64_t* bnd_ptr = nullptr;   // [N+1]
  int32_t* bnd_node = nullptr;
  // node -> incident elements, ascending element order: codes e*n + local node index
  int64_t* inc_ptr = nullptr;   // [N+1]
  int32_t* inc_code = nullptr;  // [E*n]
  int64_t max_row = 0;          // max over nodes of (free rows) x (row length)
  int64_t max_adj = 0;          // max over nodes of the adjacency list length
  int64_t device_bytes = 0;
};
// Returns a cxg_status code; on error *msg is set.
int build_pattern(int elem_type, int64_t n_nodes, int64_t n_elems, const int32_t* d_conn,
                  const int32_t* d_dof_eq, int32_t n_free, PatternOut* out, const char** msg,
                  cudaStream_t s);

}  // namespace cxg
