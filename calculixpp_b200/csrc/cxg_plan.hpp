// The plan object and the host helpers shared by the C-ABI translation units
// (cxg_api.cu: plans and assembly; cxg_batch.cu: batches of plans).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/cxg.h"
#include "cxg_internal.cuh"

namespace cxg {
// Window schedule of the two-pass assembly for one element-buffer footprint: windows of
// consecutive elements, each followed by the row gather of the nodes whose last
// incident element it holds, with element buffers of `ring` elements (slot e mod ring)
// sized to stay in L2 between the two passes. One window (ring = n_elems) when the
// mesh ordering does not allow a ring that small.
struct WinSched {
  bool built = false;
  int64_t ring = 0;
  std::vector<int64_t> win_e;      // [n_win + 1] element offsets
  std::vector<int64_t> win_n;      // [n_win + 1] offsets into node_order
  int32_t* node_order = nullptr;   // device [n_nodes]: nodes by window, mesh order within
};
}  // namespace cxg

namespace cxg {
// The reference's own sparsity pattern (cxg_plan_use_reference_pattern): the entries of
// the topological pattern with at least one nonzero element contribution in the
// reference's arithmetic, and where each sits in the topological pattern.
struct RefPattern {
  bool on = false;
  int64_t nnz = 0;
  int64_t* row_ptr = nullptr;   // [n_free + 1]
  int32_t* col_idx = nullptr;   // [nnz]
  int64_t* src = nullptr;       // [nnz] index of the entry in the topological pattern
  double* topo_vals = nullptr;  // [pat.nnz] one assembly on the topological pattern
};
// A model with multi-point constraints (cxg_plan_create_mpc): the plan itself assembles
// on the extended numbering (slave DOFs kept as equations; n_free and pat are the
// extended ones) and the linear / tangent entry points reduce to the free system.
struct MpcPlan {
  bool on = false;
  int32_t n_free = 0;            // the reference's free equations
  MpcLists lists;
  int32_t* ext_map = nullptr;    // [n_x]
  int64_t* term_ptr = nullptr;
  int32_t* term_eq = nullptr;
  double* term_coeff = nullptr;
  double* c_x = nullptr;         // [n_x] slave constants, null when all are zero
  double* vals_x = nullptr;      // [pat.nnz] one extended assembly
  double* rhs_x = nullptr;       // [n_x]
  double* tmp_x = nullptr;       // [n_x]
  double* kc_x = nullptr;        // [n_x] K_x c
};
}  // namespace cxg

inline cxg::LaunchCfg tangent_default() {
  cxg::LaunchCfg c;
  c.tile = 1;
  return c;
}

struct cxg_plan {
  int device = 0;
  int64_t n_nodes = 0, n_elems = 0, n_gauss = 0;
  int32_t type = 0, n_free = 0, precision = 0;
  double* coords = nullptr;
  int32_t* conn = nullptr;
  double* young = nullptr;
  double* poisson = nullptr;
  int32_t* elem_mat = nullptr;
  cxg::J2Mat* mats = nullptr;
  int32_t n_mats = 0;
  bool has_plastic = false;
  int32_t* dof_eq = nullptr;
  double* prescribed = nullptr;
  cxg::PatternOut pat;
  double* state[2] = {nullptr, nullptr};  // SoA [13][G]: committed, trial
  // The back stress (components 7..12) is zero in both buffers and no material has a
  // kinematic modulus, so it stays zero: the element pass and commit move only the
  // first 7 components. Cleared for good by cxg_state_set.
  bool back_stress_zero = true;
  bool kinematic = false;  // some material has h_kin != 0
  cxg::DevStatus* status = nullptr;
  void* edata = nullptr;      // per-element K blocks of the two-pass assembly
  size_t edata_bytes = 0;
  double* fdata = nullptr;    // per-element internal force (material-point mode)
  size_t fdata_bytes = 0;
  cxg::WinSched sched[2][2];  // [precision][tangent]
  int64_t ring_bytes = 0;     // element-buffer budget: <= 0 one window over the mesh
  std::vector<int32_t> node_first, node_last;  // first / last incident element per node
  cxg::RefPattern refpat;
  cxg::MpcPlan mpc;
  cudaStream_t last_stream = nullptr;
  int64_t device_bytes = 0;
  // staging buffers for host pointers, grown on demand and reused
  void* stage[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  size_t stage_bytes[6] = {0, 0, 0, 0, 0, 0};
  cxg::LaunchCfg cfg[2];   // launch shape of the linear passes per precision (FP64, mixed)
  // launch shape of the material-point (tangent) passes: 2x2 node-pair tiles by default
  // (the J2 tangent tiles carry three accumulator terms; 2x4 measured 1.6x slower)
  cxg::LaunchCfg tcfg[2] = {tangent_default(), tangent_default()};
  bool thermal = false;    // temperature plan: DOF 0 of every node, components 1 and 2 fixed
  // thermal strain (cxg_plan_set_thermal_strain): device copies, null when not set
  double* th_temp = nullptr;
  uint8_t* th_applied = nullptr;
  double* th_alpha = nullptr;
  double* th_tref = nullptr;
  double* th_load = nullptr;  // [3N] scratch: thermal-strain load (+ f_ext) of the linear assembly
  // *FILM faces of a temperature plan (cxg_thermal_plan_set_films); one device block
  cxg::FilmArgs films;
  void* film_mem = nullptr;
};


namespace cxg {
namespace api {

int set_err(int code, const std::string& msg);
int cuda_err(cudaError_t e, const char* where);
bool on_device(const void* p);
// Synchronise the plan's last stream and turn an in-kernel error into a status.
int plan_status(cxg_plan* p, int64_t* bad);
// Allocate the per-element buffers of the two-pass assembly.
// Allocate the per-element buffers of the two-pass assembly (ring-sized when the plan's
// window schedule for this precision and mode has more than one window).
int ensure_v2(cxg_plan* p, bool tangent);
// Arguments of one whole-mesh assembly; apply_windows adds the plan's window schedule
// for the current precision and mode (built by ensure_v2).
V2Args v2_args(cxg_plan* p, const double* f_ext, bool accumulate);
void apply_windows(const cxg_plan* p, bool tangent, V2Args& v);
// J2 history of the material-point assembly: allocated (zeroed) on first use; the number
// of components an assembly reads and writes (7 or 13, see back_stress_zero).
int ensure_state(cxg_plan* p, cudaStream_t s);
int state_comps(const cxg_plan* p);
ElemArgs base_args(cxg_plan* p);

}  // namespace api
}  // namespace cxg

#define CHECK_CUDA(expr, where)                                 \
  do {                                                          \
    cudaError_t _e = (expr);                                    \
    if (_e != cudaSuccess) return cxg::api::cuda_err(_e, where); \
  } while (0)
