// C ABI of libcxg.so (declared in include/cxg.h).
//
// Host-side runtime around the kernels: plan construction (mesh and DOF map made
// resident in device memory, CSR pattern built on the device), host/device pointer
// staging through plan-owned buffers, the assembly entry points, the per-Gauss-point
// history round trips and the element-level batched entry points. No exception
// crosses the ABI: every entry point returns a cxg_status and leaves a message for
// cxg_last_error().
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "cxg_faces.hpp"
#include "cxg_plan.hpp"

using namespace cxg;
using namespace cxg::api;

namespace {
thread_local std::string g_err;
}  // namespace

namespace cxg {
namespace api {

int set_err(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int cuda_err(cudaError_t e, const char* where) {
  if (e == cudaErrorMemoryAllocation)
    return set_err(CXG_ERR_OUT_OF_MEMORY, std::string(where) + ": " + cudaGetErrorString(e));
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
    return set_err(CXG_ERR_NO_GPU, std::string(where) + ": " + cudaGetErrorString(e));
  return set_err(CXG_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

bool on_device(const void* p) {
  if (!p) return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

}  // namespace api
}  // namespace cxg

namespace {

template <typename T>
cudaError_t alloc_copy(T** dst, const T* src, size_t count, cudaStream_t s, int64_t* bytes) {
  *bytes += static_cast<int64_t>(count * sizeof(T));
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(dst), std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess || !src || count == 0) return e;
  return cudaMemcpyAsync(*dst, src, count * sizeof(T), cudaMemcpyDefault, s);
}

// Device view of a caller buffer: the pointer itself when it is device memory, else a
// plan staging buffer (slot), filled from the host when `upload`.
int staged(cxg_plan* p, int slot, const void* ptr, size_t bytes, bool upload, cudaStream_t s,
           void** out) {
  if (!ptr) {
    *out = nullptr;
    return CXG_OK;
  }
  if (on_device(ptr)) {
    *out = const_cast<void*>(ptr);
    return CXG_OK;
  }
  if (p->stage_bytes[slot] < bytes) {
    cudaFree(p->stage[slot]);
    p->stage[slot] = nullptr;
    p->stage_bytes[slot] = 0;
    CHECK_CUDA(cudaMalloc(&p->stage[slot], bytes), "staging allocation");
    p->stage_bytes[slot] = bytes;
  }
  if (upload) CHECK_CUDA(cudaMemcpyAsync(p->stage[slot], ptr, bytes, cudaMemcpyHostToDevice, s), "upload");
  *out = p->stage[slot];
  return CXG_OK;
}

int build_mats(int32_t n, const cxg_material* m, std::vector<J2Mat>& out, bool* plastic) {
  out.assign(static_cast<size_t>(n), J2Mat{});
  *plastic = false;
  for (int32_t i = 0; i < n; ++i) {
    J2Mat& d = out[static_cast<size_t>(i)];
    const cxg_material& s = m[i];
    if (!(s.E > 0.0) || !(s.nu > -1.0 && s.nu < 0.5))
      return set_err(CXG_ERR_INVALID_ARGUMENT, "material needs E > 0 and -1 < nu < 0.5");
    d.plastic = s.n_plastic > 0 ? 1 : 0;
    d.n = s.n_plastic > 0 ? s.n_plastic : 1;
    d.h_kin = s.h_kin;
    if (s.n_plastic > kMaxTable)
      return set_err(CXG_ERR_UNSUPPORTED, "*PLASTIC table longer than 64 points");
    if (s.n_plastic > 0) {
      if (!s.eqplastic || !s.yield) return set_err(CXG_ERR_INVALID_ARGUMENT, "*PLASTIC table pointers are null");
      for (int k = 0; k < s.n_plastic; ++k) {
        d.ep[k] = s.eqplastic[k];
        d.sy[k] = s.yield[k];
      }
      // J2PlasticMaterial constructor (src/fem/plasticity.cpp:57-63): kinematic /
      // combined hardening takes H_kin from the first table slope when it is not given;
      // pure kinematic hardening flattens the isotropic curve to the initial yield.
      if (s.hardening == 1 || s.hardening == 2) {
        if (d.h_kin == 0.0 && s.n_plastic >= 2 && d.ep[1] > d.ep[0])
          d.h_kin = (d.sy[1] - d.sy[0]) / (d.ep[1] - d.ep[0]);
        if (s.hardening == 1)
          for (int k = 0; k < s.n_plastic; ++k) d.sy[k] = d.sy[0];
      }
      *plastic = true;
    }
  }
  return CXG_OK;
}

__global__ void fill_props_kernel(const int32_t* elem_mat, const double* E, const double* nu, int n_mats,
                                  int64_t n_elems, double* young, double* poisson, int* bad) {
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n_elems;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int m = elem_mat ? elem_mat[e] : 0;
    if (m < 0 || m >= n_mats) {
      atomicExch(bad, 1);
      m = 0;
    }
    if (young) young[e] = E[m];
    if (poisson) poisson[e] = nu[m];
  }
}

}  // namespace

namespace cxg {
namespace api {
int plan_status(cxg_plan* p, int64_t* bad) {
  CHECK_CUDA(cudaStreamSynchronize(p->last_stream), "synchronize");
  DevStatus st;
  CHECK_CUDA(cudaMemcpy(&st, p->status, sizeof st, cudaMemcpyDeviceToHost), "status read");
  if (bad) *bad = st.code ? static_cast<int64_t>(st.bad_elem) : -1;
  if (st.code) {
    DevStatus z{0, 0, ~0ull};
    cudaMemcpy(p->status, &z, sizeof z, cudaMemcpyHostToDevice);
    char buf[160];
    if (st.code == CXG_ERR_NEGATIVE_JACOBIAN)
      snprintf(buf, sizeof buf, "non-positive element Jacobian (bad connectivity?) at element index %llu",
               st.bad_elem);
    else
      snprintf(buf, sizeof buf, "in-kernel error %d at element index %llu", st.code, st.bad_elem);
    return set_err(st.code, buf);
  }
  return CXG_OK;
}
}  // namespace api
}  // namespace cxg

namespace {

// The CSR the plan's linear assembly returns: the reference's pattern when the plan uses
// it (cxg_plan_use_reference_pattern), the topological one otherwise.
// A plan with multi-point constraints returns the reduced free system.
int64_t active_nnz(const cxg_plan* p) {
  return p->mpc.on ? p->mpc.lists.nnz : p->refpat.on ? p->refpat.nnz : p->pat.nnz;
}
const int64_t* active_row_ptr(const cxg_plan* p) {
  return p->mpc.on ? p->mpc.lists.row_ptr : p->refpat.on ? p->refpat.row_ptr : p->pat.row_ptr;
}
const int32_t* active_col_idx(const cxg_plan* p) {
  return p->mpc.on ? p->mpc.lists.col_idx : p->refpat.on ? p->refpat.col_idx : p->pat.col_idx;
}
int32_t active_n_free(const cxg_plan* p) { return p->mpc.on ? p->mpc.n_free : p->n_free; }

// K_ff and rhs of a plan with multi-point constraints from its extended assembly
// (mpc.vals_x, mpc.rhs_x): vals = T^T K_x T, rhs = T^T (rhs_x - K_x c).
cudaError_t mpc_reduce(cxg_plan* p, double* vals, double* rhs, cudaStream_t s) {
  const MpcPlan& m = p->mpc;
  cudaError_t e = mpc_reduce_values(m.lists, m.vals_x, vals, s);
  if (e != cudaSuccess || !rhs) return e;
  if (m.c_x) {
    e = launch_spmv(p->n_free, p->pat.row_ptr, p->pat.col_idx, m.vals_x, m.c_x, m.kc_x, s);
    if (e != cudaSuccess) return e;
  }
  return mpc_reduce_rhs(m.lists, m.rhs_x, m.c_x ? m.kc_x : nullptr, p->n_free, m.tmp_x, m.n_free, rhs, s);
}

int reject_mpc(const cxg_plan* p) {
  return p->mpc.on ? set_err(CXG_ERR_UNSUPPORTED,
                             "plans with multi-point constraints cover the linear and tangent assembly")
                   : CXG_OK;
}

int reject_refpat(const cxg_plan* p) {
  if (p->mpc.on) return reject_mpc(p);
  return p->refpat.on ? set_err(CXG_ERR_UNSUPPORTED,
                                "the reference pattern covers the linear assembly; switch it off for this operator")
                      : CXG_OK;
}

}  // namespace

namespace cxg {
namespace api {

// History components an assembly must carry (see cxg_plan::back_stress_zero).
int state_comps(const cxg_plan* p) { return (p->back_stress_zero && !p->kinematic) ? 7 : kStateDoubles; }

int ensure_state(cxg_plan* p, cudaStream_t s) {
  if (p->state[0]) return CXG_OK;
  const size_t bytes = sizeof(double) * kStateDoubles * static_cast<size_t>(std::max<int64_t>(p->n_gauss, 1));
  for (int i = 0; i < 2; ++i) {
    CHECK_CUDA(cudaMalloc(&p->state[i], bytes), "state allocation");
    CHECK_CUDA(cudaMemsetAsync(p->state[i], 0, bytes, s), "state init");
  }
  p->device_bytes += 2 * static_cast<int64_t>(bytes);
  return CXG_OK;
}

namespace windows {

__global__ void node_span_kernel(const int64_t* inc_ptr, const int32_t* inc_code, int n, int64_t n_nodes,
                                 int32_t* first, int32_t* last) {
  for (int64_t a = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; a < n_nodes;
       a += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i0 = inc_ptr[a], i1 = inc_ptr[a + 1];
    first[a] = i1 > i0 ? inc_code[i0] / n : -1;
    last[a] = i1 > i0 ? inc_code[i1 - 1] / n : -1;
  }
}

// Smallest window worth a launch pair under the default budget: a few waves of the
// element pass. An explicit budget (cxg_plan_set_ring_bytes) is taken as given, down to
// windows of 32 elements.
constexpr int64_t kMinWindow = 8192;

// Window schedule for `bpe` bytes of element buffer per element (see cxg::WinSched).
// Window size W: the ring holds W + span elements, span being the largest distance
// between a node's first and last incident element, within the plan's budget. Node a
// is gathered in window last(a) / W; every element it needs is then among the last
// W + span elements integrated, which the ring still holds.
int build_schedule(cxg_plan* p, size_t bpe, WinSched& w) {
  w.built = true;
  w.ring = std::max<int64_t>(p->n_elems, 1);
  w.win_e.clear();
  w.win_n.clear();
  const int64_t min_w = p->ring_bytes > 0 ? 32 : kMinWindow, grain = p->ring_bytes > 0 ? 32 : 1024;
  // default (0) and negative budgets: one window. Measured on the B200, windows lost at
  // every budget tried (C3D8 J2 128^3: 11.2 ms one window, 14.2-15.6 ms windowed; C3D20
  // 64^3 mixed: 6.9 against 7.2 ms): the two passes are not HBM-bound, and every window
  // adds two launches and a tail. The tuner still tries L2-sized budgets.
  if (p->ring_bytes <= 0 || p->n_elems < 2 * min_w) return CXG_OK;
  if (p->node_first.empty()) {
    int32_t* d = nullptr;
    CHECK_CUDA(cudaMalloc(&d, sizeof(int32_t) * 2 * static_cast<size_t>(p->n_nodes)), "node spans");
    const unsigned grid = static_cast<unsigned>(std::min<int64_t>((p->n_nodes + 255) / 256, 4096));
    node_span_kernel<<<grid, 256>>>(p->pat.inc_ptr, p->pat.inc_code, nodes_of(p->type), p->n_nodes, d,
                                    d + p->n_nodes);
    cudaError_t e = cudaGetLastError();
    p->node_first.resize(static_cast<size_t>(p->n_nodes));
    p->node_last.resize(static_cast<size_t>(p->n_nodes));
    if (e == cudaSuccess)
      e = cudaMemcpy(p->node_first.data(), d, sizeof(int32_t) * p->n_nodes, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
      e = cudaMemcpy(p->node_last.data(), d + p->n_nodes, sizeof(int32_t) * p->n_nodes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) p->node_first.clear();
    CHECK_CUDA(e, "node spans");
  }
  int64_t span = 1;
  for (int64_t a = 0; a < p->n_nodes; ++a)
    if (p->node_last[a] >= 0) span = std::max<int64_t>(span, p->node_last[a] - p->node_first[a] + 1);
  const int64_t budget = p->ring_bytes;
  const int64_t W = (budget / static_cast<int64_t>(bpe) - span) / grain * grain;
  if (W < min_w || W * 2 > p->n_elems) return CXG_OK;
  const int64_t n_win = (p->n_elems + W - 1) / W;
  std::vector<int64_t> count(static_cast<size_t>(n_win) + 1, 0);
  for (int64_t a = 0; a < p->n_nodes; ++a) ++count[static_cast<size_t>(std::max(p->node_last[a], 0) / W) + 1];
  w.win_n.assign(static_cast<size_t>(n_win) + 1, 0);
  for (int64_t k = 0; k < n_win; ++k) w.win_n[k + 1] = w.win_n[k] + count[k + 1];
  std::vector<int32_t> order(static_cast<size_t>(p->n_nodes));
  std::vector<int64_t> pos(w.win_n.begin(), w.win_n.end() - 1);
  for (int64_t a = 0; a < p->n_nodes; ++a)
    order[static_cast<size_t>(pos[static_cast<size_t>(std::max(p->node_last[a], 0) / W)]++)] = static_cast<int32_t>(a);
  if (!w.node_order) {
    CHECK_CUDA(cudaMalloc(&w.node_order, sizeof(int32_t) * static_cast<size_t>(p->n_nodes)), "node order");
    p->device_bytes += static_cast<int64_t>(sizeof(int32_t) * p->n_nodes);
  }
  CHECK_CUDA(cudaMemcpy(w.node_order, order.data(), sizeof(int32_t) * p->n_nodes, cudaMemcpyHostToDevice),
             "node order");
  w.win_e.resize(static_cast<size_t>(n_win) + 1);
  for (int64_t k = 0; k <= n_win; ++k) w.win_e[static_cast<size_t>(k)] = std::min(k * W, p->n_elems);
  w.ring = W + span;
  return CXG_OK;
}

}  // namespace windows

int ensure_v2(cxg_plan* p, bool tangent) {
  WinSched& w = p->sched[p->precision][tangent ? 1 : 0];
  if (!w.built) {
    const int rc = windows::build_schedule(p, v2_bytes_per_element(p->type, p->precision, tangent), w);
    if (rc) return rc;
  }
  const size_t need = v2_edata_bytes(p->type, w.ring, p->precision);
  if (p->edata_bytes < need) {
    cudaFree(p->edata);
    p->edata = nullptr;
    p->device_bytes -= static_cast<int64_t>(p->edata_bytes);
    p->edata_bytes = 0;
    CHECK_CUDA(cudaMalloc(&p->edata, std::max<size_t>(need, 16)), "element buffer");
    p->edata_bytes = need;
    p->device_bytes += static_cast<int64_t>(need);
  }
  const size_t fb = sizeof(double) * 3 * nodes_of(p->type) * static_cast<size_t>(w.ring);
  if (tangent && p->fdata_bytes < fb) {
    cudaFree(p->fdata);
    p->fdata = nullptr;
    p->device_bytes -= static_cast<int64_t>(p->fdata_bytes);
    p->fdata_bytes = 0;
    CHECK_CUDA(cudaMalloc(&p->fdata, fb), "force buffer");
    p->fdata_bytes = fb;
    p->device_bytes += static_cast<int64_t>(fb);
  }
  return CXG_OK;
}

void apply_windows(const cxg_plan* p, bool tangent, V2Args& v) {
  const WinSched& w = p->sched[p->precision][tangent ? 1 : 0];
  if (!w.built || w.win_e.size() < 3) return;
  v.ring = w.ring;
  v.node_order = w.node_order;
  v.n_win = static_cast<int32_t>(w.win_e.size() - 1);
  v.win_e = w.win_e.data();
  v.win_n = w.win_n.data();
}

V2Args v2_args(cxg_plan* p, const double* f_ext, bool accumulate) {
  V2Args v{};
  v.edata = p->edata;
  v.fdata = p->fdata;
  v.inc_ptr = p->pat.inc_ptr;
  v.inc_code = p->pat.inc_code;
  v.f_ext = f_ext;
  v.max_adj = p->pat.max_adj;
  v.accumulate = accumulate ? 1 : 0;
  v.e_begin = 0;
  v.e_end = p->n_elems;
  v.ring = std::max<int64_t>(p->n_elems, 1);
  v.ring_base = 0;
  v.node_order = nullptr;
  v.n_begin = 0;
  v.n_end = p->n_nodes;
  v.n_win = 0;
  return v;
}

ElemArgs base_args(cxg_plan* p) {
  ElemArgs a{};
  a.n_elems = p->n_elems;
  a.n_nodes = p->n_nodes;
  a.coords = p->coords;
  a.conn = p->conn;
  a.young = p->young;
  a.poisson = p->poisson;
  a.elem_mat = p->elem_mat;
  a.mats = p->mats;
  a.node_base = p->pat.node_base;
  a.node_rowlen = p->pat.node_rowlen;
  a.node_mask = p->pat.node_mask;
  a.node_eq0 = p->pat.node_eq0;
  a.prescribed = p->prescribed;
  a.slot = p->pat.slot;
  a.adj_len = p->pat.adj_len;
  a.bnd_ptr = p->pat.bnd_ptr;
  a.bnd_node = p->pat.bnd_node;
  a.n_gauss = p->n_gauss;
  a.status = p->status;
  a.th_temp = p->th_temp;
  a.th_applied = p->th_applied;
  a.th_alpha = p->th_alpha;
  a.th_tref = p->th_tref;
  return a;
}

}  // namespace api
}  // namespace cxg

namespace {

int copy_out(void* dst, const void* dev, size_t bytes, cudaStream_t s) {
  if (!dst || dst == dev) return CXG_OK;
  CHECK_CUDA(cudaMemcpyAsync(dst, dev, bytes, cudaMemcpyDefault, s), "download");
  return CXG_OK;
}

}  // namespace

extern "C" {

const char* cxg_last_error(void) { return g_err.c_str(); }
int cxg_abi_version(void) { return CXG_ABI_VERSION; }
int cxg_nodes_per_element(int32_t t) { return nodes_of(t); }
int cxg_gauss_points_per_element(int32_t t) { return gauss_of(t); }

int cxg_plan_create(const cxg_mesh_desc* m, const cxg_dofmap_desc* d, int32_t precision, cxg_plan** out) {
  if (!m || !d || !out) return set_err(CXG_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (!supported(m->elem_type)) return set_err(CXG_ERR_UNSUPPORTED, "unsupported element type");
  if (m->n_nodes <= 0 || m->n_elems < 0 || !m->coords || (m->n_elems > 0 && !m->conn))
    return set_err(CXG_ERR_INVALID_ARGUMENT, "mesh needs n_nodes > 0, coords and conn");
  if (m->n_materials < 1 || !m->materials) return set_err(CXG_ERR_INVALID_ARGUMENT, "mesh needs >= 1 material");
  if (!d->dof_eq || !d->prescribed || d->n_free < 0) return set_err(CXG_ERR_INVALID_ARGUMENT, "bad DOF map");
  if (precision != CXG_FP64 && precision != CXG_MIXED) return set_err(CXG_ERR_INVALID_ARGUMENT, "bad precision");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_err(CXG_ERR_NO_GPU, "no CUDA device");
  }
  CHECK_CUDA(ensure_tables(), "constant tables");

  std::vector<J2Mat> mats;
  bool plastic = false;
  int rc = build_mats(m->n_materials, m->materials, mats, &plastic);
  if (rc) return rc;

  auto* p = new cxg_plan;
  cudaGetDevice(&p->device);
  p->n_nodes = m->n_nodes;
  p->n_elems = m->n_elems;
  p->type = m->elem_type;
  p->n_free = d->n_free;
  p->precision = precision;
  p->n_gauss = m->n_elems * gauss_of(m->elem_type);
  p->n_mats = m->n_materials;
  p->has_plastic = plastic;
  for (const J2Mat& jm : mats) p->kinematic = p->kinematic || jm.h_kin != 0.0;
  const int npe = nodes_of(m->elem_type);
  cudaStream_t s = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete p;
    return cuda_err(e, "stream");
  }
  auto fail = [&](int code) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    cxg_plan_destroy(p);
    return code;
  };
#define TRYC(expr, where)                    \
  do {                                       \
    cudaError_t _e = (expr);                 \
    if (_e != cudaSuccess) return fail(cuda_err(_e, where)); \
  } while (0)
  TRYC(alloc_copy(&p->coords, m->coords, 3 * static_cast<size_t>(m->n_nodes), s, &p->device_bytes), "coords");
  TRYC(alloc_copy(&p->conn, m->conn, static_cast<size_t>(m->n_elems) * npe, s, &p->device_bytes), "conn");
  TRYC(alloc_copy(&p->dof_eq, d->dof_eq, 3 * static_cast<size_t>(m->n_nodes), s, &p->device_bytes), "dof_eq");
  TRYC(alloc_copy(&p->prescribed, d->prescribed, 3 * static_cast<size_t>(m->n_nodes), s, &p->device_bytes),
       "prescribed");
  TRYC(alloc_copy(&p->mats, mats.data(), mats.size(), s, &p->device_bytes), "materials");
  if (m->elem_mat)
    TRYC(alloc_copy(&p->elem_mat, m->elem_mat, static_cast<size_t>(m->n_elems), s, &p->device_bytes), "elem_mat");
  TRYC(alloc_copy(&p->young, m->young, static_cast<size_t>(m->n_elems), s, &p->device_bytes), "young");
  TRYC(alloc_copy(&p->poisson, m->poisson, static_cast<size_t>(m->n_elems), s, &p->device_bytes), "poisson");
  {
    std::vector<double> E(static_cast<size_t>(m->n_materials)), nu(E.size());
    for (int32_t i = 0; i < m->n_materials; ++i) {
      E[static_cast<size_t>(i)] = m->materials[i].E;
      nu[static_cast<size_t>(i)] = m->materials[i].nu;
    }
    double *dE = nullptr, *dnu = nullptr;
    int* dbad = nullptr;
    int64_t dummy = 0;
    TRYC(alloc_copy(&dE, E.data(), E.size(), s, &dummy), "material E");
    TRYC(alloc_copy(&dnu, nu.data(), nu.size(), s, &dummy), "material nu");
    TRYC(cudaMalloc(&dbad, sizeof(int)), "flag");
    TRYC(cudaMemsetAsync(dbad, 0, sizeof(int), s), "flag");
    const unsigned grid = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((m->n_elems + 255) / 256, 4096)));
    fill_props_kernel<<<grid, 256, 0, s>>>(p->elem_mat, dE, dnu, m->n_materials, m->n_elems,
                                           m->young ? nullptr : p->young, m->poisson ? nullptr : p->poisson, dbad);
    TRYC(cudaGetLastError(), "material properties");
    int bad = 0;
    TRYC(cudaMemcpyAsync(&bad, dbad, sizeof(int), cudaMemcpyDeviceToHost, s), "flag");
    TRYC(cudaStreamSynchronize(s), "material properties");
    cudaFree(dE);
    cudaFree(dnu);
    cudaFree(dbad);
    if (bad) return fail(set_err(CXG_ERR_INVALID_ARGUMENT, "elem_mat index outside [0, n_materials)"));
  }
  TRYC(cudaMalloc(&p->status, sizeof(DevStatus)), "status");
  {
    DevStatus z{0, 0, ~0ull};
    TRYC(cudaMemcpyAsync(p->status, &z, sizeof z, cudaMemcpyHostToDevice, s), "status");
  }
  const char* msg = nullptr;
  rc = build_pattern(m->elem_type, m->n_nodes, m->n_elems, p->conn, p->dof_eq, d->n_free, &p->pat, &msg, s);
  if (rc) return fail(set_err(rc, std::string("pattern: ") + (msg ? msg : "")));
  p->device_bytes += p->pat.device_bytes;
  TRYC(cudaStreamSynchronize(s), "plan build");
#undef TRYC
  cudaStreamDestroy(s);
  *out = p;
  return CXG_OK;
}

int cxg_plan_create_mpc(const cxg_mesh_desc* m, const cxg_dofmap_desc* d, const cxg_mpc_desc* mpc, int32_t precision,
                        cxg_plan** out) {
  if (!m || !d || !mpc || !out) return set_err(CXG_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (mpc->n_slaves < 0) return set_err(CXG_ERR_INVALID_ARGUMENT, "negative slave count");
  if (mpc->n_slaves == 0) return cxg_plan_create(m, d, precision, out);
  if (m->n_nodes <= 0 || !d->dof_eq || !d->prescribed || d->n_free < 0 || !mpc->slave_dof || !mpc->term_ptr)
    return set_err(CXG_ERR_INVALID_ARGUMENT, "bad DOF map or constraint description");
  const int64_t ndof = 3 * m->n_nodes, ns = mpc->n_slaves;
  // host copies (the arrays may be host or device memory)
  std::vector<int32_t> deq(static_cast<size_t>(ndof));
  std::vector<double> pre(static_cast<size_t>(ndof));
  std::vector<int64_t> sdof(static_cast<size_t>(ns)), tptr(static_cast<size_t>(ns) + 1);
  std::vector<double> cst(static_cast<size_t>(ns), 0.0);
  CHECK_CUDA(cudaMemcpy(deq.data(), d->dof_eq, 4 * ndof, cudaMemcpyDefault), "dof_eq");
  CHECK_CUDA(cudaMemcpy(pre.data(), d->prescribed, 8 * ndof, cudaMemcpyDefault), "prescribed");
  CHECK_CUDA(cudaMemcpy(sdof.data(), mpc->slave_dof, 8 * ns, cudaMemcpyDefault), "slave_dof");
  CHECK_CUDA(cudaMemcpy(tptr.data(), mpc->term_ptr, 8 * (ns + 1), cudaMemcpyDefault), "term_ptr");
  if (mpc->constant) CHECK_CUDA(cudaMemcpy(cst.data(), mpc->constant, 8 * ns, cudaMemcpyDefault), "constant");
  const int64_t nt = tptr[static_cast<size_t>(ns)];
  if (tptr[0] != 0 || nt < 0 || (nt > 0 && (!mpc->term_eq || !mpc->term_coeff)))
    return set_err(CXG_ERR_INVALID_ARGUMENT, "term_ptr must start at 0 and the term arrays be given");
  std::vector<int32_t> teq(static_cast<size_t>(nt));
  std::vector<double> tco(static_cast<size_t>(nt));
  if (nt > 0) {
    CHECK_CUDA(cudaMemcpy(teq.data(), mpc->term_eq, 4 * nt, cudaMemcpyDefault), "term_eq");
    CHECK_CUDA(cudaMemcpy(tco.data(), mpc->term_coeff, 8 * nt, cudaMemcpyDefault), "term_coeff");
  }
  for (int64_t k = 0; k < ns; ++k) {
    const int64_t g = sdof[static_cast<size_t>(k)];
    if (g < 0 || g >= ndof || (k > 0 && g <= sdof[static_cast<size_t>(k) - 1]) || deq[static_cast<size_t>(g)] >= 0)
      return set_err(CXG_ERR_INVALID_ARGUMENT, "slave DOFs must be ascending, in range and not free");
    if (tptr[static_cast<size_t>(k) + 1] < tptr[static_cast<size_t>(k)])
      return set_err(CXG_ERR_INVALID_ARGUMENT, "term_ptr must not decrease");
  }
  for (int32_t e : teq)
    if (e < 0 || e >= d->n_free) return set_err(CXG_ERR_INVALID_ARGUMENT, "constraint term outside the free equations");
  // extended numbering: free DOFs and slaves in ascending global DOF order
  std::vector<int32_t> xeq(static_cast<size_t>(ndof), -1), ext_map;
  std::vector<double> cx;
  bool any_c = false;
  int32_t nx = 0;
  size_t si = 0;
  for (int64_t g = 0; g < ndof; ++g) {
    if (si < sdof.size() && sdof[si] == g) {
      xeq[static_cast<size_t>(g)] = nx++;
      ext_map.push_back(-1 - static_cast<int32_t>(si));
      cx.push_back(cst[si]);
      any_c = any_c || cst[si] != 0.0;
      pre[static_cast<size_t>(g)] = 0.0;
      ++si;
    } else if (deq[static_cast<size_t>(g)] >= 0) {
      xeq[static_cast<size_t>(g)] = nx++;
      ext_map.push_back(deq[static_cast<size_t>(g)]);
      cx.push_back(0.0);
    }
  }
  const cxg_dofmap_desc xd{xeq.data(), pre.data(), nx};
  cxg_plan* p = nullptr;
  int rc = cxg_plan_create(m, &xd, precision, &p);
  if (rc) return rc;
  MpcPlan& mp = p->mpc;
  auto up = [&](void** dst, const void* src, size_t bytes) {
    cudaError_t e = cudaMalloc(dst, std::max<size_t>(bytes, 16));
    if (e == cudaSuccess && bytes) e = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
    return e;
  };
  cudaError_t e = up(reinterpret_cast<void**>(&mp.ext_map), ext_map.data(), 4 * ext_map.size());
  if (e == cudaSuccess) e = up(reinterpret_cast<void**>(&mp.term_ptr), tptr.data(), 8 * tptr.size());
  if (e == cudaSuccess) e = up(reinterpret_cast<void**>(&mp.term_eq), teq.data(), 4 * teq.size());
  if (e == cudaSuccess) e = up(reinterpret_cast<void**>(&mp.term_coeff), tco.data(), 8 * tco.size());
  if (e == cudaSuccess && any_c) e = up(reinterpret_cast<void**>(&mp.c_x), cx.data(), 8 * cx.size());
  if (e == cudaSuccess && any_c) e = cudaMalloc(&mp.kc_x, 8 * static_cast<size_t>(std::max(nx, 1)));
  if (e == cudaSuccess) e = cudaMalloc(&mp.vals_x, 8 * static_cast<size_t>(std::max<int64_t>(p->pat.nnz, 1)));
  if (e == cudaSuccess) e = cudaMalloc(&mp.rhs_x, 8 * static_cast<size_t>(std::max(nx, 1)));
  if (e == cudaSuccess) e = cudaMalloc(&mp.tmp_x, 8 * static_cast<size_t>(std::max(nx, 1)));
  cudaStream_t s = nullptr;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e == cudaSuccess)
    e = build_mpc_reduce(p->pat.row_ptr, p->pat.col_idx, nx, p->pat.nnz, mp.ext_map, mp.term_ptr, mp.term_eq,
                         mp.term_coeff, d->n_free, &mp.lists, s);
  if (s) cudaStreamDestroy(s);
  if (e != cudaSuccess) {
    cxg_plan_destroy(p);
    return cuda_err(e, "constraint reduction");
  }
  mp.on = true;
  mp.n_free = d->n_free;
  *out = p;
  return CXG_OK;
}

namespace thermal {
void release(cxg_plan* p);
}

int cxg_plan_destroy(cxg_plan* p) {
  if (!p) return CXG_OK;
  if (p->last_stream) cudaStreamSynchronize(p->last_stream);
  thermal::release(p);
  cudaFree(p->film_mem);
  void* bufs[] = {p->coords, p->conn, p->young, p->poisson, p->elem_mat, p->mats, p->dof_eq, p->prescribed,
                  p->pat.row_ptr, p->pat.col_idx, p->pat.node_base, p->pat.node_rowlen, p->pat.node_mask,
                  p->pat.node_eq0, p->pat.slot, p->pat.adj_len, p->pat.bnd_ptr, p->pat.bnd_node, p->pat.inc_ptr, p->pat.inc_code, p->state[0], p->state[1],
                  p->status, p->edata, p->fdata};
  for (void* b : bufs) cudaFree(b);
  for (auto& row : p->sched)
    for (WinSched& w : row) cudaFree(w.node_order);
  for (void* b : {static_cast<void*>(p->refpat.row_ptr), static_cast<void*>(p->refpat.col_idx),
                  static_cast<void*>(p->refpat.src), static_cast<void*>(p->refpat.topo_vals)})
    cudaFree(b);
  const MpcPlan& mp = p->mpc;
  for (void* b : {static_cast<void*>(mp.lists.row_ptr), static_cast<void*>(mp.lists.col_idx),
                  static_cast<void*>(mp.lists.tgt_ptr), static_cast<void*>(mp.lists.src), static_cast<void*>(mp.lists.w),
                  static_cast<void*>(mp.lists.rhs_ptr), static_cast<void*>(mp.lists.rhs_src),
                  static_cast<void*>(mp.lists.rhs_w), static_cast<void*>(mp.ext_map), static_cast<void*>(mp.term_ptr),
                  static_cast<void*>(mp.term_eq), static_cast<void*>(mp.term_coeff), static_cast<void*>(mp.c_x),
                  static_cast<void*>(mp.vals_x), static_cast<void*>(mp.rhs_x), static_cast<void*>(mp.tmp_x),
                  static_cast<void*>(mp.kc_x)})
    cudaFree(b);
  for (void* b : p->stage) cudaFree(b);
  delete p;
  return CXG_OK;
}

int cxg_plan_get_info(const cxg_plan* p, cxg_plan_info* info) {
  if (!p || !info) return set_err(CXG_ERR_INVALID_ARGUMENT, "null argument");
  info->n_nodes = p->n_nodes;
  info->n_elems = p->n_elems;
  info->elem_type = p->type;
  info->n_free = active_n_free(p);
  info->nnz = active_nnz(p);
  info->n_gauss_points = p->n_gauss;
  info->precision = p->precision;
  info->device = p->device;
  info->device_bytes = p->device_bytes;
  return CXG_OK;
}

int cxg_plan_set_precision(cxg_plan* p, int32_t precision) {
  if (!p || (precision != CXG_FP64 && precision != CXG_MIXED))
    return set_err(CXG_ERR_INVALID_ARGUMENT, "bad precision");
  p->precision = precision;
  return CXG_OK;
}

int cxg_plan_get_pattern(const cxg_plan* p, int64_t* row_ptr, int32_t* col_idx) {
  if (!p) return set_err(CXG_ERR_INVALID_ARGUMENT, "null plan");
  if (row_ptr)
    CHECK_CUDA(cudaMemcpy(row_ptr, active_row_ptr(p), sizeof(int64_t) * (static_cast<size_t>(active_n_free(p)) + 1),
                          cudaMemcpyDefault), "row_ptr copy");
  if (col_idx)
    CHECK_CUDA(cudaMemcpy(col_idx, active_col_idx(p), sizeof(int32_t) * static_cast<size_t>(active_nnz(p)),
                          cudaMemcpyDefault), "col_idx copy");
  return CXG_OK;
}

int cxg_plan_pattern_device(const cxg_plan* p, const int64_t** row_ptr, const int32_t** col_idx) {
  if (!p) return set_err(CXG_ERR_INVALID_ARGUMENT, "null plan");
  if (row_ptr) *row_ptr = active_row_ptr(p);
  if (col_idx) *col_idx = active_col_idx(p);
  return CXG_OK;
}

int cxg_plan_update_coords(cxg_plan* p, const double* coords) {
  if (!p || !coords) return set_err(CXG_ERR_INVALID_ARGUMENT, "null argument");
  if (int rc = reject_refpat(p)) return rc;
  CHECK_CUDA(cudaMemcpy(p->coords, coords, sizeof(double) * 3 * static_cast<size_t>(p->n_nodes), cudaMemcpyDefault),
             "coords update");
  return CXG_OK;
}

int cxg_plan_update_young(cxg_plan* p, const double* young) {
  if (p) {
    if (int rc = reject_refpat(p)) return rc;
  }
  if (!p || !young) return set_err(CXG_ERR_INVALID_ARGUMENT, "null argument");
  CHECK_CUDA(cudaMemcpy(p->young, young, sizeof(double) * static_cast<size_t>(p->n_elems), cudaMemcpyDefault),
             "young update");
  return CXG_OK;
}

int cxg_plan_set_launch_config(cxg_plan* p, int32_t mode, int32_t tile, int32_t p1_blocks_per_sm, int32_t p2_warps) {
  if (!p || (mode != 0 && mode != 1)) return set_err(CXG_ERR_INVALID_ARGUMENT, "bad plan or mode");
  if (tile < 0 || tile > 2 || (tile == 2 && (mode == 1 || p->precision == CXG_FP64)) || p1_blocks_per_sm < 0 ||
      p2_warps < 0 || p2_warps > 8)
    return set_err(CXG_ERR_INVALID_ARGUMENT, "bad launch shape (4x4 tiles: linear pass, mixed precision only)");
  LaunchCfg& c = mode ? p->tcfg[p->precision] : p->cfg[p->precision];
  c.tile = tile;
  c.p1_blocks_per_sm = p1_blocks_per_sm;
  c.p2_warps = p2_warps;
  return CXG_OK;
}

int cxg_plan_set_j2_fp32_return(cxg_plan* p, int32_t enable) {
  if (!p) return set_err(CXG_ERR_INVALID_ARGUMENT, "null plan");
  p->tcfg[CXG_MIXED].j2_fp32 = enable ? 1 : 0;
  return CXG_OK;
}

int cxg_plan_set_ring_bytes(cxg_plan* p, int64_t bytes) {
  if (!p) return set_err(CXG_ERR_INVALID_ARGUMENT, "null plan");
  if (p->last_stream) CHECK_CUDA(cudaStreamSynchronize(p->last_stream), "synchronize");
  p->ring_bytes = bytes;
  for (auto& row : p->sched)
    for (WinSched& w : row) w.built = false;  // rebuilt at the next assembly
  return CXG_OK;
}

int cxg_plan_use_reference_pattern(cxg_plan* p, int32_t enable) {
  if (!p) return set_err(CXG_ERR_INVALID_ARGUMENT, "null plan");
  if (p->thermal) return set_err(CXG_ERR_UNSUPPORTED, "the reference pattern covers the structural linear assembly");
  if (p->mpc.on) return reject_mpc(p);
  if (p->last_stream) CHECK_CUDA(cudaStreamSynchronize(p->last_stream), "synchronize");
  RefPattern& r = p->refpat;
  if (!enable || r.on) {
    if (!enable && r.on) {
      for (void* b : {static_cast<void*>(r.row_ptr), static_cast<void*>(r.col_idx), static_cast<void*>(r.src),
                      static_cast<void*>(r.topo_vals)})
        cudaFree(b);
      p->device_bytes -= static_cast<int64_t>(8 * (p->n_free + 1) + 12 * r.nnz + 8 * p->pat.nnz);
      r = RefPattern{};
    }
    return CXG_OK;
  }
  cudaStream_t s = nullptr;
  CHECK_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
  double *flags = nullptr, *counts = nullptr;
  RefPattern nr;
  cudaError_t e = cudaMalloc(&flags, std::max<size_t>(v2_edata_bytes(p->type, p->n_elems, CXG_FP64), 16));
  if (e == cudaSuccess) e = cudaMalloc(&counts, sizeof(double) * static_cast<size_t>(std::max<int64_t>(p->pat.nnz, 1)));
  ElemArgs a = base_args(p);
  // 1.0 / 0.0 per element-matrix entry: nonzero in the reference's arithmetic or not
  if (e == cudaSuccess) e = launch_refmask(p->type, a, flags, s);
  // the FP64 row gather counts, per CSR entry, the elements contributing a nonzero value
  a.vals = counts;
  a.rhs = nullptr;
  V2Args v = v2_args(p, nullptr, false);
  v.edata = flags;
  LaunchCfg gather_only;
  gather_only.passes = 2;
  if (e == cudaSuccess) e = launch_v2(p->type, MODE_LINEAR, CXG_FP64, a, v, s, gather_only);
  if (e == cudaSuccess)
    e = compact_pattern(p->pat.row_ptr, p->pat.col_idx, p->n_free, p->pat.nnz, counts, &nr.row_ptr, &nr.col_idx,
                        &nr.src, &nr.nnz, s);
  if (e == cudaSuccess)
    e = cudaMalloc(&nr.topo_vals, sizeof(double) * static_cast<size_t>(std::max<int64_t>(p->pat.nnz, 1)));
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(flags);
  cudaFree(counts);
  cudaStreamDestroy(s);
  if (e != cudaSuccess) {
    for (void* b : {static_cast<void*>(nr.row_ptr), static_cast<void*>(nr.col_idx), static_cast<void*>(nr.src),
                    static_cast<void*>(nr.topo_vals)})
      cudaFree(b);
    return cuda_err(e, "reference pattern");
  }
  nr.on = true;
  r = nr;
  p->device_bytes += static_cast<int64_t>(8 * (p->n_free + 1) + 12 * r.nnz + 8 * p->pat.nnz);
  return CXG_OK;
}

int cxg_plan_get_windows(const cxg_plan* p, int32_t mode, int32_t* n_windows, int64_t* ring_elems) {
  if (!p || (mode != 0 && mode != 1) || !n_windows || !ring_elems)
    return set_err(CXG_ERR_INVALID_ARGUMENT, "bad argument");
  const WinSched& w = p->sched[p->precision][mode];
  *n_windows = !w.built ? 0 : (w.win_e.size() < 3 ? 1 : static_cast<int32_t>(w.win_e.size() - 1));
  *ring_elems = w.built ? w.ring : 0;
  return CXG_OK;
}

int cxg_plan_check(cxg_plan* p, int64_t* bad) {
  if (!p) return set_err(CXG_ERR_INVALID_ARGUMENT, "null plan");
  return plan_status(p, bad);
}

namespace thermal {

__global__ void add_into_kernel(int64_t n, double* a, const double* b) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    a[i] += b[i];
}

// thermal_strain_load_vector of the plan into out[3N] (device)
int load_device(cxg_plan* p, double* out, cudaStream_t s) {
  const int n = nodes_of(p->type);
  double* felem = nullptr;
  CHECK_CUDA(cudaMallocAsync(&felem, sizeof(double) * std::max<size_t>(static_cast<size_t>(p->n_elems) * 3 * n, 1), s),
             "thermal load scratch");
  ElemArgs a = base_args(p);
  a.u = nullptr;
  const cudaError_t err = launch_recover(p->type, a, p->pat.inc_ptr, p->pat.inc_code, nullptr, nullptr, felem, nullptr,
                                         nullptr, nullptr, out, true, s);
  cudaFreeAsync(felem, s);
  CHECK_CUDA(err, "thermal load kernels");
  return CXG_OK;
}

void release(cxg_plan* p) {
  for (void* b : {static_cast<void*>(p->th_temp), static_cast<void*>(p->th_applied), static_cast<void*>(p->th_alpha),
                  static_cast<void*>(p->th_tref), static_cast<void*>(p->th_load)})
    cudaFree(b);
  p->th_temp = nullptr;
  p->th_applied = nullptr;
  p->th_alpha = nullptr;
  p->th_tref = nullptr;
  p->th_load = nullptr;
}

}  // namespace thermal

int cxg_plan_set_thermal_strain(cxg_plan* p, const double* node_temp, const uint8_t* node_applied,
                                const double* elem_alpha, const double* elem_tref) {
  if (!p) return set_err(CXG_ERR_INVALID_ARGUMENT, "null plan");
  if (p->last_stream) CHECK_CUDA(cudaStreamSynchronize(p->last_stream), "synchronize");
  thermal::release(p);
  if (!node_temp) return CXG_OK;
  if (!elem_alpha || !elem_tref) return set_err(CXG_ERR_INVALID_ARGUMENT, "elem_alpha and elem_tref are required");
  if (p->thermal) return set_err(CXG_ERR_UNSUPPORTED, "thermal strain applies to displacement plans");
  const size_t N = static_cast<size_t>(std::max<int64_t>(p->n_nodes, 1)), E = static_cast<size_t>(std::max<int64_t>(p->n_elems, 1));
  cudaError_t e = cudaMalloc(&p->th_temp, sizeof(double) * N);
  if (e == cudaSuccess && node_applied) e = cudaMalloc(&p->th_applied, N);
  if (e == cudaSuccess) e = cudaMalloc(&p->th_alpha, sizeof(double) * E);
  if (e == cudaSuccess) e = cudaMalloc(&p->th_tref, sizeof(double) * E);
  if (e == cudaSuccess) e = cudaMalloc(&p->th_load, sizeof(double) * 3 * N);
  const size_t nn = static_cast<size_t>(p->n_nodes), ne = static_cast<size_t>(p->n_elems);
  if (e == cudaSuccess && nn) e = cudaMemcpy(p->th_temp, node_temp, sizeof(double) * nn, cudaMemcpyDefault);
  if (e == cudaSuccess && nn && node_applied) e = cudaMemcpy(p->th_applied, node_applied, nn, cudaMemcpyDefault);
  if (e == cudaSuccess && ne) e = cudaMemcpy(p->th_alpha, elem_alpha, sizeof(double) * ne, cudaMemcpyDefault);
  if (e == cudaSuccess && ne) e = cudaMemcpy(p->th_tref, elem_tref, sizeof(double) * ne, cudaMemcpyDefault);
  if (e != cudaSuccess) {
    thermal::release(p);
    return cuda_err(e, "thermal strain inputs");
  }
  return CXG_OK;
}

int cxg_thermal_strain_load(cxg_plan* p, double* f_th, void* stream) {
  if (!p || !f_th) return set_err(CXG_ERR_INVALID_ARGUMENT, "plan and f_th are required");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  p->last_stream = s;
  const size_t fb = sizeof(double) * 3 * static_cast<size_t>(p->n_nodes);
  if (!p->th_temp) {
    CHECK_CUDA(cudaMemsetAsync(f_th, 0, fb, s), "zero load");  // no thermal strain set
    return CXG_OK;
  }
  void* df = nullptr;
  int rc = staged(p, 2, f_th, fb, false, s, &df);
  if (!rc) rc = thermal::load_device(p, static_cast<double*>(df), s);
  if (!rc) rc = copy_out(f_th, df, fb, s);
  if (rc) return rc;
  if (df != f_th) CHECK_CUDA(cudaStreamSynchronize(s), "synchronize");
  return CXG_OK;
}

int cxg_assemble_linear(cxg_plan* p, double* vals, double* rhs, const double* f_ext, void* stream) {
  return cxg_assemble_linear_ex(p, vals, rhs, f_ext, 0, stream);
}

int cxg_assemble_linear_ex(cxg_plan* p, double* vals, double* rhs, const double* f_ext, int32_t flags,
                           void* stream) {
  if (!p || !vals) return set_err(CXG_ERR_INVALID_ARGUMENT, "plan and vals are required");
  const bool accumulate = (flags & CXG_ACCUMULATE) != 0;
  if (accumulate && (p->refpat.on || p->mpc.on))
    return set_err(CXG_ERR_UNSUPPORTED, "CXG_ACCUMULATE works on the topological pattern only");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  p->last_stream = s;
  const size_t vb = sizeof(double) * static_cast<size_t>(active_nnz(p));
  const size_t rb = sizeof(double) * static_cast<size_t>(active_n_free(p));
  const size_t fb = sizeof(double) * 3 * static_cast<size_t>(p->n_nodes);
  void *dv, *dr, *df = nullptr;
  int rc = staged(p, 0, vals, vb, accumulate, s, &dv);
  if (!rc) rc = staged(p, 1, rhs, rb, accumulate, s, &dr);
  if (!rc && !accumulate) rc = staged(p, 2, f_ext, fb, true, s, &df);
  if (rc) return rc;
  if ((rc = ensure_v2(p, false))) return rc;
  // thermal-strain equivalent load added to the external load (assembly.cpp:251-253)
  if (p->th_temp && !accumulate) {
    if ((rc = thermal::load_device(p, p->th_load, s))) return rc;
    if (df) {
      const int64_t n3 = 3 * p->n_nodes;
      thermal::add_into_kernel<<<static_cast<unsigned>(std::min<int64_t>((n3 + 255) / 256, 148 * 16) + 1), 256, 0, s>>>(
          n3, p->th_load, static_cast<const double*>(df));
      CHECK_CUDA(cudaGetLastError(), "thermal load");
    }
    df = p->th_load;
  }
  ElemArgs a = base_args(p);
  // with the reference's pattern, the assembly runs on the topological pattern and the
  // kept entries are gathered into the caller's values
  a.vals = p->mpc.on ? p->mpc.vals_x : p->refpat.on ? p->refpat.topo_vals : static_cast<double*>(dv);
  a.rhs = p->mpc.on ? p->mpc.rhs_x : static_cast<double*>(dr);
  V2Args v = v2_args(p, static_cast<const double*>(df), accumulate);
  apply_windows(p, false, v);
  CHECK_CUDA(launch_v2(p->type, MODE_LINEAR, p->precision, a, v, s, p->cfg[p->precision]), "assembly kernels");
  if (p->refpat.on)
    CHECK_CUDA(gather_values(p->refpat.src, p->refpat.topo_vals, p->refpat.nnz, static_cast<double*>(dv), s),
               "reference pattern");
  if (p->mpc.on) CHECK_CUDA(mpc_reduce(p, static_cast<double*>(dv), static_cast<double*>(dr), s), "constraint reduction");
  if ((rc = copy_out(vals, dv, vb, s))) return rc;
  if ((rc = copy_out(rhs, dr, rb, s))) return rc;
  if (dv != vals || (rhs && dr != rhs)) CHECK_CUDA(cudaStreamSynchronize(s), "synchronize");
  return CXG_OK;
}

int cxg_assemble_tangent(cxg_plan* p, const double* u, double* vals, double* f_int, double* rhs,
                         const double* f_ext, void* stream) {
  if (!p || !u || !vals) return set_err(CXG_ERR_INVALID_ARGUMENT, "plan, u and vals are required");
  if (p->refpat.on) return reject_refpat(p);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  p->last_stream = s;
  int rc = ensure_state(p, s);
  if (rc) return rc;
  const size_t vb = sizeof(double) * static_cast<size_t>(active_nnz(p));
  const size_t rb = sizeof(double) * static_cast<size_t>(active_n_free(p));
  const size_t fb = sizeof(double) * 3 * static_cast<size_t>(p->n_nodes);
  void *dv, *dr, *df, *du, *dfi;
  rc = staged(p, 0, vals, vb, false, s, &dv);
  if (!rc) rc = staged(p, 1, rhs, rb, false, s, &dr);
  if (!rc) rc = staged(p, 2, f_ext, fb, true, s, &df);
  if (!rc) rc = staged(p, 3, u, fb, true, s, &du);
  if (!rc) rc = staged(p, 4, f_int, fb, false, s, &dfi);
  if (rc) return rc;
  if ((rc = ensure_v2(p, true))) return rc;
  ElemArgs a = base_args(p);
  a.vals = p->mpc.on ? p->mpc.vals_x : static_cast<double*>(dv);
  a.rhs = p->mpc.on ? p->mpc.rhs_x : static_cast<double*>(dr);
  a.f_int = static_cast<double*>(dfi);
  a.u = static_cast<const double*>(du);
  a.state_c = p->state[0];
  a.state_t = p->state[1];
  a.state_comps = state_comps(p);
  V2Args v = v2_args(p, static_cast<const double*>(df), false);
  apply_windows(p, true, v);
  CHECK_CUDA(launch_v2(p->type, MODE_TANGENT, p->precision, a, v, s, p->tcfg[p->precision]), "assembly kernels");
  if (p->mpc.on) CHECK_CUDA(mpc_reduce(p, static_cast<double*>(dv), static_cast<double*>(dr), s), "constraint reduction");
  if ((rc = copy_out(vals, dv, vb, s))) return rc;
  if ((rc = copy_out(rhs, dr, rb, s))) return rc;
  if ((rc = copy_out(f_int, dfi, fb, s))) return rc;
  if (dv != vals || (rhs && dr != rhs) || (f_int && dfi != f_int)) CHECK_CUDA(cudaStreamSynchronize(s), "sync");
  return CXG_OK;
}

namespace {

// The scalar-block operators (mass, geometric stiffness) on the FP64 element buffer
// and the FP64 row gather; the rhs side effect of prescribed columns is discarded, as
// in the reference (src/fem/assembly.cpp:286-288, 320-322).
int assemble_scalar(cxg_plan* p, int kind, const double* input, size_t input_bytes, double* vals, void* stream) {
  if (int rc0 = reject_refpat(p)) return rc0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  p->last_stream = s;
  const size_t vb = sizeof(double) * static_cast<size_t>(p->pat.nnz);
  void *dv, *din = nullptr;
  int rc = staged(p, 0, vals, vb, false, s, &dv);
  if (!rc && input) rc = staged(p, 5, input, input_bytes, true, s, &din);
  if (rc) return rc;
  const size_t need = v2_edata_bytes(p->type, p->n_elems, CXG_FP64);
  if (p->edata_bytes < need) {
    cudaFree(p->edata);
    p->edata = nullptr;
    p->device_bytes -= static_cast<int64_t>(p->edata_bytes);
    p->edata_bytes = 0;
    CHECK_CUDA(cudaMalloc(&p->edata, std::max<size_t>(need, 16)), "element buffer");
    p->edata_bytes = need;
    p->device_bytes += static_cast<int64_t>(need);
  }
  ElemArgs a = base_args(p);
  a.vals = static_cast<double*>(dv);
  a.rhs = nullptr;
  const V2Args v = v2_args(p, nullptr, false);
  const double* d = static_cast<const double*>(din);
  CHECK_CUDA(launch_scalar_pass(p->type, kind, a, v, kind == 3 ? nullptr : d, kind == 3 ? d : nullptr, s),
             "element pass");
  LaunchCfg gather_only;
  gather_only.passes = 2;
  CHECK_CUDA(launch_v2(p->type, MODE_LINEAR, CXG_FP64, a, v, s, gather_only), "row gather");
  if ((rc = copy_out(vals, dv, vb, s))) return rc;
  if (dv != vals) CHECK_CUDA(cudaStreamSynchronize(s), "synchronize");
  return CXG_OK;
}

}  // namespace

int cxg_assemble_mass(cxg_plan* p, const double* density, int32_t lumped, double* vals, void* stream) {
  if (!p || !density || !vals) return set_err(CXG_ERR_INVALID_ARGUMENT, "plan, density and vals are required");
  return assemble_scalar(p, lumped ? 2 : 1, density, sizeof(double) * static_cast<size_t>(p->n_elems), vals, stream);
}

int cxg_assemble_geometric(cxg_plan* p, const double* gp_stress, double* vals, void* stream) {
  if (!p || !vals) return set_err(CXG_ERR_INVALID_ARGUMENT, "plan and vals are required");
  return assemble_scalar(p, 3, gp_stress, sizeof(double) * 6 * static_cast<size_t>(p->n_gauss), vals, stream);
}

int cxg_thermal_plan_create(const cxg_mesh_desc* m, const int32_t* t_dof_eq, const double* t_prescribed,
                            int32_t n_free, cxg_plan** out) {
  if (!m || !t_dof_eq || !t_prescribed || !out || m->n_nodes <= 0)
    return set_err(CXG_ERR_INVALID_ARGUMENT, "mesh, temperature DOF map and output are required");
  const size_t N = static_cast<size_t>(m->n_nodes);
  std::vector<int32_t> teq(N);
  std::vector<double> tpre(N);
  CHECK_CUDA(cudaMemcpy(teq.data(), t_dof_eq, 4 * N, cudaMemcpyDefault), "temperature DOF map");
  CHECK_CUDA(cudaMemcpy(tpre.data(), t_prescribed, 8 * N, cudaMemcpyDefault), "prescribed temperatures");
  // the temperature is component 0 of every node; components 1 and 2 are fixed at 0
  std::vector<int32_t> deq(3 * N, -1);
  std::vector<double> pre(3 * N, 0.0);
  for (size_t a = 0; a < N; ++a) {
    deq[3 * a] = teq[a];
    pre[3 * a] = teq[a] < 0 ? tpre[a] : 0.0;
  }
  cxg_dofmap_desc d{deq.data(), pre.data(), n_free};
  int rc = cxg_plan_create(m, &d, CXG_FP64, out);
  if (rc) return rc;
  (*out)->thermal = true;
  return CXG_OK;
}

int cxg_thermal_plan_set_films(cxg_plan* p, int64_t n_films, const int64_t* elem, const int32_t* face,
                               const double* h, const double* sink) {
  if (!p || n_films < 0 || (n_films > 0 && (!elem || !face || !h || !sink)))
    return set_err(CXG_ERR_INVALID_ARGUMENT, "bad argument");
  if (!p->thermal) return set_err(CXG_ERR_INVALID_ARGUMENT, "films need a plan from cxg_thermal_plan_create");
  if (n_films >= (int64_t{1} << 28)) return set_err(CXG_ERR_UNSUPPORTED, "too many films");
  if (p->last_stream) CHECK_CUDA(cudaStreamSynchronize(p->last_stream), "synchronize");
  cudaFree(p->film_mem);
  p->film_mem = nullptr;
  p->films = FilmArgs{};
  if (n_films == 0) return CXG_OK;
  // host arrays (staged copies when the caller passed device pointers)
  std::vector<int64_t> fe(static_cast<size_t>(n_films));
  std::vector<int32_t> ff(static_cast<size_t>(n_films));
  std::vector<double> fh(static_cast<size_t>(n_films)), fs(static_cast<size_t>(n_films));
  CHECK_CUDA(cudaMemcpy(fe.data(), elem, sizeof(int64_t) * fe.size(), cudaMemcpyDefault), "film elements");
  CHECK_CUDA(cudaMemcpy(ff.data(), face, sizeof(int32_t) * ff.size(), cudaMemcpyDefault), "film faces");
  CHECK_CUDA(cudaMemcpy(fh.data(), h, sizeof(double) * fh.size(), cudaMemcpyDefault), "film coefficients");
  CHECK_CUDA(cudaMemcpy(fs.data(), sink, sizeof(double) * fs.size(), cudaMemcpyDefault), "film sinks");
  std::vector<int32_t> conn(static_cast<size_t>(p->n_elems) * nodes_of(p->type));
  CHECK_CUDA(cudaMemcpy(conn.data(), p->conn, sizeof(int32_t) * conn.size(), cudaMemcpyDeviceToHost), "connectivity");
  const int n = nodes_of(p->type);
  // films grouped by element, film order kept within each element
  std::vector<int32_t> order(static_cast<size_t>(n_films));
  for (int32_t i = 0; i < n_films; ++i) order[static_cast<size_t>(i)] = i;
  for (int64_t i = 0; i < n_films; ++i) {
    int fn[8], nf = 0;
    bool quad = false;
    if (fe[static_cast<size_t>(i)] < 0 || fe[static_cast<size_t>(i)] >= p->n_elems)
      return set_err(CXG_ERR_INVALID_ARGUMENT, "*FILM references unknown element (film " + std::to_string(i) + ")");
    if (!face_nodes_of(p->type, ff[static_cast<size_t>(i)], fn, &nf, &quad))
      return set_err(CXG_ERR_INVALID_ARGUMENT, "face number out of range for this element type (film " +
                                                   std::to_string(i) + ")");
  }
  std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return fe[x] < fe[y]; });
  std::vector<int64_t> felem;
  std::vector<int32_t> fptr(1, 0);
  for (size_t k = 0; k < order.size(); ++k) {
    if (k == 0 || fe[static_cast<size_t>(order[k])] != fe[static_cast<size_t>(order[k - 1])]) {
      if (k) fptr.push_back(static_cast<int32_t>(k));
      felem.push_back(fe[static_cast<size_t>(order[k])]);
    }
  }
  fptr.push_back(static_cast<int32_t>(order.size()));
  // per face node, its (film, local index) entries in film order
  std::vector<std::pair<int64_t, int32_t>> inc;
  for (int32_t i = 0; i < n_films; ++i) {
    int fn[8], nf = 0;
    bool quad = false;
    face_nodes_of(p->type, ff[static_cast<size_t>(i)], fn, &nf, &quad);
    for (int j = 0; j < nf; ++j)
      inc.emplace_back(conn[static_cast<size_t>(fe[static_cast<size_t>(i)]) * n + fn[j]], i * 8 + j);
  }
  std::stable_sort(inc.begin(), inc.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
  std::vector<int64_t> fnode;
  std::vector<int32_t> fnptr(1, 0), fnlist;
  for (size_t k = 0; k < inc.size(); ++k) {
    if (k == 0 || inc[k].first != inc[k - 1].first) {
      if (k) fnptr.push_back(static_cast<int32_t>(k));
      fnode.push_back(inc[k].first);
    }
    fnlist.push_back(inc[k].second);
  }
  fnptr.push_back(static_cast<int32_t>(inc.size()));
  // one device block: int64 arrays, doubles, then int32 arrays
  const size_t nF = static_cast<size_t>(n_films);
  const size_t bytes = 8 * (felem.size() + fnode.size() + 3 * nF + 8 * nF) +
                       4 * (fptr.size() + order.size() + nF + fnptr.size() + fnlist.size()) + 64;
  char* mem = nullptr;
  CHECK_CUDA(cudaMalloc(&mem, bytes), "film arrays");
  p->film_mem = mem;
  size_t off = 0;
  auto put = [&](const void* src, size_t b) {
    char* dst = mem + off;
    off += (b + 7) / 8 * 8;
    return cudaMemcpy(dst, src, b, cudaMemcpyHostToDevice) == cudaSuccess ? dst : nullptr;
  };
  FilmArgs& F = p->films;
  F.n_films = n_films;
  F.n_felem = static_cast<int64_t>(felem.size());
  F.n_fnode = static_cast<int64_t>(fnode.size());
  F.felem = reinterpret_cast<const int64_t*>(put(felem.data(), 8 * felem.size()));
  F.fnode = reinterpret_cast<const int64_t*>(put(fnode.data(), 8 * fnode.size()));
  F.h = reinterpret_cast<const double*>(put(fh.data(), 8 * nF));
  F.sink = reinterpret_cast<const double*>(put(fs.data(), 8 * nF));
  F.load = reinterpret_cast<double*>(mem + off);
  off += 8 * 8 * nF;
  F.fptr = reinterpret_cast<const int32_t*>(put(fptr.data(), 4 * fptr.size()));
  F.flist = reinterpret_cast<const int32_t*>(put(order.data(), 4 * order.size()));
  F.face = reinterpret_cast<const int32_t*>(put(ff.data(), 4 * nF));
  F.fnptr = reinterpret_cast<const int32_t*>(put(fnptr.data(), 4 * fnptr.size()));
  F.fnlist = reinterpret_cast<const int32_t*>(put(fnlist.data(), 4 * fnlist.size()));
  if (off > bytes || !F.felem || !F.fnode || !F.h || !F.sink || !F.fptr || !F.flist || !F.face || !F.fnptr ||
      !F.fnlist) {
    cudaFree(p->film_mem);
    p->film_mem = nullptr;
    p->films = FilmArgs{};
    return set_err(CXG_ERR_CUDA, "film arrays upload");
  }
  return CXG_OK;
}

int cxg_assemble_conduction(cxg_plan* p, const double* conductivity, const double* flux, double* vals, double* rhs,
                            void* stream) {
  if (!p || !conductivity || !vals) return set_err(CXG_ERR_INVALID_ARGUMENT, "plan, conductivity and vals are required");
  if (!p->thermal) return set_err(CXG_ERR_INVALID_ARGUMENT, "conduction needs a plan from cxg_thermal_plan_create");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  p->last_stream = s;
  const size_t vb = sizeof(double) * static_cast<size_t>(p->pat.nnz);
  const size_t rb = sizeof(double) * static_cast<size_t>(p->n_free);
  const size_t N = static_cast<size_t>(p->n_nodes);
  void *dv, *dr, *dk, *df = nullptr;
  int rc = staged(p, 0, vals, vb, false, s, &dv);
  if (!rc) rc = staged(p, 1, rhs, rb, false, s, &dr);
  if (!rc) rc = staged(p, 5, conductivity, sizeof(double) * static_cast<size_t>(p->n_elems), true, s, &dk);
  if (rc) return rc;
  if (flux || p->films.n_films > 0) {
    // nodal flux (and film loads) into component 0 of a 3N load vector (plan staging slot 2)
    if (p->stage_bytes[2] < 24 * N) {
      cudaFree(p->stage[2]);
      p->stage[2] = nullptr;
      p->stage_bytes[2] = 0;
      CHECK_CUDA(cudaMalloc(&p->stage[2], 24 * N), "flux staging");
      p->stage_bytes[2] = 24 * N;
    }
    df = p->stage[2];
    CHECK_CUDA(cudaMemsetAsync(df, 0, 24 * N, s), "flux staging");
    if (flux) CHECK_CUDA(cudaMemcpy2DAsync(df, 24, flux, 8, 8, N, cudaMemcpyDefault, s), "flux upload");
  }
  const size_t need = v2_edata_bytes(p->type, p->n_elems, CXG_FP64);
  if (p->edata_bytes < need) {
    cudaFree(p->edata);
    p->edata = nullptr;
    p->device_bytes -= static_cast<int64_t>(p->edata_bytes);
    p->edata_bytes = 0;
    CHECK_CUDA(cudaMalloc(&p->edata, std::max<size_t>(need, 16)), "element buffer");
    p->edata_bytes = need;
    p->device_bytes += static_cast<int64_t>(need);
  }
  ElemArgs a = base_args(p);
  a.vals = static_cast<double*>(dv);
  a.rhs = static_cast<double*>(dr);
  const V2Args v = v2_args(p, static_cast<const double*>(df), false);
  CHECK_CUDA(launch_scalar_pass(p->type, 4, a, v, static_cast<const double*>(dk), nullptr, s), "element pass");
  if (p->films.n_films > 0)
    CHECK_CUDA(launch_films(p->type, a, p->films, static_cast<double*>(p->edata), static_cast<double*>(df), s),
               "film faces");
  LaunchCfg gather_only;
  gather_only.passes = 2;
  CHECK_CUDA(launch_v2(p->type, MODE_LINEAR, CXG_FP64, a, v, s, gather_only), "row gather");
  if ((rc = copy_out(vals, dv, vb, s))) return rc;
  if ((rc = copy_out(rhs, dr, rb, s))) return rc;
  if (dv != vals || (rhs && dr != rhs)) CHECK_CUDA(cudaStreamSynchronize(s), "synchronize");
  return CXG_OK;
}

int cxg_recover_gauss_stress(cxg_plan* p, const double* u, double* gp_stress, void* stream) {
  if (!p || !u || !gp_stress) return set_err(CXG_ERR_INVALID_ARGUMENT, "plan, u and gp_stress are required");
  if (p->has_plastic) return set_err(CXG_ERR_UNSUPPORTED, "Gauss-point stress recovery is for linear elasticity");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  p->last_stream = s;
  const size_t ub = sizeof(double) * 3 * static_cast<size_t>(p->n_nodes);
  const size_t gb = sizeof(double) * 6 * static_cast<size_t>(p->n_gauss);
  void *du, *dg;
  int rc = staged(p, 3, u, ub, true, s, &du);
  if (!rc) rc = staged(p, 0, gp_stress, gb, false, s, &dg);
  if (rc) return rc;
  ElemArgs a = base_args(p);
  a.u = static_cast<const double*>(du);
  CHECK_CUDA(launch_recover(p->type, a, nullptr, nullptr, static_cast<double*>(dg), nullptr, nullptr, nullptr, nullptr,
                            nullptr, nullptr, false, s),
             "recovery kernel");
  if ((rc = copy_out(gp_stress, dg, gb, s))) return rc;
  if (dg != gp_stress) CHECK_CUDA(cudaStreamSynchronize(s), "synchronize");
  return CXG_OK;
}

int cxg_recover_fields(cxg_plan* p, const double* u, const double* f_ext, double* strain, double* stress,
                       double* reaction, void* stream) {
  if (!p || !u) return set_err(CXG_ERR_INVALID_ARGUMENT, "plan and u are required");
  if (p->has_plastic) return set_err(CXG_ERR_UNSUPPORTED, "field recovery here is for linear elasticity");
  if (p->type == C3D8R)
    return set_err(CXG_ERR_UNSUPPORTED, "field recovery of the hourglass-stabilised C3D8R is not provided");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  p->last_stream = s;
  const size_t ub = sizeof(double) * 3 * static_cast<size_t>(p->n_nodes);
  const size_t sb = 2 * ub;
  void *du, *df = nullptr, *dst = nullptr, *dss = nullptr, *drf = nullptr;
  int rc = staged(p, 3, u, ub, true, s, &du);
  if (!rc) rc = staged(p, 2, f_ext, ub, true, s, &df);
  if (!rc) rc = staged(p, 1, strain, sb, false, s, &dst);
  if (!rc) rc = staged(p, 4, stress, sb, false, s, &dss);
  if (!rc) rc = staged(p, 5, reaction, ub, false, s, &drf);
  if (rc) return rc;
  const int n = nodes_of(p->type);
  double* scratch = nullptr;
  const int sets = p->type == C3D10 ? n : 1;  // value sets per element, see cxg_recover.cu
  const size_t scratch_doubles = static_cast<size_t>(p->n_elems) * (12 * sets + 3 * n);
  CHECK_CUDA(cudaMallocAsync(&scratch, sizeof(double) * std::max<size_t>(scratch_doubles, 1), s), "recovery scratch");
  ElemArgs a = base_args(p);
  a.u = static_cast<const double*>(du);
  const cudaError_t err = launch_recover(p->type, a, p->pat.inc_ptr, p->pat.inc_code, nullptr, scratch,
                                         scratch + 12 * static_cast<size_t>(sets) * static_cast<size_t>(p->n_elems),
                                         static_cast<const double*>(df), static_cast<double*>(dst),
                                         static_cast<double*>(dss), static_cast<double*>(drf), false, s);
  cudaFreeAsync(scratch, s);
  CHECK_CUDA(err, "recovery kernels");
  if ((rc = copy_out(strain, dst, sb, s))) return rc;
  if ((rc = copy_out(stress, dss, sb, s))) return rc;
  if ((rc = copy_out(reaction, drf, ub, s))) return rc;
  if ((strain && dst != strain) || (stress && dss != stress) || (reaction && drf != reaction))
    CHECK_CUDA(cudaStreamSynchronize(s), "synchronize");
  return CXG_OK;
}

int cxg_state_get(const cxg_plan* cp, int32_t slot, double* out) {
  auto* p = const_cast<cxg_plan*>(cp);
  if (!p || !out || (slot != 0 && slot != 1)) return set_err(CXG_ERR_INVALID_ARGUMENT, "bad argument");
  const size_t bytes = sizeof(double) * kStateDoubles * static_cast<size_t>(p->n_gauss);
  int rc = ensure_state(p, nullptr);
  if (rc) return rc;
  CHECK_CUDA(cudaStreamSynchronize(p->last_stream), "synchronize");
  void* tmp = nullptr;
  CHECK_CUDA(cudaMalloc(&tmp, std::max<size_t>(bytes, 8)), "state staging");
  cudaError_t e = launch_state_transpose(p->state[slot], static_cast<double*>(tmp), p->n_gauss, false, nullptr);
  if (e == cudaSuccess) e = cudaMemcpy(out, tmp, bytes, cudaMemcpyDefault);
  cudaFree(tmp);
  CHECK_CUDA(e, "state read");
  return CXG_OK;
}

int cxg_state_set(cxg_plan* p, int32_t slot, const double* in) {
  if (!p || !in || (slot != 0 && slot != 1)) return set_err(CXG_ERR_INVALID_ARGUMENT, "bad argument");
  const size_t bytes = sizeof(double) * kStateDoubles * static_cast<size_t>(p->n_gauss);
  int rc = ensure_state(p, nullptr);
  if (rc) return rc;
  CHECK_CUDA(cudaStreamSynchronize(p->last_stream), "synchronize");
  void* tmp = nullptr;
  CHECK_CUDA(cudaMalloc(&tmp, std::max<size_t>(bytes, 8)), "state staging");
  cudaError_t e = cudaMemcpy(tmp, in, bytes, cudaMemcpyDefault);
  if (e == cudaSuccess) e = launch_state_transpose(static_cast<double*>(tmp), p->state[slot], p->n_gauss, true, nullptr);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaFree(tmp);
  CHECK_CUDA(e, "state write");
  p->back_stress_zero = false;  // the caller may have set a back stress
  return CXG_OK;
}

int cxg_state_commit(cxg_plan* p, void* stream) {
  if (!p) return set_err(CXG_ERR_INVALID_ARGUMENT, "null plan");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = ensure_state(p, s);
  if (rc) return rc;
  p->last_stream = s;
  // SoA layout: the first state_comps components are the leading state_comps*G doubles
  CHECK_CUDA(cudaMemcpyAsync(p->state[0], p->state[1], sizeof(double) * state_comps(p) * static_cast<size_t>(p->n_gauss),
                             cudaMemcpyDeviceToDevice, s), "commit");
  return CXG_OK;
}

namespace {

// Shared body of the two element-level entry points.
int element_level(int32_t t, int64_t n_elems, const double* coords, const double* ue, const double* young,
                  const double* poisson, const cxg_material* material, const double* sc, double* st,
                  int32_t precision, double* Ke, double* fe, cudaStream_t s, bool tangent) {
  if (!supported(t)) return set_err(CXG_ERR_UNSUPPORTED, "unsupported element type");
  if (n_elems < 0 || !coords || !Ke) return set_err(CXG_ERR_INVALID_ARGUMENT, "coords and Ke are required");
  if (tangent && (!ue || !material || !fe)) return set_err(CXG_ERR_INVALID_ARGUMENT, "ue, material, fe required");
  if (precision != 0 && precision != 1) return set_err(CXG_ERR_INVALID_ARGUMENT, "bad precision");
  CHECK_CUDA(ensure_tables(), "constant tables");
  const int n = nodes_of(t), nq = gauss_of(t), nd = 3 * n;
  const size_t E = static_cast<size_t>(n_elems);
  std::vector<void*> owned;
  auto cleanup = [&]() {
    for (void* b : owned) cudaFree(b);
  };
  auto dev_in = [&](const void* ptr, size_t bytes, void** outp) -> cudaError_t {
    if (!ptr) {
      *outp = nullptr;
      return cudaSuccess;
    }
    if (on_device(ptr)) {
      *outp = const_cast<void*>(ptr);
      return cudaSuccess;
    }
    cudaError_t e = cudaMalloc(outp, std::max<size_t>(bytes, 8));
    if (e != cudaSuccess) return e;
    owned.push_back(*outp);
    return cudaMemcpyAsync(*outp, ptr, bytes, cudaMemcpyHostToDevice, s);
  };
  auto dev_out = [&](void* ptr, size_t bytes, void** outp) -> cudaError_t {
    if (!ptr) {
      *outp = nullptr;
      return cudaSuccess;
    }
    if (on_device(ptr)) {
      *outp = ptr;
      return cudaSuccess;
    }
    cudaError_t e = cudaMalloc(outp, std::max<size_t>(bytes, 8));
    if (e == cudaSuccess) owned.push_back(*outp);
    return e;
  };
  ElemArgs a{};
  a.n_elems = n_elems;
  void *dc = nullptr, *du = nullptr, *dE = nullptr, *dnu = nullptr, *dK = nullptr, *dfe = nullptr;
  cudaError_t e = dev_in(coords, sizeof(double) * E * nd, &dc);
  if (e == cudaSuccess) e = dev_in(ue, sizeof(double) * E * nd, &du);
  std::vector<double> hE, hnu;
  if (e == cudaSuccess) {
    if (tangent) {
      hE.assign(std::max<size_t>(E, 1), material->E);
      hnu.assign(std::max<size_t>(E, 1), material->nu);
      e = dev_in(hE.data(), sizeof(double) * E, &dE);
      if (e == cudaSuccess) e = dev_in(hnu.data(), sizeof(double) * E, &dnu);
    } else {
      e = dev_in(young, sizeof(double) * E, &dE);
      if (e == cudaSuccess) e = dev_in(poisson, sizeof(double) * E, &dnu);
    }
  }
  if (e == cudaSuccess) e = dev_out(Ke, sizeof(double) * E * nd * nd, &dK);
  if (e == cudaSuccess && tangent) e = dev_out(fe, sizeof(double) * E * nd, &dfe);
  if (e != cudaSuccess) {
    cleanup();
    return cuda_err(e, "element-level staging");
  }
  if (!dE || !dnu) {
    cleanup();
    return set_err(CXG_ERR_INVALID_ARGUMENT, "young and poisson are required");
  }
  DevStatus* dst = nullptr;
  J2Mat* dmat = nullptr;
  double *dsc = nullptr, *dst_t = nullptr, *aos = nullptr;
  const int64_t G = n_elems * nq;
  const size_t sbytes = sizeof(double) * kStateDoubles * static_cast<size_t>(std::max<int64_t>(G, 1));
  e = cudaMalloc(&dst, sizeof(DevStatus));
  if (e == cudaSuccess) owned.push_back(dst);
  DevStatus z{0, 0, ~0ull};
  if (e == cudaSuccess) e = cudaMemcpyAsync(dst, &z, sizeof z, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && tangent) {
    std::vector<J2Mat> mats;
    bool plastic = false;
    int rc = build_mats(1, material, mats, &plastic);
    if (rc) {
      cleanup();
      return rc;
    }
    int64_t counted = 0;
    e = alloc_copy(&dmat, mats.data(), 1, s, &counted);
    if (e == cudaSuccess) owned.push_back(dmat);
    if (e == cudaSuccess) e = cudaMalloc(&dsc, sbytes);
    if (e == cudaSuccess) owned.push_back(dsc);
    if (e == cudaSuccess) e = cudaMalloc(&dst_t, sbytes);
    if (e == cudaSuccess) owned.push_back(dst_t);
    if (e == cudaSuccess) e = cudaMalloc(&aos, sbytes);
    if (e == cudaSuccess) owned.push_back(aos);
    if (e == cudaSuccess) {
      if (sc)
        e = cudaMemcpyAsync(aos, sc, sizeof(double) * kStateDoubles * G, cudaMemcpyDefault, s);
      else
        e = cudaMemsetAsync(aos, 0, sbytes, s);
    }
    if (e == cudaSuccess) e = launch_state_transpose(aos, dsc, G, true, s);
  }
  if (e != cudaSuccess) {
    cleanup();
    return cuda_err(e, "element-level setup");
  }
  a.elem_coords = static_cast<const double*>(dc);
  a.u = static_cast<const double*>(du);
  a.young = static_cast<const double*>(dE);
  a.poisson = static_cast<const double*>(dnu);
  a.mats = dmat;
  a.state_c = dsc;
  a.state_t = dst_t;
  a.n_gauss = G;
  a.Ke = static_cast<double*>(dK);
  a.fe = static_cast<double*>(dfe);
  a.status = dst;
  e = launch_element_kernel(t, tangent ? MODE_TANGENT : MODE_LINEAR, true, precision, a, s);
  if (e == cudaSuccess && Ke != dK) e = cudaMemcpyAsync(Ke, dK, sizeof(double) * E * nd * nd, cudaMemcpyDefault, s);
  if (e == cudaSuccess && tangent && fe != dfe) e = cudaMemcpyAsync(fe, dfe, sizeof(double) * E * nd, cudaMemcpyDefault, s);
  if (e == cudaSuccess && tangent && st) {
    e = launch_state_transpose(dst_t, aos, G, false, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(st, aos, sizeof(double) * kStateDoubles * G, cudaMemcpyDefault, s);
  }
  DevStatus hs{};
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hs, dst, sizeof hs, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cleanup();
  if (e != cudaSuccess) return cuda_err(e, "element-level kernel");
  if (hs.code) {
    char buf[160];
    snprintf(buf, sizeof buf, "non-positive element Jacobian (bad connectivity?) at element index %llu", hs.bad_elem);
    return set_err(hs.code, buf);
  }
  return CXG_OK;
}

}  // namespace

int cxg_element_stiffness(int32_t t, int64_t n_elems, const double* coords, const double* young,
                          const double* poisson, int32_t precision, double* Ke, void* stream) {
  return element_level(t, n_elems, coords, nullptr, young, poisson, nullptr, nullptr, nullptr, precision, Ke,
                       nullptr, static_cast<cudaStream_t>(stream), false);
}

int cxg_element_tangent_force(int32_t t, int64_t n_elems, const double* coords, const double* ue,
                              const cxg_material* material, const double* sc, double* st, int32_t precision,
                              double* Ke, double* fe, void* stream) {
  return element_level(t, n_elems, coords, ue, nullptr, nullptr, material, sc, st, precision, Ke, fe,
                       static_cast<cudaStream_t>(stream), true);
}

int cxg_adjoint_compliance(cxg_plan* p, const double* u, double* dc_dE, double* dc_dX, void* stream) {
  if (!p || !u) return set_err(CXG_ERR_INVALID_ARGUMENT, "plan and u are required");
  if (p->type == C3D8R)
    return set_err(CXG_ERR_UNSUPPORTED, "compliance adjoint of the hourglass-stabilised C3D8R is not provided");
  if (p->has_plastic) return set_err(CXG_ERR_UNSUPPORTED, "compliance adjoint is for linear elasticity");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  p->last_stream = s;
  const size_t ub = sizeof(double) * 3 * static_cast<size_t>(p->n_nodes);
  const size_t eb = sizeof(double) * static_cast<size_t>(p->n_elems);
  void *du, *dE, *dX;
  int rc = staged(p, 3, u, ub, true, s, &du);
  if (!rc) rc = staged(p, 1, dc_dE, eb, false, s, &dE);
  if (!rc) rc = staged(p, 4, dc_dX, ub, false, s, &dX);
  if (rc) return rc;
  if (dX) CHECK_CUDA(cudaMemsetAsync(dX, 0, ub, s), "zero dc_dX");
  ElemArgs a = base_args(p);
  a.u = static_cast<const double*>(du);
  CHECK_CUDA(launch_adjoint(p->type, a, static_cast<double*>(dE), static_cast<double*>(dX), s), "adjoint kernel");
  if ((rc = copy_out(dc_dE, dE, eb, s))) return rc;
  if ((rc = copy_out(dc_dX, dX, ub, s))) return rc;
  if ((dc_dE && dE != dc_dE) || (dc_dX && dX != dc_dX)) CHECK_CUDA(cudaStreamSynchronize(s), "sync");
  return CXG_OK;
}

int cxg_spmv(cxg_plan* p, const double* vals, const double* x, double* y, void* stream) {
  if (!p || !vals || !x || !y) return set_err(CXG_ERR_INVALID_ARGUMENT, "plan, vals, x, y are required");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  p->last_stream = s;
  const size_t vb = sizeof(double) * static_cast<size_t>(active_nnz(p));
  const size_t nb = sizeof(double) * static_cast<size_t>(active_n_free(p));
  void *dv, *dx, *dy;
  int rc = staged(p, 0, vals, vb, true, s, &dv);
  if (!rc) rc = staged(p, 2, x, nb, true, s, &dx);
  if (!rc) rc = staged(p, 1, y, nb, false, s, &dy);
  if (rc) return rc;
  CHECK_CUDA(launch_spmv(active_n_free(p), active_row_ptr(p), active_col_idx(p), static_cast<const double*>(dv),
                         static_cast<const double*>(dx), static_cast<double*>(dy), s), "spmv");
  if ((rc = copy_out(y, dy, nb, s))) return rc;
  if (dy != y) CHECK_CUDA(cudaStreamSynchronize(s), "sync");
  return CXG_OK;
}

int cxg_solve_cg(cxg_plan* p, const double* vals, const double* rhs, double* x, double rtol, int32_t max_iter,
                 int32_t* iterations, double* rel_residual, void* stream) {
  if (!p || !vals || !rhs || !x || max_iter < 0) return set_err(CXG_ERR_INVALID_ARGUMENT, "bad argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  p->last_stream = s;
  const size_t vb = sizeof(double) * static_cast<size_t>(active_nnz(p));
  const size_t nb = sizeof(double) * static_cast<size_t>(active_n_free(p));
  void *dv, *db, *dx;
  int rc = staged(p, 0, vals, vb, true, s, &dv);
  if (!rc) rc = staged(p, 1, rhs, nb, true, s, &db);
  if (!rc) rc = staged(p, 2, x, nb, true, s, &dx);
  if (rc) return rc;
  const size_t wb = sizeof(double) * (5 * static_cast<size_t>(active_n_free(p)) + 2056);
  if (p->stage_bytes[5] < wb) {
    cudaFree(p->stage[5]);
    p->stage[5] = nullptr;
    p->stage_bytes[5] = 0;
    CHECK_CUDA(cudaMalloc(&p->stage[5], wb), "solver work");
    p->stage_bytes[5] = wb;
  }
  int it = 0;
  double rel = 0.0;
  CHECK_CUDA(cg_solve(active_n_free(p), active_row_ptr(p), active_col_idx(p), static_cast<const double*>(dv),
                      static_cast<const double*>(db), static_cast<double*>(dx), rtol, max_iter,
                      static_cast<double*>(p->stage[5]), &it, &rel, s), "cg");
  if ((rc = copy_out(x, dx, nb, s))) return rc;
  CHECK_CUDA(cudaStreamSynchronize(s), "sync");
  if (iterations) *iterations = it;
  if (rel_residual) *rel_residual = rel;
  if (!(rel <= rtol)) {
    char buf[160];
    snprintf(buf, sizeof buf, "CG did not converge (relative residual %.3e after %d iterations)", rel, it);
    return set_err(CXG_ERR_NOT_CONVERGED, buf);
  }
  return CXG_OK;
}

}  // extern "C"

// ---- element_tangent_force without device allocation -------------------------------
// The scratch of cxg_element_tangent_force (J2 history in the kernel's point-major
// layout, per-element elastic constants, the material record and the error word)
// lives in this file-scope device buffer instead of cudaMalloc'ed memory. Host code
// never dereferences the symbol: its device address is looked up once per device
// with cudaGetSymbolAddress and passed to the kernels.
namespace {

constexpr int64_t kNoallocPoints = CXG_NOALLOC_MAX_GAUSS_POINTS;
constexpr size_t kNoallocStateBytes = sizeof(double) * kStateDoubles * kNoallocPoints;
constexpr size_t kNoallocPropBytes = sizeof(double) * kNoallocPoints;
constexpr size_t kNoallocMatOffset = 2 * kNoallocStateBytes + 2 * kNoallocPropBytes;
constexpr size_t kNoallocStatusOffset = kNoallocMatOffset + ((sizeof(J2Mat) + 255) / 256) * 256;
static_assert(kNoallocStatusOffset + sizeof(DevStatus) <= CXG_NOALLOC_SCRATCH_BYTES, "scratch layout");

static __device__ __align__(256) unsigned char g_noalloc_scratch[CXG_NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mu;
void* g_noalloc_addr[64] = {};

__global__ void fill_pair_kernel(double* a, double va, double* b, double vb, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    a[i] = va;
    b[i] = vb;
  }
}

}  // namespace

extern "C" int cxg_element_tangent_force_noalloc(int32_t t, int64_t n_elems, const double* coords, const double* ue,
                                                 const cxg_material* material, const double* sc, double* st,
                                                 int32_t precision, double* Ke, double* fe, void* stream) {
  if (!supported(t)) return set_err(CXG_ERR_UNSUPPORTED, "unsupported element type");
  if (n_elems < 0 || !coords || !ue || !material || !Ke || !fe)
    return set_err(CXG_ERR_INVALID_ARGUMENT, "coords, ue, material, Ke and fe are required");
  if (precision != 0 && precision != 1) return set_err(CXG_ERR_INVALID_ARGUMENT, "bad precision");
  const int64_t G = n_elems * gauss_of(t);
  if (G > kNoallocPoints)
    return set_err(CXG_ERR_INVALID_ARGUMENT,
                   "batch of " + std::to_string(G) + " Gauss points exceeds the no-allocation limit of " +
                       std::to_string(kNoallocPoints) + " (CXG_NOALLOC_MAX_GAUSS_POINTS); split the batch");
  const void* arrays[] = {coords, ue, Ke, fe, sc, st};
  for (const void* ptr : arrays)
    if (ptr && !on_device(ptr))
      return set_err(CXG_ERR_INVALID_ARGUMENT, "every array argument must be device memory");
  std::vector<J2Mat> mats;
  bool plastic = false;
  int rc = build_mats(1, material, mats, &plastic);
  if (rc) return rc;
  int dev = 0;
  CHECK_CUDA(cudaGetDevice(&dev), "device");
  if (dev < 0 || dev >= 64) return set_err(CXG_ERR_UNSUPPORTED, "device ordinal above 63");
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      void* addr = nullptr;
      CHECK_CUDA(cudaGetSymbolAddress(&addr, g_noalloc_scratch), "scratch address");
      g_noalloc_addr[dev] = addr;
    }
    base = static_cast<unsigned char*>(g_noalloc_addr[dev]);
  }
  CHECK_CUDA(ensure_tables(), "constant tables");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* d_sc = reinterpret_cast<double*>(base);
  double* d_st = reinterpret_cast<double*>(base + kNoallocStateBytes);
  double* d_E = reinterpret_cast<double*>(base + 2 * kNoallocStateBytes);
  double* d_nu = reinterpret_cast<double*>(base + 2 * kNoallocStateBytes + kNoallocPropBytes);
  J2Mat* d_mat = reinterpret_cast<J2Mat*>(base + kNoallocMatOffset);
  DevStatus* d_status = reinterpret_cast<DevStatus*>(base + kNoallocStatusOffset);
  if (n_elems == 0) return CXG_OK;
  const DevStatus clear{0, 0, ~0ull};
  CHECK_CUDA(cudaMemcpyAsync(d_mat, mats.data(), sizeof(J2Mat), cudaMemcpyHostToDevice, s), "material");
  CHECK_CUDA(cudaMemcpyAsync(d_status, &clear, sizeof clear, cudaMemcpyHostToDevice, s), "status");
  const unsigned grid = static_cast<unsigned>(std::min<int64_t>((n_elems + 255) / 256, 1024));
  fill_pair_kernel<<<grid, 256, 0, s>>>(d_E, material->E, d_nu, material->nu, n_elems);
  CHECK_CUDA(cudaGetLastError(), "constants");
  if (sc)
    CHECK_CUDA(launch_state_transpose(sc, d_sc, G, true, s), "state in");
  else
    CHECK_CUDA(cudaMemsetAsync(d_sc, 0, sizeof(double) * kStateDoubles * G, s), "state in");
  ElemArgs a{};
  a.n_elems = n_elems;
  a.elem_coords = coords;
  a.u = ue;
  a.young = d_E;
  a.poisson = d_nu;
  a.mats = d_mat;
  a.state_c = d_sc;
  a.state_t = d_st;
  a.n_gauss = G;
  a.Ke = Ke;
  a.fe = fe;
  a.status = d_status;
  CHECK_CUDA(launch_element_kernel(t, MODE_TANGENT, true, precision, a, s), "element kernel");
  if (st) CHECK_CUDA(launch_state_transpose(d_st, st, G, false, s), "state out");
  DevStatus hs{};
  CHECK_CUDA(cudaMemcpyAsync(&hs, d_status, sizeof hs, cudaMemcpyDeviceToHost, s), "status read");
  CHECK_CUDA(cudaStreamSynchronize(s), "synchronize");
  if (hs.code) {
    char buf[160];
    snprintf(buf, sizeof buf, "non-positive element Jacobian (bad connectivity?) at element index %llu", hs.bad_elem);
    return set_err(hs.code, buf);
  }
  return CXG_OK;
}

