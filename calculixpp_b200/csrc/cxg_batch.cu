// Batches of independent models (cxg_batch_* in include/cxg.h): linear elastic, or J2
// plastic with a batched material-point (tangent) assembly.
//
// Models are grouped by element type. A group is one plan over the disjoint union of
// its models: node, element and equation numbers of model k are shifted by the totals
// of models 0..k-1, so the group's CSR is block diagonal, every model's rows are a
// contiguous range of it, and the row gather sums each model's entries in the same
// element order as a plan of that model alone (identical results). By default one
// assembly of the batch is one element pass plus one row gather per group, and the
// graph form captures the groups as independent branches so small groups run side by
// side. In the one-launch mode (cxg_batch_set_launch) the whole batch is one element
// pass and one row gather: every group is a slot of the same two kernels, with a share
// of the persistent grid in proportion to its measured (or estimated) pass time.
//
// The autotuner times candidate launch shapes of each pass with CUDA events on the
// batch's own data and keeps the fastest; a JSON file caches the choices.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "cxg_plan.hpp"

using namespace cxg;
using namespace cxg::api;

namespace {

struct Group {
  int32_t type = 0;
  cxg_plan* plan = nullptr;
  // one-launch mode, per precision: element-pass tile and the slot's pass times in ms
  // from the tuner (0: estimated from the element count and family)
  int ftile[2] = {1, 1};
  double fms1[2] = {0.0, 0.0}, fms2[2] = {0.0, 0.0};
  int64_t node0 = 0, vals0 = 0, rhs0 = 0;  // offsets in the batch's node / vals / rhs order
  cudaStream_t side = nullptr;               // branch stream of the graph
  cudaEvent_t join = nullptr;
  std::vector<int32_t> models;
};

struct Model {
  int32_t group = 0;
  int64_t n_nodes = 0, n_elems = 0, node0 = 0;  // node0 inside the group
  int32_t n_free = 0, row0 = 0;                  // row0 inside the group
  int64_t nnz = 0, nnz0 = 0;                     // nnz0 inside the group
  int64_t e0 = 0;                                // first element inside the group
};

__global__ void shift_kernel(int32_t* v, int64_t n, int32_t add, int only_nonneg) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    if (!only_nonneg || v[i] >= 0) v[i] += add;
}

__global__ void props_kernel(const int32_t* elem_mat, const double* E, const double* nu, int n_mats, int64_t n,
                             double* young, double* poisson, int* bad) {
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n;
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

unsigned grid_for(int64_t n) {
  return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4096)));
}

}  // namespace

struct cxg_batch {
  int device = 0;
  int32_t precision = 0;
  std::vector<Group> groups;
  std::vector<Model> models;
  int64_t n_nodes = 0, n_elems = 0, n_free = 0, nnz = 0;
  cudaEvent_t fork = nullptr;
  // captured graph and the launch it replays
  cudaGraphExec_t exec = nullptr;
  const void* key[3] = {nullptr, nullptr, nullptr};
  int32_t key_precision = -1;
  uint64_t key_cfg = 0;
  int32_t launch = CXG_BATCH_PER_GROUP;
  int fwarps[2] = {0, 0};  // one-launch row gather: warps per block (0: as many as fit, <= 8)
};

namespace {

uint64_t cfg_hash(const cxg_batch* b) {
  uint64_t h = 1469598103934665603ull;
  for (const Group& g : b->groups)
    for (int pr = 0; pr < 2; ++pr) {
      const LaunchCfg& c = g.plan->cfg[pr];
      for (int v : {c.tile, c.p1_blocks_per_sm, c.p2_warps, c.p2_blocks_per_sm}) h = (h ^ static_cast<uint64_t>(v + 7)) * 1099511628211ull;
      uint64_t w1 = 0, w2 = 0;
      std::memcpy(&w1, &g.fms1[pr], 8);
      std::memcpy(&w2, &g.fms2[pr], 8);
      for (uint64_t v : {static_cast<uint64_t>(g.ftile[pr]), w1, w2}) h = (h ^ v) * 1099511628211ull;
    }
  for (int v : {b->launch, b->fwarps[0], b->fwarps[1]}) h = (h ^ static_cast<uint64_t>(v + 7)) * 1099511628211ull;
  return h;
}

void destroy_batch(cxg_batch* b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (Group& g : b->groups) {
    if (g.side) cudaStreamSynchronize(g.side);
    cxg_plan_destroy(g.plan);
    if (g.side) cudaStreamDestroy(g.side);
    if (g.join) cudaEventDestroy(g.join);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  delete b;
}

// Issue one group's two passes on stream s (device buffers of the whole batch).
cudaError_t launch_group(cxg_batch* b, Group& g, double* vals, double* rhs, const double* f_ext, cudaStream_t s,
                         const LaunchCfg* override_cfg = nullptr) {
  cxg_plan* p = g.plan;
  p->last_stream = s;
  ElemArgs a = base_args(p);
  a.vals = vals + g.vals0;
  a.rhs = rhs ? rhs + g.rhs0 : nullptr;
  V2Args v = v2_args(p, f_ext ? f_ext + 3 * g.node0 : nullptr, false);
  apply_windows(p, false, v);
  return launch_v2(p->type, MODE_LINEAR, b->precision, a, v, s, override_cfg ? *override_cfg : p->cfg[b->precision]);
}

// Pass-time estimates of a group when the tuner has not measured it: element pass ~
// node pairs x (Gauss points + block stores), row gather ~ stored blocks.
double p1_estimate(int t, int64_t ne) {
  const double n = nodes_of(t), nq = gauss_of(t);
  return static_cast<double>(ne) * n * n * (nq + 4.0);
}
double p2_estimate(int t, int64_t ne) {
  const double n = nodes_of(t);
  return static_cast<double>(ne) * n * (n + 1.0) / 2.0;
}

// Every group as one slot of the one-launch kernels. Linear mode when u is null, else
// the material-point (tangent) assembly. Weights are the tuned times when every group
// has one, else the estimates.
int fill_slots(cxg_batch* b, const double* u, double* vals, double* f_int, double* rhs, const double* f_ext,
               cudaStream_t s, std::vector<BatchSlotIn>& slots) {
  const int pr = b->precision ? 1 : 0;
  const bool tan = u != nullptr;
  if (b->groups.size() > static_cast<size_t>(kMaxBatchSlots))
    return set_err(CXG_ERR_UNSUPPORTED, "one-launch batch holds at most 8 element-type groups");
  bool tuned = true;
  for (const Group& g : b->groups) tuned = tuned && g.fms1[pr] > 0.0 && g.fms2[pr] > 0.0;
  slots.clear();
  for (Group& g : b->groups) {
    cxg_plan* p = g.plan;
    p->last_stream = s;
    BatchSlotIn in;
    in.a = base_args(p);
    in.a.vals = vals + g.vals0;
    in.a.rhs = rhs ? rhs + g.rhs0 : nullptr;
    if (tan) {
      in.a.f_int = f_int ? f_int + 3 * g.node0 : nullptr;
      in.a.u = u + 3 * g.node0;
      in.a.state_c = p->state[0];
      in.a.state_t = p->state[1];
      in.a.state_comps = state_comps(p);
    }
    in.v = v2_args(p, f_ext ? f_ext + 3 * g.node0 : nullptr, false);
    apply_windows(p, tan, in.v);
    if (in.v.n_win > 1 || in.v.node_order)
      return set_err(CXG_ERR_UNSUPPORTED, "one-launch batch assembles every group as one window (no element-buffer budget)");
    in.type = g.type;
    in.cfg = tan ? p->tcfg[pr] : p->cfg[pr];
    in.cfg.tile = tan ? 1 : g.ftile[pr];
    in.cfg.p2_warps = b->fwarps[pr];
    in.p1_weight = tuned ? g.fms1[pr] : p1_estimate(g.type, p->n_elems);
    in.p2_weight = tuned ? g.fms2[pr] : p2_estimate(g.type, p->n_elems);
    slots.push_back(in);
  }
  return CXG_OK;
}

cudaError_t launch_one(cxg_batch* b, const std::vector<BatchSlotIn>& slots, int mode, int passes, cudaStream_t s) {
  return launch_v2_batch(mode, b->precision, slots.data(), static_cast<int>(slots.size()), passes, s);
}

int prepare(cxg_batch* b) {
  for (Group& g : b->groups) {
    g.plan->precision = b->precision;
    int rc = ensure_v2(g.plan, false);
    if (rc) return rc;
  }
  return CXG_OK;
}

const char* type_name(int t) {
  switch (t) {
    case C3D4: return "C3D4";
    case C3D10: return "C3D10";
    case C3D8: return "C3D8";
    case C3D8R: return "C3D8R";
    case C3D20: return "C3D20";
    case C3D20R: return "C3D20R";
    case C3D6: return "C3D6";
    case C3D15: return "C3D15";
    default: return "unknown";
  }
}

// ---- tuning cache: {"<key>": {"tile": t, "p1_blocks_per_sm": a, "p2_warps": w}, ...}
struct CacheEntry {
  int tile = 0, p1 = 0, warps = 0;
  double p1_ms = 0.0, p2_ms = 0.0;
};

std::map<std::string, CacheEntry> read_cache(const char* path) {
  std::map<std::string, CacheEntry> out;
  if (!path) return out;
  FILE* f = fopen(path, "r");
  if (!f) return out;
  char line[512];
  while (fgets(line, sizeof line, f)) {
    char key[256];
    CacheEntry c;
    if (sscanf(line, " \"%255[^\"]\": {\"tile\": %d, \"p1_blocks_per_sm\": %d, \"p2_warps\": %d, \"p1_ms\": %lf, \"p2_ms\": %lf",
               key, &c.tile, &c.p1, &c.warps, &c.p1_ms, &c.p2_ms) == 6)
      out[key] = c;
  }
  fclose(f);
  return out;
}

bool write_cache(const char* path, const std::map<std::string, CacheEntry>& m) {
  if (!path) return true;
  const std::string tmp = std::string(path) + ".tmp";
  FILE* f = fopen(tmp.c_str(), "w");
  if (!f) return false;
  fprintf(f, "{\n");
  size_t i = 0;
  for (const auto& kv : m) {
    const CacheEntry& c = kv.second;
    fprintf(f, "  \"%s\": {\"tile\": %d, \"p1_blocks_per_sm\": %d, \"p2_warps\": %d, \"p1_ms\": %.6f, \"p2_ms\": %.6f}%s\n",
            kv.first.c_str(), c.tile, c.p1, c.warps, c.p1_ms, c.p2_ms, ++i < m.size() ? "," : "");
  }
  fprintf(f, "}\n");
  fclose(f);
  return rename(tmp.c_str(), path) == 0;
}

std::string cache_key(const cxg_batch* b, const Group& g) {
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  const int bucket = g.plan->n_elems > 0 ? static_cast<int>(std::floor(std::log2(static_cast<double>(g.plan->n_elems)))) : 0;
  char buf[128];
  snprintf(buf, sizeof buf, "sm%d/%s/%s/e2^%d", sms, type_name(g.type), b->precision ? "mixed" : "fp64", bucket);
  return buf;
}

// Median of `reps` timed launches of one pass (after one untimed launch).
int time_pass(cxg_batch* b, Group& g, double* vals, double* rhs, const double* f_ext, const LaunchCfg& c,
              cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1, double* ms_out) {
  const int reps = 3;
  std::vector<float> t;
  for (int r = 0; r <= reps; ++r) {
    CHECK_CUDA(cudaEventRecord(e0, s), "tune event");
    cudaError_t err = launch_group(b, g, vals, rhs, f_ext, s, &c);
    if (err != cudaSuccess) {
      cudaGetLastError();
      *ms_out = -1.0;  // shape not launchable here (e.g. shared memory): skip it
      return cudaStreamSynchronize(s) == cudaSuccess ? CXG_OK : cuda_err(cudaErrorLaunchFailure, "tune");
    }
    CHECK_CUDA(cudaEventRecord(e1, s), "tune event");
    CHECK_CUDA(cudaEventSynchronize(e1), "tune sync");
    float ms = 0.f;
    CHECK_CUDA(cudaEventElapsedTime(&ms, e0, e1), "tune time");
    if (r > 0) t.push_back(ms);
  }
  std::sort(t.begin(), t.end());
  *ms_out = t[t.size() / 2];
  return CXG_OK;
}

// Median of `reps` timed one-launch passes over `slots` (after one untimed launch);
// -1 when the shape cannot launch here.
int time_one(cxg_batch* b, const std::vector<BatchSlotIn>& slots, int passes, cudaStream_t s, cudaEvent_t e0,
             cudaEvent_t e1, double* ms_out) {
  const int reps = 3;
  std::vector<float> t;
  for (int r = 0; r <= reps; ++r) {
    CHECK_CUDA(cudaEventRecord(e0, s), "tune event");
    if (launch_one(b, slots, MODE_LINEAR, passes, s) != cudaSuccess) {
      cudaGetLastError();
      *ms_out = -1.0;
      return cudaStreamSynchronize(s) == cudaSuccess ? CXG_OK : cuda_err(cudaErrorLaunchFailure, "tune");
    }
    CHECK_CUDA(cudaEventRecord(e1, s), "tune event");
    CHECK_CUDA(cudaEventSynchronize(e1), "tune sync");
    float ms = 0.f;
    CHECK_CUDA(cudaEventElapsedTime(&ms, e0, e1), "tune time");
    if (r > 0) t.push_back(ms);
  }
  std::sort(t.begin(), t.end());
  *ms_out = t[t.size() / 2];
  return CXG_OK;
}

// One-launch tuner: per group, the element-pass tile (2x2, and 2x4 in mixed precision)
// timed as a slot alone, whose time becomes its share weight; then the row gather's
// warps per block over the whole batch, and each group's gather time alone at that
// shape. Cache keys carry "/one-launch".
int tune_one_launch(cxg_batch* b, double* vals, double* rhs, const double* f_ext,
                    std::map<std::string, CacheEntry>& cache, bool* changed, cudaStream_t s) {
  const int pr = b->precision ? 1 : 0;
  std::vector<BatchSlotIn> all;
  int rc = fill_slots(b, nullptr, vals, nullptr, rhs, f_ext, s, all);
  if (rc) return rc;
  bool cached = true;
  for (Group& g : b->groups) {
    auto it = cache.find(cache_key(b, g) + "/one-launch");
    if (it == cache.end()) {
      cached = false;
      break;
    }
  }
  if (cached) {
    for (Group& g : b->groups) {
      const CacheEntry& c = cache[cache_key(b, g) + "/one-launch"];
      g.ftile[pr] = c.tile;
      g.fms1[pr] = c.p1_ms;
      g.fms2[pr] = c.p2_ms;
      b->fwarps[pr] = c.warps;
    }
  } else {
    cudaEvent_t e0, e1;
    CHECK_CUDA(cudaEventCreate(&e0), "event");
    CHECK_CUDA(cudaEventCreate(&e1), "event");
    for (size_t gi = 0; gi < b->groups.size() && !rc; ++gi) {
      Group& g = b->groups[gi];
      double best = 1e30;
      int best_tile = 1;
      for (int tile : {1, 0}) {
        if (!batch_tile_ok(MODE_LINEAR, b->precision, tile)) continue;
        std::vector<BatchSlotIn> one(1, all[gi]);
        one[0].cfg.tile = tile;
        double ms = 0.0;
        if ((rc = time_one(b, one, 1, s, e0, e1, &ms))) break;
        if (ms >= 0.0 && ms < best) {
          best = ms;
          best_tile = tile;
        }
      }
      g.ftile[pr] = best_tile;
      all[gi].cfg.tile = best_tile;
      g.fms1[pr] = best < 1e30 ? best : 0.0;
    }
    double best = 1e30;
    int best_warps = 0;
    for (int warps : {8, 4, 2}) {
      if (rc) break;
      std::vector<BatchSlotIn> sl = all;
      for (BatchSlotIn& in : sl) in.cfg.p2_warps = warps;
      double ms = 0.0;
      if ((rc = time_one(b, sl, 2, s, e0, e1, &ms))) break;
      if (ms >= 0.0 && ms < best) {
        best = ms;
        best_warps = warps;
      }
    }
    b->fwarps[pr] = best_warps;
    for (size_t gi = 0; gi < b->groups.size() && !rc; ++gi) {
      std::vector<BatchSlotIn> one(1, all[gi]);
      one[0].cfg.p2_warps = best_warps;
      double ms = 0.0;
      if ((rc = time_one(b, one, 2, s, e0, e1, &ms))) break;
      b->groups[gi].fms2[pr] = ms > 0.0 ? ms : 0.0;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    for (Group& g : b->groups) {
      CacheEntry c;
      c.tile = g.ftile[pr];
      c.warps = b->fwarps[pr];
      c.p1_ms = g.fms1[pr];
      c.p2_ms = g.fms2[pr];
      cache[cache_key(b, g) + "/one-launch"] = c;
    }
    *changed = true;
  }
  // leave a complete assembly with the chosen shapes in vals / rhs
  if ((rc = fill_slots(b, nullptr, vals, nullptr, rhs, f_ext, s, all))) return rc;
  CHECK_CUDA(launch_one(b, all, MODE_LINEAR, 3, s), "batch assembly (one launch)");
  CHECK_CUDA(cudaStreamSynchronize(s), "tuning");
  return CXG_OK;
}

}  // namespace

extern "C" {

int cxg_batch_create(int32_t n_models, const cxg_mesh_desc* meshes, const cxg_dofmap_desc* dofs, int32_t precision,
                     cxg_batch** out) {
  if (!out || !meshes || !dofs || n_models <= 0) return set_err(CXG_ERR_INVALID_ARGUMENT, "batch needs >= 1 model");
  *out = nullptr;
  if (precision != CXG_FP64 && precision != CXG_MIXED) return set_err(CXG_ERR_INVALID_ARGUMENT, "bad precision");
  for (int32_t k = 0; k < n_models; ++k) {
    const cxg_mesh_desc& m = meshes[k];
    if (!supported(m.elem_type)) return set_err(CXG_ERR_UNSUPPORTED, "unsupported element type in batch");
    if (m.n_nodes <= 0 || m.n_elems < 0 || !m.coords || (m.n_elems > 0 && !m.conn))
      return set_err(CXG_ERR_INVALID_ARGUMENT, "batch mesh needs n_nodes > 0, coords and conn");
    if (m.n_materials < 1 || !m.materials) return set_err(CXG_ERR_INVALID_ARGUMENT, "batch mesh needs >= 1 material");
    for (int32_t i = 0; i < m.n_materials; ++i) {
      if (!(m.materials[i].E > 0.0) || !(m.materials[i].nu > -1.0 && m.materials[i].nu < 0.5))
        return set_err(CXG_ERR_INVALID_ARGUMENT, "material needs E > 0 and -1 < nu < 0.5");
    }
    if (!dofs[k].dof_eq || !dofs[k].prescribed || dofs[k].n_free < 0)
      return set_err(CXG_ERR_INVALID_ARGUMENT, "bad DOF map in batch");
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_err(CXG_ERR_NO_GPU, "no CUDA device");
  }
  auto* b = new cxg_batch;
  cudaGetDevice(&b->device);
  b->precision = precision;
  b->models.resize(static_cast<size_t>(n_models));
  for (int t = kFirstType; t <= kLastType; ++t) {
    Group g;
    g.type = t;
    for (int32_t k = 0; k < n_models; ++k)
      if (meshes[k].elem_type == t) g.models.push_back(k);
    if (!g.models.empty()) b->groups.push_back(g);
  }
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
    delete b;
    return cuda_err(cudaGetLastError(), "stream");
  }
  int rc = CXG_OK;
  std::vector<void*> tmp;
  auto dalloc = [&](void** p, size_t bytes) -> bool {
    if (cudaMalloc(p, std::max<size_t>(bytes, 16)) != cudaSuccess) {
      rc = cuda_err(cudaErrorMemoryAllocation, "batch staging");
      return false;
    }
    tmp.push_back(*p);
    return true;
  };
  for (size_t gi = 0; gi < b->groups.size() && rc == CXG_OK; ++gi) {
    Group& g = b->groups[gi];
    const int npe = nodes_of(g.type);
    int64_t N = 0, E = 0, F = 0;
    for (int32_t k : g.models) {
      Model& md = b->models[static_cast<size_t>(k)];
      md.group = static_cast<int32_t>(gi);
      md.n_nodes = meshes[k].n_nodes;
      md.n_elems = meshes[k].n_elems;
      md.node0 = N;
      md.row0 = static_cast<int32_t>(F);
      md.n_free = dofs[k].n_free;
      N += md.n_nodes;
      E += md.n_elems;
      F += md.n_free;
    }
    if (F > INT32_MAX) {
      rc = set_err(CXG_ERR_UNSUPPORTED, "more than 2^31-1 free equations in one element-type group");
      break;
    }
    double *coords, *young, *poisson, *pres;
    int32_t *conn, *deq, *gem;
    if (!dalloc(reinterpret_cast<void**>(&coords), 24 * N) || !dalloc(reinterpret_cast<void**>(&pres), 24 * N) ||
        !dalloc(reinterpret_cast<void**>(&deq), 12 * N) || !dalloc(reinterpret_cast<void**>(&conn), 4 * E * npe) ||
        !dalloc(reinterpret_cast<void**>(&young), 8 * E) || !dalloc(reinterpret_cast<void**>(&poisson), 8 * E) ||
        !dalloc(reinterpret_cast<void**>(&gem), 4 * E))
      break;
    // the group's materials: every model's list in turn; elem_mat shifted by the model's
    // offset in that list (E and nu come per element, the *PLASTIC tables from here)
    std::vector<cxg_material> gmats;
    int* dbad = nullptr;
    if (!dalloc(reinterpret_cast<void**>(&dbad), sizeof(int))) break;
    cudaMemsetAsync(dbad, 0, sizeof(int), s);
    int64_t e_off = 0;
    for (int32_t k : g.models) {
      const cxg_mesh_desc& m = meshes[k];
      Model& md = b->models[static_cast<size_t>(k)];
      md.e0 = e_off;
      const int32_t mat0 = static_cast<int32_t>(gmats.size());
      gmats.insert(gmats.end(), m.materials, m.materials + m.n_materials);
      if (md.n_elems > 0) {
        if (m.elem_mat)
          cudaMemcpyAsync(gem + e_off, m.elem_mat, 4 * md.n_elems, cudaMemcpyDefault, s);
        else
          cudaMemsetAsync(gem + e_off, 0, 4 * md.n_elems, s);
        shift_kernel<<<grid_for(md.n_elems), 256, 0, s>>>(gem + e_off, md.n_elems, mat0, 0);
      }
      const int64_t n3 = 3 * md.n_nodes;
      cudaMemcpyAsync(coords + 3 * md.node0, m.coords, 8 * n3, cudaMemcpyDefault, s);
      cudaMemcpyAsync(pres + 3 * md.node0, dofs[k].prescribed, 8 * n3, cudaMemcpyDefault, s);
      cudaMemcpyAsync(deq + 3 * md.node0, dofs[k].dof_eq, 4 * n3, cudaMemcpyDefault, s);
      shift_kernel<<<grid_for(n3), 256, 0, s>>>(deq + 3 * md.node0, n3, md.row0, 1);
      if (md.n_elems > 0) {
        cudaMemcpyAsync(conn + e_off * npe, m.conn, 4 * md.n_elems * npe, cudaMemcpyDefault, s);
        shift_kernel<<<grid_for(md.n_elems * npe), 256, 0, s>>>(conn + e_off * npe, md.n_elems * npe,
                                                                static_cast<int32_t>(md.node0), 0);
        if (m.young) cudaMemcpyAsync(young + e_off, m.young, 8 * md.n_elems, cudaMemcpyDefault, s);
        if (m.poisson) cudaMemcpyAsync(poisson + e_off, m.poisson, 8 * md.n_elems, cudaMemcpyDefault, s);
        if (!m.young || !m.poisson) {
          std::vector<double> hE(static_cast<size_t>(m.n_materials)), hnu(hE.size());
          for (int32_t i = 0; i < m.n_materials; ++i) {
            hE[static_cast<size_t>(i)] = m.materials[i].E;
            hnu[static_cast<size_t>(i)] = m.materials[i].nu;
          }
          double *dE, *dnu;
          int32_t* dem = nullptr;
          if (!dalloc(reinterpret_cast<void**>(&dE), 8 * hE.size()) || !dalloc(reinterpret_cast<void**>(&dnu), 8 * hE.size()))
            break;
          cudaMemcpyAsync(dE, hE.data(), 8 * hE.size(), cudaMemcpyHostToDevice, s);
          cudaMemcpyAsync(dnu, hnu.data(), 8 * hE.size(), cudaMemcpyHostToDevice, s);
          if (m.elem_mat) {
            if (!dalloc(reinterpret_cast<void**>(&dem), 4 * md.n_elems)) break;
            cudaMemcpyAsync(dem, m.elem_mat, 4 * md.n_elems, cudaMemcpyDefault, s);
          }
          props_kernel<<<grid_for(md.n_elems), 256, 0, s>>>(dem, dE, dnu, m.n_materials, md.n_elems,
                                                            m.young ? nullptr : young + e_off,
                                                            m.poisson ? nullptr : poisson + e_off, dbad);
          // the host vectors above must outlive the copies
          cudaStreamSynchronize(s);
        }
      }
      e_off += md.n_elems;
    }
    if (rc) break;
    int bad = 0;
    cudaMemcpyAsync(&bad, dbad, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
      rc = cuda_err(cudaGetLastError(), "batch concatenation");
      break;
    }
    if (bad) {
      rc = set_err(CXG_ERR_INVALID_ARGUMENT, "elem_mat index outside [0, n_materials)");
      break;
    }
    cxg_mesh_desc desc{N, E, g.type, coords, conn, young, poisson, gem, static_cast<int32_t>(gmats.size()),
                       gmats.data()};
    cxg_dofmap_desc dd{deq, pres, static_cast<int32_t>(F)};
    rc = cxg_plan_create(&desc, &dd, precision, &g.plan);
    for (void* p : tmp) cudaFree(p);
    tmp.clear();
    if (rc) break;
    // per-model nnz from the group's row_ptr
    std::vector<int64_t> rp(static_cast<size_t>(F) + 1);
    if (cudaMemcpy(rp.data(), g.plan->pat.row_ptr, 8 * rp.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
      rc = cuda_err(cudaGetLastError(), "row_ptr read");
      break;
    }
    for (int32_t k : g.models) {
      Model& md = b->models[static_cast<size_t>(k)];
      md.nnz0 = rp[static_cast<size_t>(md.row0)];
      md.nnz = rp[static_cast<size_t>(md.row0) + md.n_free] - md.nnz0;
    }
    g.node0 = b->n_nodes;
    g.vals0 = b->nnz;
    g.rhs0 = b->n_free;
    b->n_nodes += N;
    b->n_elems += E;
    b->n_free += F;
    b->nnz += g.plan->pat.nnz;
    if (cudaStreamCreateWithFlags(&g.side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&g.join, cudaEventDisableTiming) != cudaSuccess) {
      rc = cuda_err(cudaGetLastError(), "branch stream");
      break;
    }
  }
  for (void* p : tmp) cudaFree(p);
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  if (!rc && cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
    rc = cuda_err(cudaGetLastError(), "fork event");
  if (rc) {
    const std::string msg = cxg_last_error();
    destroy_batch(b);
    return set_err(rc, msg);
  }
  *out = b;
  return CXG_OK;
}

int cxg_batch_destroy(cxg_batch* b) {
  destroy_batch(b);
  return CXG_OK;
}

int cxg_batch_get_info(const cxg_batch* b, cxg_batch_info* info) {
  if (!b || !info) return set_err(CXG_ERR_INVALID_ARGUMENT, "null argument");
  info->n_models = static_cast<int32_t>(b->models.size());
  info->n_groups = static_cast<int32_t>(b->groups.size());
  info->n_nodes = b->n_nodes;
  info->n_elems = b->n_elems;
  info->n_free = b->n_free;
  info->nnz = b->nnz;
  int64_t bytes = 0;
  for (const Group& g : b->groups) bytes += g.plan->device_bytes;
  info->device_bytes = bytes;
  return CXG_OK;
}

int cxg_batch_get_model_info(const cxg_batch* b, int32_t k, cxg_batch_model_info* info) {
  if (!b || !info || k < 0 || k >= static_cast<int32_t>(b->models.size()))
    return set_err(CXG_ERR_INVALID_ARGUMENT, "bad model index");
  const Model& md = b->models[static_cast<size_t>(k)];
  const Group& g = b->groups[static_cast<size_t>(md.group)];
  info->elem_type = g.type;
  info->group = md.group;
  info->n_nodes = md.n_nodes;
  info->n_elems = md.n_elems;
  info->n_free = md.n_free;
  info->nnz = md.nnz;
  info->vals_offset = g.vals0 + md.nnz0;
  info->rhs_offset = g.rhs0 + md.row0;
  info->node_offset = g.node0 + md.node0;
  return CXG_OK;
}

int cxg_batch_get_pattern(const cxg_batch* b, int32_t k, int64_t* row_ptr, int32_t* col_idx) {
  if (!b || k < 0 || k >= static_cast<int32_t>(b->models.size()))
    return set_err(CXG_ERR_INVALID_ARGUMENT, "bad model index");
  const Model& md = b->models[static_cast<size_t>(k)];
  const Group& g = b->groups[static_cast<size_t>(md.group)];
  if (row_ptr) {
    std::vector<int64_t> rp(static_cast<size_t>(md.n_free) + 1);
    CHECK_CUDA(cudaMemcpy(rp.data(), g.plan->pat.row_ptr + md.row0, 8 * rp.size(), cudaMemcpyDeviceToHost), "row_ptr");
    for (int64_t& v : rp) v -= md.nnz0;
    CHECK_CUDA(cudaMemcpy(row_ptr, rp.data(), 8 * rp.size(), cudaMemcpyDefault), "row_ptr");
  }
  if (col_idx && md.nnz > 0) {
    std::vector<int32_t> ci(static_cast<size_t>(md.nnz));
    CHECK_CUDA(cudaMemcpy(ci.data(), g.plan->pat.col_idx + md.nnz0, 4 * ci.size(), cudaMemcpyDeviceToHost), "col_idx");
    for (int32_t& v : ci) v -= md.row0;
    CHECK_CUDA(cudaMemcpy(col_idx, ci.data(), 4 * ci.size(), cudaMemcpyDefault), "col_idx");
  }
  return CXG_OK;
}

int cxg_batch_set_precision(cxg_batch* b, int32_t precision) {
  if (!b || (precision != CXG_FP64 && precision != CXG_MIXED)) return set_err(CXG_ERR_INVALID_ARGUMENT, "bad precision");
  b->precision = precision;
  return CXG_OK;
}

int cxg_batch_set_launch(cxg_batch* b, int32_t mode) {
  if (!b || (mode != CXG_BATCH_PER_GROUP && mode != CXG_BATCH_ONE_LAUNCH))
    return set_err(CXG_ERR_INVALID_ARGUMENT, "bad batch launch mode");
  if (mode == CXG_BATCH_ONE_LAUNCH && b->groups.size() > static_cast<size_t>(kMaxBatchSlots))
    return set_err(CXG_ERR_UNSUPPORTED, "one-launch batch holds at most 8 element-type groups");
  b->launch = mode;
  return CXG_OK;
}

int cxg_batch_get_launch(const cxg_batch* b, int32_t* mode) {
  if (!b || !mode) return set_err(CXG_ERR_INVALID_ARGUMENT, "bad argument");
  *mode = b->launch;
  return CXG_OK;
}

int cxg_batch_assemble(cxg_batch* b, double* vals, double* rhs, const double* f_ext, void* stream) {
  if (!b || !vals) return set_err(CXG_ERR_INVALID_ARGUMENT, "batch and vals are required");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = prepare(b);
  if (rc) return rc;
  const bool hv = !on_device(vals), hr = rhs && !on_device(rhs), hf = f_ext && !on_device(f_ext);
  double *dv = vals, *dr = rhs, *df = const_cast<double*>(f_ext);
  if (hv) CHECK_CUDA(cudaMallocAsync(&dv, 8 * std::max<int64_t>(b->nnz, 1), s), "vals staging");
  if (hr) CHECK_CUDA(cudaMallocAsync(&dr, 8 * std::max<int64_t>(b->n_free, 1), s), "rhs staging");
  if (hf) {
    CHECK_CUDA(cudaMallocAsync(&df, 24 * b->n_nodes, s), "load staging");
    CHECK_CUDA(cudaMemcpyAsync(df, f_ext, 24 * b->n_nodes, cudaMemcpyHostToDevice, s), "load upload");
  }
  if (b->launch == CXG_BATCH_ONE_LAUNCH) {
    std::vector<BatchSlotIn> slots;
    rc = fill_slots(b, nullptr, dv, nullptr, dr, df, s, slots);
    if (rc) {
      if (hv) cudaFreeAsync(dv, s);
      if (hr) cudaFreeAsync(dr, s);
      if (hf) cudaFreeAsync(df, s);
      return rc;
    }
    CHECK_CUDA(launch_one(b, slots, MODE_LINEAR, 3, s), "batch assembly (one launch)");
  } else {
    for (Group& g : b->groups) CHECK_CUDA(launch_group(b, g, dv, dr, df, s), "batch assembly");
  }
  if (hv) CHECK_CUDA(cudaMemcpyAsync(vals, dv, 8 * b->nnz, cudaMemcpyDeviceToHost, s), "vals download");
  if (hr) CHECK_CUDA(cudaMemcpyAsync(rhs, dr, 8 * b->n_free, cudaMemcpyDeviceToHost, s), "rhs download");
  if (hv) cudaFreeAsync(dv, s);
  if (hr) cudaFreeAsync(dr, s);
  if (hf) cudaFreeAsync(df, s);
  if (hv || hr) CHECK_CUDA(cudaStreamSynchronize(s), "synchronize");
  return CXG_OK;
}

int cxg_batch_graph_launch(cxg_batch* b, double* vals, double* rhs, const double* f_ext, void* stream) {
  if (!b || !vals) return set_err(CXG_ERR_INVALID_ARGUMENT, "batch and vals are required");
  if (!on_device(vals) || (rhs && !on_device(rhs)) || (f_ext && !on_device(f_ext)))
    return set_err(CXG_ERR_INVALID_ARGUMENT, "graph launch needs device buffers");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const uint64_t h = cfg_hash(b);
  if (!b->exec || b->key[0] != vals || b->key[1] != rhs || b->key[2] != f_ext || b->key_precision != b->precision ||
      b->key_cfg != h) {
    if (b->exec) {
      cudaGraphExecDestroy(b->exec);
      b->exec = nullptr;
    }
    int rc = prepare(b);
    if (rc) return rc;
    const bool one = b->launch == CXG_BATCH_ONE_LAUNCH;
    std::vector<BatchSlotIn> slots;
    if (one && (rc = fill_slots(b, nullptr, vals, nullptr, rhs, f_ext, s, slots))) return rc;
    // launch once outside capture so kernel attributes are set before capturing
    if (one)
      CHECK_CUDA(launch_one(b, slots, MODE_LINEAR, 3, s), "batch assembly (one launch)");
    else
      for (Group& g : b->groups) CHECK_CUDA(launch_group(b, g, vals, rhs, f_ext, s), "batch assembly");
    cudaStream_t cs = nullptr;
    CHECK_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "capture stream");
    CHECK_CUDA(cudaStreamSynchronize(s), "synchronize");
    cudaGraph_t graph = nullptr;
    cudaError_t err = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (err == cudaSuccess && one) err = launch_one(b, slots, MODE_LINEAR, 3, cs);
    if (err == cudaSuccess && !one) err = cudaEventRecord(b->fork, cs);
    for (Group& g : b->groups) {
      if (err != cudaSuccess || one) break;
      err = cudaStreamWaitEvent(g.side, b->fork, 0);
      if (err == cudaSuccess) err = launch_group(b, g, vals, rhs, f_ext, g.side);
      if (err == cudaSuccess) err = cudaEventRecord(g.join, g.side);
      if (err == cudaSuccess) err = cudaStreamWaitEvent(cs, g.join, 0);
    }
    const cudaError_t end = cudaStreamEndCapture(cs, &graph);
    if (err == cudaSuccess) err = end;
    if (err == cudaSuccess) err = cudaGraphInstantiate(&b->exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cs);
    if (err != cudaSuccess) {
      b->exec = nullptr;
      return cuda_err(err, "graph capture");
    }
    b->key[0] = vals;
    b->key[1] = rhs;
    b->key[2] = f_ext;
    b->key_precision = b->precision;
    b->key_cfg = h;
  }
  for (Group& g : b->groups) g.plan->last_stream = s;
  CHECK_CUDA(cudaGraphLaunch(b->exec, s), "graph launch");
  return CXG_OK;
}

int cxg_batch_check(cxg_batch* b) {
  if (!b) return set_err(CXG_ERR_INVALID_ARGUMENT, "null batch");
  for (Group& g : b->groups) {
    if (!g.plan->last_stream) g.plan->last_stream = g.side;
    int rc = plan_status(g.plan, nullptr);
    if (rc) return rc;
  }
  return CXG_OK;
}

int cxg_batch_tune(cxg_batch* b, double* vals, double* rhs, const double* f_ext, const char* cache_path,
                   void* stream) {
  if (!b || !vals || !on_device(vals) || (rhs && !on_device(rhs)) || (f_ext && !on_device(f_ext)))
    return set_err(CXG_ERR_INVALID_ARGUMENT, "tuning needs the batch and device buffers");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = prepare(b);
  if (rc) return rc;
  std::map<std::string, CacheEntry> cache = read_cache(cache_path);
  bool changed = false;
  if (b->launch == CXG_BATCH_ONE_LAUNCH) {
    rc = tune_one_launch(b, vals, rhs, f_ext, cache, &changed, s);
    if (!rc && changed && !write_cache(cache_path, cache))
      rc = set_err(CXG_ERR_INVALID_ARGUMENT, std::string("cannot write tuning cache ") + cache_path);
    return rc;
  }
  cudaEvent_t e0, e1;
  CHECK_CUDA(cudaEventCreate(&e0), "event");
  CHECK_CUDA(cudaEventCreate(&e1), "event");
  for (Group& g : b->groups) {
    const std::string key = cache_key(b, g);
    LaunchCfg& cfg = g.plan->cfg[b->precision];
    auto it = cache.find(key);
    if (it != cache.end()) {
      cfg.tile = it->second.tile;
      cfg.p1_blocks_per_sm = it->second.p1;
      cfg.p2_warps = it->second.warps;
      continue;
    }
    // element pass: tile x persistent grid; the row gather reads what it wrote
    CacheEntry best;
    best.p1_ms = 1e30;
    const std::vector<int> tiles = b->precision ? std::vector<int>{0, 1, 2} : std::vector<int>{0, 1};
    for (int tile : tiles)
      for (int bps : {0, 1, 2}) {
        LaunchCfg c;
        c.tile = tile;
        c.p1_blocks_per_sm = bps;
        c.passes = 1;
        double ms = 0.0;
        if ((rc = time_pass(b, g, vals, rhs, f_ext, c, s, e0, e1, &ms))) goto done;
        if (ms >= 0.0 && ms < best.p1_ms) {
          best.p1_ms = ms;
          best.tile = tile;
          best.p1 = bps;
        }
      }
    best.p2_ms = 1e30;
    for (int warps : {2, 4, 8}) {
      LaunchCfg c;
      c.p2_warps = warps;
      c.passes = 2;
      double ms = 0.0;
      if ((rc = time_pass(b, g, vals, rhs, f_ext, c, s, e0, e1, &ms))) goto done;
      if (ms >= 0.0 && ms < best.p2_ms) {
        best.p2_ms = ms;
        best.warps = warps;
      }
    }
    cfg.tile = best.tile;
    cfg.p1_blocks_per_sm = best.p1;
    cfg.p2_warps = best.warps;
    cache[key] = best;
    changed = true;
  }
  // leave a complete assembly with the chosen shapes in vals / rhs
  for (Group& g : b->groups) {
    if (launch_group(b, g, vals, rhs, f_ext, s) != cudaSuccess) {
      rc = cuda_err(cudaGetLastError(), "batch assembly");
      goto done;
    }
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) rc = cuda_err(cudaGetLastError(), "tuning");
  if (!rc && changed && !write_cache(cache_path, cache))
    rc = set_err(CXG_ERR_INVALID_ARGUMENT, std::string("cannot write tuning cache ") + cache_path);
done:
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

int cxg_batch_group_config(const cxg_batch* b, int32_t gi, int32_t* type, int32_t* tile, int32_t* p1, int32_t* warps) {
  if (!b || gi < 0 || gi >= static_cast<int32_t>(b->groups.size())) return set_err(CXG_ERR_INVALID_ARGUMENT, "bad group");
  const Group& g = b->groups[static_cast<size_t>(gi)];
  const LaunchCfg& c = g.plan->cfg[b->precision];
  if (b->launch == CXG_BATCH_ONE_LAUNCH) {
    const int pr = b->precision ? 1 : 0;
    if (type) *type = g.type;
    if (tile) *tile = g.ftile[pr];
    if (p1) *p1 = 0;
    if (warps) *warps = b->fwarps[pr];
    return CXG_OK;
  }
  if (type) *type = g.type;
  if (tile) *tile = c.tile;
  if (p1) *p1 = c.p1_blocks_per_sm;
  if (warps) *warps = c.p2_warps;
  return CXG_OK;
}

int cxg_batch_set_group_config(cxg_batch* b, int32_t gi, int32_t tile, int32_t p1, int32_t warps) {
  if (!b || gi < 0 || gi >= static_cast<int32_t>(b->groups.size())) return set_err(CXG_ERR_INVALID_ARGUMENT, "bad group");
  if (tile < 0 || tile > 2 || (tile == 2 && b->precision == CXG_FP64) || p1 < 0 || warps < 0 || warps > 8)
    return set_err(CXG_ERR_INVALID_ARGUMENT, "bad launch shape (4x4 tiles need mixed precision)");
  if (b->launch == CXG_BATCH_ONE_LAUNCH) {
    if (!batch_tile_ok(MODE_LINEAR, b->precision, tile))
      return set_err(CXG_ERR_INVALID_ARGUMENT, "one-launch batch takes 2x2 tiles (and 2x4 in mixed precision)");
    const int pr = b->precision ? 1 : 0;
    b->groups[static_cast<size_t>(gi)].ftile[pr] = tile;
    b->fwarps[pr] = warps;
    return CXG_OK;
  }
  LaunchCfg& c = b->groups[static_cast<size_t>(gi)].plan->cfg[b->precision];
  c.tile = tile;
  c.p1_blocks_per_sm = p1;
  c.p2_warps = warps;
  return CXG_OK;
}

int cxg_batch_assemble_tangent(cxg_batch* b, const double* u, double* vals, double* f_int, double* rhs,
                               const double* f_ext, void* stream) {
  if (!b || !u || !vals) return set_err(CXG_ERR_INVALID_ARGUMENT, "batch, u and vals are required");
  if (!on_device(u) || !on_device(vals) || (f_int && !on_device(f_int)) || (rhs && !on_device(rhs)) ||
      (f_ext && !on_device(f_ext)))
    return set_err(CXG_ERR_INVALID_ARGUMENT, "batched tangent assembly needs device buffers");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (b->launch == CXG_BATCH_ONE_LAUNCH) {
    for (Group& g : b->groups) {
      g.plan->precision = b->precision;
      int rc = ensure_state(g.plan, s);
      if (!rc) rc = ensure_v2(g.plan, true);
      if (rc) return rc;
    }
    std::vector<BatchSlotIn> slots;
    const int rc = fill_slots(b, u, vals, f_int, rhs, f_ext, s, slots);
    if (rc) return rc;
    CHECK_CUDA(launch_one(b, slots, MODE_TANGENT, 3, s), "batch tangent (one launch)");
    return CXG_OK;
  }
  for (Group& g : b->groups) {
    cxg_plan* p = g.plan;
    p->precision = b->precision;
    p->last_stream = s;
    int rc = ensure_state(p, s);
    if (!rc) rc = ensure_v2(p, true);
    if (rc) return rc;
    ElemArgs a = base_args(p);
    a.vals = vals + g.vals0;
    a.rhs = rhs ? rhs + g.rhs0 : nullptr;
    a.f_int = f_int ? f_int + 3 * g.node0 : nullptr;
    a.u = u + 3 * g.node0;
    a.state_c = p->state[0];
    a.state_t = p->state[1];
    a.state_comps = state_comps(p);
    V2Args v = v2_args(p, f_ext ? f_ext + 3 * g.node0 : nullptr, false);
    apply_windows(p, true, v);
    CHECK_CUDA(launch_v2(p->type, MODE_TANGENT, b->precision, a, v, s, p->tcfg[b->precision]), "batch tangent");
  }
  return CXG_OK;
}

int cxg_batch_commit(cxg_batch* b, void* stream) {
  if (!b) return set_err(CXG_ERR_INVALID_ARGUMENT, "null batch");
  for (Group& g : b->groups) {
    const int rc = cxg_state_commit(g.plan, stream);
    if (rc) return rc;
  }
  return CXG_OK;
}

int cxg_batch_get_state(const cxg_batch* b, int32_t k, int32_t slot, double* out) {
  if (!b || k < 0 || k >= static_cast<int32_t>(b->models.size()) || !out || (slot != 0 && slot != 1))
    return set_err(CXG_ERR_INVALID_ARGUMENT, "bad argument");
  const Model& md = b->models[static_cast<size_t>(k)];
  cxg_plan* p = b->groups[static_cast<size_t>(md.group)].plan;
  const size_t nq = static_cast<size_t>(gauss_of(p->type));
  const size_t all = static_cast<size_t>(kStateDoubles) * static_cast<size_t>(p->n_gauss);
  double* tmp = nullptr;
  CHECK_CUDA(cudaMalloc(&tmp, std::max<size_t>(all, 1) * sizeof(double)), "state staging");
  int rc = cxg_state_get(p, slot, tmp);
  if (!rc) {
    const cudaError_t e = cudaMemcpy(out, tmp + kStateDoubles * nq * static_cast<size_t>(md.e0),
                                     sizeof(double) * kStateDoubles * nq * static_cast<size_t>(md.n_elems),
                                     cudaMemcpyDefault);
    if (e != cudaSuccess) rc = cuda_err(e, "state copy");
  }
  cudaFree(tmp);
  return rc;
}

}  // extern "C"
