// The plan object and the host helpers shared by the C-ABI translation units
// (cxg_api.cu: plans and assembly; cxg_batch.cu: batches of plans).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "../../include/cxg.h"
#include "cxg_internal.cuh"

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
  cxg::DevStatus* status = nullptr;
  void* edata = nullptr;      // per-element K blocks of the two-pass assembly
  size_t edata_bytes = 0;
  double* fdata = nullptr;    // per-element internal force (material-point mode)
  cudaStream_t last_stream = nullptr;
  int64_t device_bytes = 0;
  // staging buffers for host pointers, grown on demand and reused
  void* stage[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  size_t stage_bytes[6] = {0, 0, 0, 0, 0, 0};
  cxg::LaunchCfg cfg[2];   // launch shape of the linear passes per precision (FP64, mixed)
  cxg::LaunchCfg tcfg[2];  // launch shape of the material-point (tangent) passes
  bool thermal = false;    // temperature plan: DOF 0 of every node, components 1 and 2 fixed
};


namespace cxg {
namespace api {

int set_err(int code, const std::string& msg);
int cuda_err(cudaError_t e, const char* where);
bool on_device(const void* p);
// Synchronise the plan's last stream and turn an in-kernel error into a status.
int plan_status(cxg_plan* p, int64_t* bad);
// Allocate the per-element buffers of the two-pass assembly.
int ensure_v2(cxg_plan* p, bool tangent);
V2Args v2_args(cxg_plan* p, const double* f_ext, bool accumulate);
ElemArgs base_args(cxg_plan* p);

}  // namespace api
}  // namespace cxg

#define CHECK_CUDA(expr, where)                                 \
  do {                                                          \
    cudaError_t _e = (expr);                                    \
    if (_e != cudaSuccess) return cxg::api::cuda_err(_e, where); \
  } while (0)
